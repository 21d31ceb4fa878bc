"""Seeded procedural scenes (no mesh assets ship with the reference; every mesh is generated).

A SceneDesc is plain arrays; it is turned into a host scene of this library
(xenon_b200.HostScene) or, in the tests, into the reference's own Scene (oracle/ref.py), so
both sides render identical inputs. All geometry is computed in float64 and rounded to float32
once, so a given seed gives the same bytes on every machine.

  cornell(...)          config 1: Cornell-style box, 5 wall quads, 2 rotated boxes, ceiling light
  icosphere_scene(...)  config 2: displaced icosphere (GGX conductor) on a ground quad, sun + sky
  prim_showcase(...)    the five analytic primitives (sphere, box, disk, quad, plane) + sky
  instanced_grid(...)   config 3 style: TLAS over transformed instances of procedural meshes
  guiding_room(...)     config 4: closed room, small light behind a baffle, glass sphere
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class MeshDesc:
    positions: np.ndarray                 # (N, 3) float32
    indices: np.ndarray                   # (M, 3) int32
    normals: np.ndarray | None = None     # (N, 3) float32; None → area-weighted smooth normals
    mat_ids: np.ndarray | None = None     # (M,) int32; None → default_mat
    default_mat: int = 0
    transform: tuple | None = None        # (translation, scale, rot_deg) baked into vertices


@dataclass
class SceneDesc:
    materials: list = field(default_factory=list)      # float32[21] xb_material each
    material_names: list = field(default_factory=list)
    meshes: list = field(default_factory=list)
    prims: list = field(default_factory=list)          # PRIM_DTYPE arrays of length 1
    lights: list = field(default_factory=list)         # (mesh_id, tri_idx, emission3, area)
    suns: list = field(default_factory=list)           # (direction3, color3, intensity)
    sky: np.ndarray = field(default_factory=lambda: sky_array())
    instances: list = field(default_factory=list)      # (geom, translation3, scale, rot3, id)
    eye: tuple = (0.0, 5.0, 20.0)
    target: tuple = (0.0, 5.0, 0.0)
    fov: float = 40.0
    width: int = 800
    height: int = 600
    spp: int = 64
    min_bounces: int = 3
    max_bounces: int = 8
    name: str = "scene"

    def add_material(self, name: str, m: np.ndarray) -> int:
        self.materials.append(np.asarray(m, np.float32))
        self.material_names.append(name)
        return len(self.materials) - 1

    def add_mesh(self, mesh: MeshDesc) -> int:
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    @property
    def num_triangles(self) -> int:
        return sum(len(m.indices) for m in self.meshes)


def sky_array(zenith=(0.10, 0.30, 0.80), horizon=(0.55, 0.70, 0.85), ground=(0.10, 0.08, 0.05),
              sharpness=3.0, intensity=1.0) -> np.ndarray:
    """xb_sky as float32[11]; defaults are Environment's (src/scene/environment.h:15-19)."""
    return np.array(list(zenith) + list(horizon) + list(ground) + [sharpness, intensity], np.float32)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float64).astype(np.float32))


def quad_mesh(origin, u, v, mat: int) -> MeshDesc:
    """Parallelogram origin + s*u + t*v as two triangles, geometric normal along u x v."""
    o, u, v = (np.asarray(x, np.float64) for x in (origin, u, v))
    pos = np.stack([o, o + u, o + u + v, o + v])
    n = np.cross(u, v)
    n /= np.linalg.norm(n)
    return MeshDesc(f32(pos), np.array([[0, 1, 2], [0, 2, 3]], np.int32), f32(np.tile(n, (4, 1))),
                    None, mat)


def _rot_y(deg: float) -> np.ndarray:
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def box_mesh(center, size, rot_y_deg: float, mat: int) -> MeshDesc:
    """Axis-aligned box rotated about y; 24 vertices so every face has a flat normal."""
    c = np.asarray(center, np.float64)
    h = np.asarray(size, np.float64) / 2
    R = _rot_y(rot_y_deg)
    faces = []  # (normal axis, sign)
    pos, nrm, idx = [], [], []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = sgn
            a1, a2 = (axis + 1) % 3, (axis + 2) % 3
            e1 = np.zeros(3); e1[a1] = 1.0
            e2 = np.zeros(3); e2[a2] = 1.0
            if sgn < 0:
                e1, e2 = e2, e1
            corners = [n * h + (-e1 - e2) * h, n * h + (e1 - e2) * h, n * h + (e1 + e2) * h,
                       n * h + (-e1 + e2) * h]
            base = len(pos)
            for q in corners:
                pos.append(c + R @ q)
                nrm.append(R @ n)
            idx += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
            faces.append((axis, sgn))
    return MeshDesc(f32(pos), np.array(idx, np.int32), f32(nrm), None, mat)


# ── config 1 ────────────────────────────────────────────────────────────────────
def cornell(width: int = 256, height: int = 256, spp: int = 64, max_bounces: int = 8,
            min_bounces: int = 3) -> SceneDesc:
    """Config 1: 10x10x10 box open at +z, walls as two-triangle quads facing inward, a 3x3x3
    box rotated 18 deg and a 3x6x3 box rotated -15 deg, a 2.5x2.5 ceiling light with emission
    (17,12,4) (two `light` triangles with their true areas), sky off, pinhole at fov 40."""
    d = SceneDesc(name="cornell", width=width, height=height, spp=spp, min_bounces=min_bounces,
                  max_bounces=max_bounces)
    white = d.add_material("white", abi.material(base_color=(0.73, 0.73, 0.73), roughness=1.0))
    red = d.add_material("left", abi.material(base_color=(0.63, 0.065, 0.05), roughness=1.0))
    green = d.add_material("right", abi.material(base_color=(0.14, 0.45, 0.09), roughness=1.0))
    lightm = d.add_material("light", abi.material(base_color=(0.78, 0.78, 0.78), roughness=1.0,
                                                  emission=(17.0, 12.0, 4.0)))
    L = 10.0
    # box spans x,z in [-5, 5], y in [0, 10]; normals point inward
    d.add_mesh(quad_mesh((-5, 0, 5), (L, 0, 0), (0, 0, -L), white))       # floor   n=+y
    d.add_mesh(quad_mesh((-5, L, -5), (L, 0, 0), (0, 0, L), white))       # ceiling n=-y
    d.add_mesh(quad_mesh((-5, 0, -5), (L, 0, 0), (0, L, 0), white))       # back    n=+z
    d.add_mesh(quad_mesh((-5, 0, 5), (0, 0, -L), (0, L, 0), red))         # left    n=+x
    d.add_mesh(quad_mesh((5, 0, -5), (0, 0, L), (0, L, 0), green))        # right   n=-x
    d.add_mesh(box_mesh((1.6, 1.5, 1.2), (3, 3, 3), 18.0, white))
    d.add_mesh(box_mesh((-1.7, 3.0, -1.5), (3, 6, 3), -15.0, white))
    s = 2.5
    lm = d.add_mesh(quad_mesh((-s / 2, L - 0.01, -s / 2), (s, 0, 0), (0, 0, s), lightm))  # n=-y
    area = s * s / 2
    for tri in (0, 1):
        d.lights.append((lm, tri, (17.0, 12.0, 4.0), area))
    d.sky = sky_array(zenith=(0, 0, 0), horizon=(0, 0, 0), ground=(0, 0, 0), sharpness=3.0, intensity=0.0)
    d.eye, d.target, d.fov = (0.0, 5.0, 18.7), (0.0, 5.0, 0.0), 40.0
    return d


# ── procedural meshes ───────────────────────────────────────────────────────────
def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**level triangles (level 8: 1,310,720), outward winding."""
    t = (1.0 + 5 ** 0.5) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (len(v) + 1), uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mids = inv.reshape(3, -1).T + len(v)
        v = np.concatenate([v, mid])
        i0, i1, i2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = mids[:, 0], mids[:, 1], mids[:, 2]
        f = np.concatenate([np.stack([i0, m01, m20], 1), np.stack([i1, m12, m01], 1),
                            np.stack([i2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f.astype(np.int32)


def geodesic_sphere(freq: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit geodesic sphere: every face of the icosahedron split into freq x freq triangles on a
    barycentric grid, the points projected onto the sphere; 20 * freq**2 triangles (freq 158:
    499,280), outward winding, closed (vertices on the icosahedron's edges are shared)."""
    n = int(freq)
    if n < 1:
        raise ValueError("geodesic_sphere: freq >= 1")
    v0, f0 = icosphere(0)
    edges = {}
    pts = [v0]
    count = len(v0)
    for a, b, c in f0:
        for p, q in ((a, b), (b, c), (a, c)):
            key = (min(p, q), max(p, q))
            if key not in edges and n > 1:
                k = np.arange(1, n)[:, None] / n
                pts.append(v0[key[0]] + (v0[key[1]] - v0[key[0]]) * k)
                edges[key] = count
                count += n - 1

    def edge_point(p, q, k):
        """Vertex index of the point k/n of the way from corner p to corner q (0 < k < n)."""
        if p < q:
            return edges[(p, q)] + k - 1
        return edges[(q, p)] + (n - k) - 1

    tris = []
    for a, b, c in f0:
        idx = {}
        for i in range(n + 1):
            for j in range(n + 1 - i):
                if i == 0 and j == 0:
                    idx[i, j] = a
                elif i == n:
                    idx[i, j] = b
                elif j == n:
                    idx[i, j] = c
                elif j == 0:
                    idx[i, j] = edge_point(a, b, i)
                elif i == 0:
                    idx[i, j] = edge_point(a, c, j)
                elif i + j == n:
                    idx[i, j] = edge_point(b, c, j)
        inner = [(i, j) for i in range(1, n) for j in range(1, n - i)]
        if inner:
            ij = np.array(inner, np.float64)
            pts.append(v0[a] + (v0[b] - v0[a]) * ij[:, :1] / n + (v0[c] - v0[a]) * ij[:, 1:] / n)
            for k, key in enumerate(inner):
                idx[key] = count + k
            count += len(inner)
        for i in range(n):
            for j in range(n - i):
                tris.append((idx[i, j], idx[i + 1, j], idx[i, j + 1]))
                if i + j < n - 1:
                    tris.append((idx[i + 1, j], idx[i + 1, j + 1], idx[i, j + 1]))
    v = np.concatenate(pts)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, np.array(tris, np.int32)


def value_noise(p: np.ndarray, seed: int, octaves: int = 4, base_freq: float = 1.5) -> np.ndarray:
    """Seeded lattice value noise in [-1, 1]: smoothstep-trilinear, `octaves` octaves with
    doubling frequency and halving amplitude, normalised by the amplitude sum."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256)
    perm = np.concatenate([perm, perm])
    vals = rng.uniform(-1.0, 1.0, 256)

    def lattice(ix, iy, iz):
        return vals[perm[perm[perm[ix & 255] + (iy & 255)] + (iz & 255)]]

    total = np.zeros(len(p))
    amp, freq, norm = 1.0, base_freq, 0.0
    for _ in range(octaves):
        q = p * freq + 17.0
        i = np.floor(q).astype(np.int64)
        fr = q - i
        s = fr * fr * (3 - 2 * fr)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = (s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) * \
                        (s[:, 2] if dz else 1 - s[:, 2])
                    acc += w * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def displaced_icosphere(level: int, radius: float, center, seed: int, amplitude: float = 0.15):
    v, f = icosphere(level)
    disp = value_noise(v, seed) * amplitude * radius
    pos = np.asarray(center, np.float64) + v * (radius + disp)[:, None]
    return pos, f


# ── config 2 ────────────────────────────────────────────────────────────────────
def icosphere_scene(level: int = 8, width: int = 1920, height: int = 1080, spp: int = 256,
                    max_bounces: int = 10, min_bounces: int = 3, seed: int = 1) -> SceneDesc:
    """Config 2: icosphere (level 8 = 1,310,720 tris) displaced along its normals by 4-octave
    value noise of amplitude 0.15 r; GGX conductor roughness 0.3, F0 (0.95, 0.64, 0.54)
    (metallic 1, baseColor = F0); 50x50 diffuse ground quad, albedo 0.5; directional sun of
    intensity 3.0 and the gradient sky. Sphere and ground are one mesh: a single BLAS."""
    d = SceneDesc(name=f"icosphere_l{level}", width=width, height=height, spp=spp,
                  min_bounces=min_bounces, max_bounces=max_bounces)
    metal = d.add_material("copper", abi.material(base_color=(0.95, 0.64, 0.54), metallic=1.0, roughness=0.3))
    ground = d.add_material("ground", abi.material(base_color=(0.5, 0.5, 0.5), roughness=1.0))
    r = 2.0
    pos, f = displaced_icosphere(level, r, (0.0, r * 1.15, 0.0), seed)
    g = 25.0
    gpos = np.array([[-g, 0, g], [g, 0, g], [g, 0, -g], [-g, 0, -g]], np.float64)
    gf = np.array([[0, 1, 2], [0, 2, 3]], np.int32) + len(pos)
    allpos = np.concatenate([pos, gpos])
    allf = np.concatenate([f, gf]).astype(np.int32)
    mats = np.concatenate([np.full(len(f), metal, np.int32), np.full(2, ground, np.int32)])
    d.add_mesh(MeshDesc(f32(allpos), allf, None, mats, metal))
    d.suns.append(((-0.5, 0.8, 0.3), (1.0, 0.97, 0.88), 3.0))
    d.sky = sky_array()
    d.eye, d.target, d.fov = (0.0, 3.2, 9.5), (0.0, 2.2, 0.0), 40.0
    return d


# ── analytic primitives ─────────────────────────────────────────────────────────
def prim_showcase(width: int = 160, height: int = 120, spp: int = 8, max_bounces: int = 8) -> SceneDesc:
    """Sphere, box, disk, quad and plane with sky light (the reference's prim_types layout)."""
    d = SceneDesc(name="prims", width=width, height=height, spp=spp, max_bounces=max_bounces)
    m_plane = d.add_material("plane", abi.material(base_color=(0.72, 0.70, 0.68), roughness=0.8))
    m_sph = d.add_material("sphere", abi.material(base_color=(0.85, 0.12, 0.08), roughness=0.3))
    m_box = d.add_material("box", abi.material(base_color=(0.10, 0.45, 0.80), roughness=0.5))
    m_disk = d.add_material("disk", abi.material(base_color=(0.90, 0.75, 0.10), roughness=0.4))
    m_quad = d.add_material("quad", abi.material(base_color=(0.15, 0.80, 0.25), roughness=0.5))
    m_met = d.add_material("metal", abi.material(base_color=(0.9, 0.9, 0.9), metallic=1.0, roughness=0.05))
    m_glass = d.add_material("glass", abi.material(base_color=(0.95, 0.95, 0.95), roughness=0.0,
                                                   transmission=1.0, ior=1.45))
    n = np.array([0.0, 0.5, 1.0]); n /= np.linalg.norm(n)
    d.prims += [abi.prim(abi.XB_PRIM_PLANE, m_plane, 0, 1, 0, 0.0),
                abi.prim(abi.XB_PRIM_SPHERE, m_sph, -7.0, 1.4, 0.0, 1.4),
                abi.prim(abi.XB_PRIM_BOX, m_box, -3.5, 1.2, 0.0, 1.2, 1.2, 1.2),
                abi.prim(abi.XB_PRIM_DISK, m_disk, 0.0, 1.8, 0.5, *n.astype(np.float32), 1.3),
                abi.prim(abi.XB_PRIM_QUAD, m_quad, 2.8, 0.0, -0.8, 2.4, 0.0, 0.0, 0.0, 2.8, -0.8),
                abi.prim(abi.XB_PRIM_BOX, m_met, 7.0, 0.5, 0.0, 1.6, 0.5, 1.0),
                abi.prim(abi.XB_PRIM_SPHERE, m_glass, 0.0, 0.8, 3.0, 0.8)]
    d.sky = sky_array((0.15, 0.25, 0.55), (0.65, 0.72, 0.80), (0.15, 0.12, 0.10), 3.0, 0.8)
    d.eye, d.target, d.fov = (0.0, 5.0, 20.0), (0.0, 2.0, 0.0), 50.0
    return d


def lumpy_mesh(level: int, seed: int, amplitude: float = 0.25) -> MeshDesc:
    pos, f = displaced_icosphere(level, 1.0, (0, 0, 0), seed, amplitude)
    return MeshDesc(f32(pos), f, None, None, 0)


# ── config 3 style ──────────────────────────────────────────────────────────────
def instanced_grid(grid: int = 16, levels=(6, 6, 7, 7), width: int = 1920, height: int = 1080,
                   spp: int = 512, max_bounces: int = 12, seed: int = 3, with_prims: bool = False) -> SceneDesc:
    """TLAS over a grid x grid field of instances of 4 seeded procedural meshes (levels 6-7:
    82k-328k tris at full size). Each instance: random rotation, scale U[0.5, 1.5], +-0.2
    jitter. The reference has no per-instance material, so each base mesh comes in three
    material variants (diffuse albedo U[0.2, 0.8], conductor roughness U[0.05, 0.5],
    dielectric IOR 1.5 roughness U[0, 0.2]); an instance picks one of the 12 at random.
    Lighting: the sky plus 4 emissive quads (one identity instance each)."""
    rng = np.random.default_rng(seed)
    d = SceneDesc(name=f"instanced_{grid}x{grid}", width=width, height=height, spp=spp,
                  max_bounces=max_bounces)
    variants = []
    for mi, lv in enumerate(levels):
        base = lumpy_mesh(lv, seed * 100 + mi)
        for kind in range(3):
            if kind == 0:
                m = abi.material(base_color=tuple(rng.uniform(0.2, 0.8, 3)), roughness=1.0)
            elif kind == 1:
                m = abi.material(base_color=tuple(rng.uniform(0.5, 0.95, 3)), metallic=1.0,
                                 roughness=float(rng.uniform(0.05, 0.5)))
            else:
                m = abi.material(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5,
                                 roughness=float(rng.uniform(0.0, 0.2)))
            mat = d.add_material(f"m{mi}_{kind}", m)
            variants.append(d.add_mesh(MeshDesc(base.positions, base.indices, None, None, mat)))
    lightm = d.add_material("light", abi.material(base_color=(0.8, 0.8, 0.8), emission=(6.0, 6.0, 6.0)))
    ground = d.add_material("ground", abi.material(base_color=(0.5, 0.5, 0.5), roughness=1.0))
    spacing = 4.0
    ext = grid * spacing / 2 + 2.0
    gm = d.add_mesh(quad_mesh((-ext, -2.2, ext), (2 * ext, 0, 0), (0, 0, -2 * ext), ground))
    lights = []
    for k in range(4):
        cx, cz = (-ext / 2 if k % 2 == 0 else ext / 2), (-ext / 2 if k < 2 else ext / 2)
        s = 3.0
        lm = d.add_mesh(quad_mesh((cx - s / 2, 8.0, cz - s / 2), (s, 0, 0), (0, 0, s), lightm))
        lights.append(lm)
        for tri in (0, 1):
            d.lights.append((lm, tri, (6.0, 6.0, 6.0), s * s / 2))
    # identity instances for ground and lights carry their mesh index as instance id, so each
    # `light` entry (mesh_id, tri_idx) matches the hits on its own quad
    d.instances.append((gm, (0, 0, 0), 1.0, (0, 0, 0), gm))
    for lm in lights:
        d.instances.append((lm, (0, 0, 0), 1.0, (0, 0, 0), lm))
    iid = len(d.meshes)
    for gx in range(grid):
        for gz in range(grid):
            v = int(rng.integers(len(variants)))
            t = ((gx - (grid - 1) / 2) * spacing + rng.uniform(-0.2, 0.2), rng.uniform(-0.2, 0.2),
                 (gz - (grid - 1) / 2) * spacing + rng.uniform(-0.2, 0.2))
            s = float(rng.uniform(0.5, 1.5))
            rot = tuple(rng.uniform(0, 360, 3))
            d.instances.append((variants[v], t, s, rot, iid))
            iid += 1
    if with_prims:
        m = d.add_material("psphere", abi.material(base_color=(0.9, 0.2, 0.2), roughness=0.4))
        d.prims.append(abi.prim(abi.XB_PRIM_SPHERE, m, 0.0, 3.0, 0.0, 1.0))
        d.prims.append(abi.prim(abi.XB_PRIM_BOX, m, 4.0, 2.0, 1.0, 0.6, 0.8, 0.5))
        d.instances.append((abi.XB_GEOM_PRIMS, (0, 0, 0), 1.0, (0, 0, 0), iid))
    d.sky = sky_array()
    d.eye, d.target, d.fov = (0.0, ext * 0.6, ext * 1.1), (0.0, -1.0, 0.0), 45.0
    return d


# ── config 4 ────────────────────────────────────────────────────────────────────
def guiding_room(level: int | None = None, width: int = 1280, height: int = 720, max_bounces: int = 16,
                 spp: int = 64, freq: int = 158) -> SceneDesc:
    """Config 4: closed 10x10x10 diffuse room (albedo 0.7), the only light an emissive quad of
    0.5 units^2 (0.5 % of the ceiling) hidden above a diffuse baffle, and a smooth glass sphere
    mesh (IOR 1.5, roughness 0 → delta). By default the sphere is the geodesic sphere of
    frequency 158: 499,280 tris, the configuration's 500k; `level` instead takes the icosphere of
    that level (20 * 4**level tris: level 7 = 327,680), for smaller test scenes.
    The walls have IOR 1 (F0 = 0): a purely Lambertian BSDF whose sampled and evaluated forms
    agree, so the guided and the plain estimator converge to the same image."""
    d = SceneDesc(name="guiding_room", width=width, height=height, spp=spp, max_bounces=max_bounces)
    wall = d.add_material("wall", abi.material(base_color=(0.7, 0.7, 0.7), roughness=1.0, ior=1.0))
    glass = d.add_material("glass", abi.material(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.5,
                                                 roughness=0.0))
    lightm = d.add_material("light", abi.material(base_color=(0.8, 0.8, 0.8), emission=(400.0, 380.0, 340.0)))
    L = 10.0
    d.add_mesh(quad_mesh((-5, 0, 5), (L, 0, 0), (0, 0, -L), wall))       # floor   n=+y
    d.add_mesh(quad_mesh((-5, L, -5), (L, 0, 0), (0, 0, L), wall))       # ceiling n=-y
    d.add_mesh(quad_mesh((-5, 0, -5), (L, 0, 0), (0, L, 0), wall))       # back    n=+z
    d.add_mesh(quad_mesh((-5, 0, 5), (0, 0, -L), (0, L, 0), wall))       # left    n=+x
    d.add_mesh(quad_mesh((5, 0, -5), (0, 0, L), (0, L, 0), wall))        # right   n=-x
    d.add_mesh(quad_mesh((5, 0, 5), (-L, 0, 0), (0, L, 0), wall))        # front   n=-z
    # baffle: horizontal panel under the light, both sides facing out
    d.add_mesh(quad_mesh((2.0, 8.5, -4.0), (2.8, 0, 0), (0, 0, 3.0), wall))   # n=-y (faces the room)
    d.add_mesh(quad_mesh((2.0, 8.52, -4.0), (0, 0, 3.0), (2.8, 0, 0), wall))  # n=+y (faces the light)
    s = 0.5 ** 0.5
    lm = d.add_mesh(quad_mesh((3.4 - s / 2, L - 0.01, -2.5 - s / 2), (s, 0, 0), (0, 0, s), lightm))
    for tri in (0, 1):
        d.lights.append((lm, tri, (400.0, 380.0, 340.0), s * s / 2))
    if level is None:
        v, f = geodesic_sphere(freq)
        pos = np.asarray((-1.0, 1.6, -0.5), np.float64) + v * 1.6
    else:
        pos, f = displaced_icosphere(level, 1.6, (-1.0, 1.6, -0.5), 7, amplitude=0.0)
    d.add_mesh(MeshDesc(f32(pos), f, None, None, glass))
    d.sky = sky_array(intensity=0.0)
    d.eye, d.target, d.fov = (0.0, 5.0, 4.8), (0.0, 3.5, -5.0), 60.0
    return d


def random_rays(desc_bounds: tuple, n: int, seed: int, tmin: float = 1e-4) -> np.ndarray:
    """Incoherent rays: origins uniform in the box, directions uniform on the sphere."""
    lo, hi = (np.asarray(b, np.float64) for b in desc_bounds)
    rng = np.random.default_rng(seed)
    org = lo + (hi - lo) * rng.random((n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return abi.make_rays(f32(org), f32(d), tmin=tmin)


def scene_bounds(desc: SceneDesc) -> tuple:
    pts = [m.positions for m in desc.meshes]
    allp = np.concatenate(pts) if pts else np.zeros((1, 3), np.float32)
    return allp.min(0), allp.max(0)


# ── config 5 ────────────────────────────────────────────────────────────────────
VIEW_SIZES = (256, 512, 768, 1024)
VIEW_SPP = (16, 64, 256, 1024)


def orbit_views(desc: SceneDesc, n: int = 32, seed: int = 1, sizes=VIEW_SIZES, spps=VIEW_SPP) -> list:
    """Config 5: n cameras from the seed, looking at the scene's centre from random directions on
    the upper hemisphere at 1.2-2.0 scene radii; square images of a size from `sizes` and a
    sample count from `spps`. Returns [(eye, target, fov, width, height, spp), ...]."""
    lo, hi = scene_bounds(desc)
    c = (lo + hi) / 2
    rad = float(np.linalg.norm(hi - lo)) / 2
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = rng.normal(size=3)
        d[1] = abs(d[1]) + 0.2
        d /= np.linalg.norm(d)
        eye = c + d * rad * rng.uniform(1.2, 2.0)
        s = int(rng.choice(sizes))
        out.append((tuple(float(x) for x in eye), tuple(float(x) for x in c), 40.0, s, s, int(rng.choice(spps))))
    return out


def config5_views(desc: SceneDesc, n: int = 32, seed: int = 1, max_spp: int | None = None) -> list:
    """Config 5: n square views of the scene from the seed — side log-uniform in [256, 1024] px,
    spp from {16, 64, 256, 1024} (capped at max_spp when given), bounce limit uniform in 6..16 —
    looking at the scene's centre from the upper hemisphere at 0.6-1.2 scene radii.
    Returns [(eye, target, fov, width, height, spp, max_bounces), ...]."""
    lo, hi = scene_bounds(desc)
    c = (lo + hi) / 2
    rad = float(np.linalg.norm(hi - lo)) / 2
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = rng.normal(size=3)
        d[1] = abs(d[1]) + 0.3
        d /= np.linalg.norm(d)
        eye = c + d * rad * rng.uniform(0.6, 1.2)
        side = int(round(float(np.exp(rng.uniform(np.log(256), np.log(1024))))))
        spp = int(rng.choice(VIEW_SPP))
        if max_spp:
            spp = min(spp, max_spp)
        out.append((tuple(float(x) for x in eye), tuple(float(x) for x in c), 45.0, side, side, spp,
                    int(rng.integers(6, 17))))
    return out
