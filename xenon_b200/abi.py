"""Python mirrors of the POD structs in include/xenon_b200.h (numpy dtypes and ctypes)."""
from __future__ import annotations

import ctypes

import numpy as np

# ── status codes ──────────────────────────────────────────────────────────────
XB_OK = 0
XB_E_INVALID = -1
XB_E_CUDA = -2
XB_E_OOM = -3
XB_E_STATE = -4
XB_E_IO = -5
XB_E_OVERFLOW = -6
XB_E_TIMEOUT = -7
XB_E_UNSUPPORTED = -8
STATUS_NAMES = {0: "XB_OK", -1: "XB_E_INVALID", -2: "XB_E_CUDA", -3: "XB_E_OOM", -4: "XB_E_STATE",
                -5: "XB_E_IO", -6: "XB_E_OVERFLOW", -7: "XB_E_TIMEOUT", -8: "XB_E_UNSUPPORTED"}

XB_PRIM_SPHERE, XB_PRIM_PLANE, XB_PRIM_BOX, XB_PRIM_DISK, XB_PRIM_QUAD = range(5)
XB_GEOM_PRIMS = -1
XB_BUILD_RECURSIVE, XB_BUILD_LEVELS, XB_BUILD_DEVICE = 0, 1, 2
XB_TRACE_CLOSEST, XB_TRACE_ANY = 0, 1
XB_FLAG_FP64_ACCUM = 1
XB_FLAG_THREAD_PER_RAY = 2
XB_FLAG_SUN_NEE = 4
XB_FLAG_SKY_IS = 8
XB_FLAG_WATERTIGHT = 16
XB_MAT_CONDUCTOR, XB_MAT_TRANSMISSIVE, XB_MAT_SUBSURFACE, XB_MAT_DELTA, XB_MAT_EMISSIVE = 1, 2, 4, 8, 16

# xb_material: 22 floats, field order of the C struct
MATERIAL_FIELDS = {
    "base_color": slice(0, 3), "roughness": 3, "metallic": 4, "ior": 5, "transmission": 6,
    "subsurface": 7, "subsurface_color": slice(8, 11), "anisotropy": 11, "emission": slice(12, 15),
    "subsurface_mfp": slice(15, 18), "clearcoat": 18, "clearcoat_roughness": 19,
    "emission_temperature": 20,
}
MATERIAL_FLOATS = 21


def material(**kw) -> np.ndarray:
    """xb_material as float32[21] with the reference defaults (src/material/material.h:23-35)."""
    m = np.zeros(MATERIAL_FLOATS, np.float32)
    m[0:3] = 0.5
    m[3] = 0.5
    m[5] = 1.5
    m[8:11] = 1.0
    m[15:18] = 1.0
    m[19] = 0.03
    m[20] = 6500.0
    for k, v in kw.items():
        m[MATERIAL_FIELDS[k]] = v
    return m


PRIM_DTYPE = np.dtype([("type", np.int32), ("mat_id", np.int32), ("p", np.float32, 10)])
RAY_DTYPE = np.dtype([("org", np.float32, 3), ("tmin", np.float32), ("dir", np.float32, 3),
                      ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32), ("prim_id", np.int32),
                      ("instance_id", np.int32), ("mat_id", np.int32), ("front_face", np.int32),
                      ("pos", np.float32, 3), ("normal", np.float32, 3), ("geo_normal", np.float32, 3)])
NODE_DTYPE = np.dtype([("mn", np.float32, 3), ("mx", np.float32, 3), ("child", np.uint32),
                       ("count", np.uint32)])
assert PRIM_DTYPE.itemsize == 48 and RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 64
assert NODE_DTYPE.itemsize == 32


def prim(type_: int, mat_id: int, *params) -> np.ndarray:
    p = np.zeros(1, PRIM_DTYPE)
    p["type"] = type_
    p["mat_id"] = mat_id
    p["p"][0, :len(params)] = params
    return p


def make_rays(org: np.ndarray, dirs: np.ndarray, tmin=1e-4, tmax=np.inf) -> np.ndarray:
    r = np.zeros(len(org), RAY_DTYPE)
    r["org"] = org
    r["dir"] = dirs
    r["tmin"] = tmin
    r["tmax"] = tmax
    return r


# ── ctypes structures (for passing views between libraries) ───────────────────
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)
_up = ctypes.POINTER(ctypes.c_uint32)


class MeshView(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_int32), ("num_triangles", ctypes.c_int32),
                ("vx", _fp), ("vy", _fp), ("vz", _fp), ("nx", _fp), ("ny", _fp), ("nz", _fp),
                ("indices", _ip), ("mat_ids", _ip), ("blas_nodes", ctypes.c_void_p),
                ("num_blas_nodes", ctypes.c_int32), ("blas_prims", _up)]


class InstanceView(ctypes.Structure):
    _fields_ = [("geom", ctypes.c_int32), ("instance_id", ctypes.c_int32),
                ("local_to_world", ctypes.c_float * 12), ("world_to_local", ctypes.c_float * 12)]


class Sky(ctypes.Structure):
    _fields_ = [("zenith", ctypes.c_float * 3), ("horizon", ctypes.c_float * 3),
                ("ground", ctypes.c_float * 3), ("sharpness", ctypes.c_float),
                ("intensity", ctypes.c_float)]


class SceneView(ctypes.Structure):
    _fields_ = [("num_meshes", ctypes.c_int32), ("meshes", ctypes.POINTER(MeshView)),
                ("num_prims", ctypes.c_int32), ("prims", ctypes.c_void_p),
                ("prim_nodes", ctypes.c_void_p), ("num_prim_nodes", ctypes.c_int32),
                ("prim_indices", _up),
                ("num_instances", ctypes.c_int32), ("instances", ctypes.POINTER(InstanceView)),
                ("tlas_nodes", ctypes.c_void_p), ("num_tlas_nodes", ctypes.c_int32),
                ("tlas_inst_indices", _up),
                ("num_materials", ctypes.c_int32), ("materials", ctypes.c_void_p),
                ("num_lights", ctypes.c_int32), ("lights", ctypes.c_void_p),
                ("num_suns", ctypes.c_int32), ("suns", ctypes.c_void_p),
                ("sky", Sky)]


class Camera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("lower_left", ctypes.c_float * 3),
                ("horizontal", ctypes.c_float * 3), ("vertical", ctypes.c_float * 3)]

    @staticmethod
    def from_array(a) -> "Camera":
        c = Camera()
        a = np.asarray(a, np.float32).reshape(12)
        for i, f in enumerate(("eye", "lower_left", "horizontal", "vertical")):
            getattr(c, f)[:] = [float(x) for x in a[3 * i:3 * i + 3]]
        return c

    def to_array(self) -> np.ndarray:
        return np.array(list(self.eye) + list(self.lower_left) + list(self.horizontal) +
                        list(self.vertical), np.float32)


class Config(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("max_bounces", ctypes.c_int32), ("min_bounces", ctypes.c_int32),
                ("device", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("wave_paths", ctypes.c_int32), ("block_size", ctypes.c_int32)]


class RenderStats(ctypes.Structure):
    _fields_ = [("rays_closest", ctypes.c_int64), ("rays_shadow", ctypes.c_int64),
                ("paths", ctypes.c_int64), ("overflow", ctypes.c_int64), ("last_ms", ctypes.c_float),
                ("nonfinite", ctypes.c_int64)]


XB_PROFILE_STAGE_TIMES, XB_PROFILE_COUNT_TRAVERSAL = 1, 2


class Tuning(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("extend_persistent_from_depth", "shadow_persistent", "refill",
                                              "extend_blocks_per_sm", "shadow_blocks_per_sm",
                                              "shade_blocks_per_sm", "wave_paths", "shadow_order", "overlap",
                                              "waves", "lane_stagger", "graph", "guided_form",
                                              "shade_occupancy", "shared_stack", "pixel_order")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Profile(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("raygen_ms", "extend_ms", "shade_ms", "shadow_ms",
                                               "accumulate_ms")] + \
               [(k, ctypes.c_int64) for k in ("raygen_launches", "extend_launches", "shade_launches",
                                              "shadow_launches", "accumulate_launches",
                                              "ext_blas_nodes", "ext_tris", "ext_tlas_nodes", "ext_instances",
                                              "sh_blas_nodes", "sh_tris", "sh_tlas_nodes", "sh_instances")] + \
               [("train_ms", ctypes.c_double), ("train_launches", ctypes.c_int64)] + \
               [(k, ctypes.c_double) for k in ("extend_busy_ms", "shade_busy_ms", "shadow_busy_ms")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


GUIDE_PARAMS = 15600        # XB_GUIDE_PARAMS
GUIDE_LOBE_FLOATS = 40
GUIDE_OUT_FLOATS = 41
GUIDE_RECORD_FLOATS = 24


class Guiding(ctypes.Structure):
    """xb_guiding: learned path guiding (0 fields take their defaults)."""
    _fields_ = [("enabled", ctypes.c_int32), ("train_spp", ctypes.c_int32), ("steps_per_spp", ctypes.c_int32),
                ("batch", ctypes.c_int32), ("learning_rate", ctypes.c_float), ("guide_fraction", ctypes.c_float),
                ("max_records", ctypes.c_int32), ("record_stride", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("bounds_min", ctypes.c_float * 3), ("bounds_max", ctypes.c_float * 3),
                ("keep_training_samples", ctypes.c_int32), ("fixed_fraction", ctypes.c_int32),
                ("guided_bounces", ctypes.c_int32), ("ratio_cap", ctypes.c_float)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["bounds_min"] = list(self.bounds_min)
        d["bounds_max"] = list(self.bounds_max)
        return d


class NoiseStats(ctypes.Structure):
    """xb_noise_stats: the reference's blur-residual noise statistics of an image."""
    _fields_ = [(k, ctypes.c_float) for k in ("mean_squared_score", "rms_score", "mean_absolute",
                                              "median_absolute", "p95_absolute", "max_absolute",
                                              "avg_luminance", "edge_threshold", "epsilon")] + \
               [("valid_pixel_count", ctypes.c_int32), ("total_interior_pixel_count", ctypes.c_int32),
                ("valid_pixel_ratio", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GuidingStats(ctypes.Structure):
    _fields_ = [("adam_steps", ctypes.c_int64), ("records", ctypes.c_int64), ("records_dropped", ctypes.c_int64),
                ("last_loss", ctypes.c_float), ("training", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SceneConfig(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("samples", ctypes.c_int32),
                ("min_bounces", ctypes.c_int32), ("max_bounces", ctypes.c_int32)]


class View(ctypes.Structure):
    """xb_view: one camera of xb_render_views and its host output buffer."""
    _fields_ = [("camera", Camera), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("spp", ctypes.c_int32), ("max_bounces", ctypes.c_int32), ("out_rgb", ctypes.c_void_p)]


assert ctypes.sizeof(View) == 72


class CameraDesc(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("target", ctypes.c_float * 3), ("fov_y_deg", ctypes.c_float)]


class MaterialDerived(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_float), ("alpha_x", ctypes.c_float), ("alpha_y", ctypes.c_float),
                ("f0", ctypes.c_float * 3), ("flags", ctypes.c_int32)]


def view_arrays(v: SceneView) -> dict:
    """Copies the arrays behind an xb_scene_view into numpy (for comparing two builds)."""
    out = {"meshes": []}
    for i in range(v.num_meshes):
        mv = v.meshes[i]
        nn = mv.num_blas_nodes
        nodes = np.frombuffer((ctypes.c_char * (nn * 32)).from_address(mv.blas_nodes), NODE_DTYPE).copy() if nn else np.zeros(0, NODE_DTYPE)
        prims = np.ctypeslib.as_array(mv.blas_prims, (mv.num_triangles,)).copy() if mv.num_triangles else np.zeros(0, np.uint32)
        nv = mv.num_vertices
        pos = np.stack([np.ctypeslib.as_array(getattr(mv, k), (nv,)) for k in ("vx", "vy", "vz")], 1).copy()
        nrm = None
        if mv.nx:
            nrm = np.stack([np.ctypeslib.as_array(getattr(mv, k), (nv,)) for k in ("nx", "ny", "nz")], 1).copy()
        nt = mv.num_triangles
        idx = np.ctypeslib.as_array(mv.indices, (nt, 3)).copy() if nt and mv.indices else np.zeros((0, 3), np.int32)
        mat = np.ctypeslib.as_array(mv.mat_ids, (nt,)).copy() if nt and mv.mat_ids else np.zeros(0, np.int32)
        out["meshes"].append({"nodes": nodes, "prims": prims, "pos": pos, "nrm": nrm, "indices": idx,
                              "mat_ids": mat})
    n = v.num_tlas_nodes
    out["tlas_nodes"] = np.frombuffer((ctypes.c_char * (n * 32)).from_address(v.tlas_nodes), NODE_DTYPE).copy() if n else np.zeros(0, NODE_DTYPE)
    out["tlas_inst"] = np.ctypeslib.as_array(v.tlas_inst_indices, (v.num_instances,)).copy() if v.num_instances else np.zeros(0, np.uint32)
    n = v.num_prim_nodes
    out["prim_nodes"] = np.frombuffer((ctypes.c_char * (n * 32)).from_address(v.prim_nodes), NODE_DTYPE).copy() if n else np.zeros(0, NODE_DTYPE)
    out["prim_indices"] = np.ctypeslib.as_array(v.prim_indices, (v.num_prims,)).copy() if v.num_prims else np.zeros(0, np.uint32)
    insts = []
    for i in range(v.num_instances):
        iv = v.instances[i]
        insts.append((iv.geom, iv.instance_id, np.array(iv.local_to_world[:], np.float32),
                      np.array(iv.world_to_local[:], np.float32)))
    out["instances"] = insts
    return out
