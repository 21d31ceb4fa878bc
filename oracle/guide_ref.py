"""FP64 oracle for the path-guiding network. Test infrastructure only.

Parity unpinned: the reference has no learned component, so nothing here restates reference code;
this is the project's own specification of the network, checked against finite differences and
quadrature (tests/test_guide_oracle.py) and used to check the GPU kernels. The reference-pinned
quantity for guiding is the image (the guided estimator converges to the plain tracer's image).

Network (the GPU kernels in xenon_b200/csrc/guide.cu follow this exactly, in BF16/FP32):
  input   64 features of a surface point: for position p in [0,1]^3 (scene bounds), shading
          normal n and outgoing direction wo:
            sin/cos(2^k pi p_a),  k = 0..5, a = x,y,z     36
            sin/cos(2^k pi n_a),  k = 0..1                 12
            sin/cos(2^k pi wo_a), k = 0..1                 12
            p_x, p_y, p_z, 1                                4
  layers  64 -> 64 -> 64 -> 64 (ReLU) -> 48 (linear); 40 outputs used
  lobes   k = 0..7 from raw[5k .. 5k+4]:
            mu_k    = m / sqrt(|m|^2 + 1e-8),  m = raw[5k:5k+3]
            kappa_k = exp(clamp(raw[5k+3], -4, 6))
            w       = softmax(raw[5k+4])
  select  a = A_MIN + (A_MAX - A_MIN) sigmoid(raw[40]): the probability of sampling q at the vertex
  pdf     q(w) = sum_k w_k kappa_k / (2 pi (1 - exp(-2 kappa_k))) exp(kappa_k (mu_k . w - 1))
  mixture p(w) = a q(w) + (1 - a) p_bsdf(w), the density the renderer samples
  loss    sum_b c_b (-log p_b(omega_b)) / sum_b c_b   (c_b >= 0: the integrand over the sampling
          density; p_bsdf(omega_b) is recorded with the sample) — the weighted negative
          log-likelihood of the mixture (Mueller et al., Neural Importance Sampling, 2019)
"""
from __future__ import annotations

import numpy as np

N_IN = 64
N_HID = 64
N_OUT = 48
N_LOBES = 8
KAPPA_MIN, KAPPA_MAX = -4.0, 6.0
A_MIN, A_MAX = 0.05, 0.6   # the network's selection range (xenon_b200/csrc/guide.h kAMin, kAMax)
SELECT = 40                     # raw output holding the selection logit
LAYERS = [(N_HID, N_IN), (N_HID, N_HID), (N_HID, N_HID), (N_OUT, N_HID)]  # (out, in)


def encode(p01: np.ndarray, n: np.ndarray, wo: np.ndarray) -> np.ndarray:
    p01, n, wo = (np.asarray(x, np.float64) for x in (p01, n, wo))
    feats = []
    for arr, nf in ((p01, 6), (n, 2), (wo, 2)):
        for a in range(3):
            for k in range(nf):
                x = (2.0 ** k) * np.pi * arr[:, a]
                feats += [np.sin(x), np.cos(x)]
    feats += [p01[:, 0], p01[:, 1], p01[:, 2], np.ones(len(p01))]
    return np.stack(feats, 1)


def init_params(seed: int = 0) -> dict:
    """He-uniform hidden layers; a small output layer (near-uniform mixture at start)."""
    rng = np.random.default_rng(seed)
    P = {}
    for i, (o, k) in enumerate(LAYERS):
        bound = np.sqrt(6.0 / k) * (0.1 if i == len(LAYERS) - 1 else 1.0)
        P[f"W{i}"] = rng.uniform(-bound, bound, (o, k))
        P[f"b{i}"] = np.zeros(o)
    return P


def flatten(P: dict) -> np.ndarray:
    """Parameter dict -> the flat vector W0 b0 W1 b1 W2 b2 W3 b3 (each W row-major [out][in])."""
    return np.concatenate([np.concatenate([P[f"W{i}"].ravel(), P[f"b{i}"]]) for i in range(len(LAYERS))])


def unflatten(v: np.ndarray) -> dict:
    v = np.asarray(v, np.float64)
    P, o = {}, 0
    for i, (out, k) in enumerate(LAYERS):
        P[f"W{i}"] = v[o:o + out * k].reshape(out, k)
        o += out * k
        P[f"b{i}"] = v[o:o + out].copy()
        o += out
    assert o == len(v)
    return P


def features(f9: np.ndarray) -> np.ndarray:
    """Rows of (position in [0,1]^3, normal, outgoing direction) -> the 64 encoded inputs."""
    f9 = np.asarray(f9, np.float64)
    return encode(f9[:, 0:3], f9[:, 3:6], f9[:, 6:9])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even) and back, as the tensor-core operands are."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return (((u + r) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def forward(P: dict, X: np.ndarray, emulate_bf16: bool = False):
    """Returns (activations [X, a1, a2, a3], raw outputs). With emulate_bf16 the MMA operands
    (inputs, activations, weights) are rounded to bf16 and everything else stays exact."""
    q = bf16 if emulate_bf16 else (lambda v: v)
    acts = [q(X)]
    h = acts[0]
    for i in range(len(LAYERS)):
        z = h @ q(P[f"W{i}"]).T + P[f"b{i}"]
        if i < len(LAYERS) - 1:
            h = q(np.maximum(z, 0.0))
            acts.append(h)
        else:
            return acts, z
    raise AssertionError


def lobes(raw: np.ndarray):
    r = raw[:, :5 * N_LOBES].reshape(-1, N_LOBES, 5)
    m = r[..., 0:3]
    s = np.sqrt((m * m).sum(-1) + 1e-8)
    mu = m / s[..., None]
    kraw = r[..., 3]
    kappa = np.exp(np.clip(kraw, KAPPA_MIN, KAPPA_MAX))
    logits = r[..., 4]
    e = np.exp(logits - logits.max(-1, keepdims=True))
    w = e / e.sum(-1, keepdims=True)
    return mu, kappa, w, s, kraw


def selection(raw: np.ndarray) -> np.ndarray:
    return A_MIN + (A_MAX - A_MIN) / (1.0 + np.exp(-raw[:, SELECT]))


def vmf_norm(kappa):
    return kappa / (2.0 * np.pi * (-np.expm1(-2.0 * kappa)))


def pdf(raw: np.ndarray, omega: np.ndarray) -> np.ndarray:
    mu, kappa, w, _, _ = lobes(raw)
    cos = (mu * omega[:, None, :]).sum(-1)
    v = vmf_norm(kappa) * np.exp(kappa * (cos - 1.0))
    return (w * v).sum(-1)


def loss_grad_raw(raw: np.ndarray, omega: np.ndarray, c: np.ndarray, pb: np.ndarray | None = None):
    """Loss and dLoss/draw for the weighted negative log-likelihood of the mixture
    p = a q + (1 - a) pb (pb = None: of q alone, a fixed at 1)."""
    mu, kappa, w, s, kraw = lobes(raw)
    cos = (mu * omega[:, None, :]).sum(-1)
    v = vmf_norm(kappa) * np.exp(kappa * (cos - 1.0))
    q = (w * v).sum(-1)
    if pb is None:
        a = np.ones(len(raw))
        pm = q
    else:
        a = selection(raw)
        pm = a * q + (1.0 - a) * pb
    csum = c.sum()
    loss = float((c * -np.log(pm)).sum() / csum)
    cb = (c / csum)
    rho = a * q / pm                      # the share of the mixture density that q holds
    cq = (cb * rho)[:, None]              # d(-log pm) = rho * d(-log q) for q's parameters
    r = w * v / q[:, None]
    g = np.zeros_like(raw)
    gl = g[:, :5 * N_LOBES].reshape(-1, N_LOBES, 5)
    gl[..., 4] = cq * (w - r)
    dlogv_dk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (cos - 1.0)
    inside = (kraw > KAPPA_MIN) & (kraw < KAPPA_MAX)
    gl[..., 3] = -cq * r * dlogv_dk * kappa * inside
    dmu = -(cq * r * kappa)[..., None] * omega[:, None, :]
    proj = (dmu * mu).sum(-1, keepdims=True)
    gl[..., 0:3] = (dmu - proj * mu) / s[..., None]
    if pb is not None:
        sig = (a - A_MIN) / (A_MAX - A_MIN)
        g[:, SELECT] = cb * (-(q - pb) / pm) * (A_MAX - A_MIN) * sig * (1.0 - sig)
    return loss, g


def backward(P: dict, acts: list, graw: np.ndarray, emulate_bf16: bool = False) -> dict:
    q = bf16 if emulate_bf16 else (lambda v: v)
    G = {}
    delta = graw
    for i in reversed(range(len(LAYERS))):
        G[f"W{i}"] = delta.T @ acts[i]
        G[f"b{i}"] = delta.sum(0)
        if i > 0:
            delta = (delta @ q(P[f"W{i}"])) * (acts[i] > 0)
    return G


def loss_and_grads(P: dict, X: np.ndarray, omega: np.ndarray, c: np.ndarray, emulate_bf16: bool = False,
                   pb: np.ndarray | None = None):
    acts, raw = forward(P, X, emulate_bf16)
    loss, graw = loss_grad_raw(raw, omega, c, pb)
    return loss, backward(P, acts, graw, emulate_bf16), raw


def adam(P: dict, G: dict, M: dict, V: dict, t: int, lr=5e-3, b1=0.9, b2=0.99, eps=1e-8):
    for k in P:
        M[k] = b1 * M[k] + (1 - b1) * G[k]
        V[k] = b2 * V[k] + (1 - b2) * G[k] ** 2
        mh = M[k] / (1 - b1 ** t)
        vh = V[k] / (1 - b2 ** t)
        P[k] = P[k] - lr * mh / (np.sqrt(vh) + eps)


def sample(raw: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Directions from the mixture: u[:, 0] picks the lobe, u[:, 1:3] the vMF direction."""
    mu, kappa, w, _, _ = lobes(raw)
    cdf = np.cumsum(w, -1)
    k = np.minimum((u[:, :1] > cdf).sum(-1), N_LOBES - 1)
    idx = np.arange(len(raw))
    m, kp = mu[idx, k], kappa[idx, k]
    cos = 1.0 + np.log(u[:, 1] + (1.0 - u[:, 1]) * np.exp(-2.0 * kp)) / kp
    sin = np.sqrt(np.maximum(0.0, 1.0 - cos * cos))
    phi = 2.0 * np.pi * u[:, 2]
    a = np.where(np.abs(m[:, 0:1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    t = np.cross(m, a)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(m, t)
    return cos[:, None] * m + sin[:, None] * (np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * b)
