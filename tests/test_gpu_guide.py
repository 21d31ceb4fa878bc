"""The guiding network's tensor-core path (tcgen05 BF16 MMA, FP32 accumulation in TMEM)."""
import ctypes

import numpy as np
import pytest

import xenon_b200 as xb


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bit patterns."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16_to_f32(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 48, 64])
@pytest.mark.parametrize("rows", [128, 300])
def test_tc_gemm_matches_fp64(n, rows):
    rng = np.random.default_rng(n * 1000 + rows)
    a = bf16_bits(rng.normal(size=(rows, 64)))
    b = bf16_bits(rng.normal(size=(n, 64)))
    d = np.zeros((rows, n), np.float32)
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    xb.native.check(xb.lib().xb_tc_gemm_bf16(p(a), p(b), rows, n, p(d)))
    want = bf16_to_f32(a).astype(np.float64) @ bf16_to_f32(b).astype(np.float64).T
    err = np.abs(d - want) / (np.abs(want) + 1.0)
    assert err.max() < 1e-4, (err.max(), np.unravel_index(err.argmax(), err.shape))


# ── the guiding network against its FP64 oracle (oracle/guide_ref.py) ───────────────
from oracle import guide_ref as G  # noqa: E402


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _feats(rng, n):
    return np.concatenate([rng.random((n, 3)), _unit(rng, n), _unit(rng, n)], 1).astype(np.float32)


def _params(seed, out_scale=10.0):
    P = G.init_params(seed)
    P["W3"] = P["W3"] * out_scale           # sharper, more distinct lobes than at initialisation
    rng = np.random.default_rng(seed + 100)
    for i in range(4):
        P[f"b{i}"] = rng.normal(scale=0.1, size=P[f"b{i}"].shape)
    return G.flatten(P).astype(np.float32)


def _records(rng, n, mixture=True):
    R = np.zeros((n, 24), np.float32)
    R[:, 0:9] = _feats(rng, n)
    R[:, 9:12] = _unit(rng, n)
    R[:, 12] = rng.random(n) * 2.0
    if mixture:
        R[:, 20] = rng.random(n) * 0.5          # density of the BSDF sampler at the direction
        R[::7, 20] = 0.0                        # directions the BSDF cannot produce
    else:
        R[:, 20] = -1.0                         # loss of q alone
    return R


def _oracle_loss(params, R, emulate=True):
    mixture = R[0, 20] >= 0
    return G.loss_and_grads(G.unflatten(params), G.features(R[:, 0:9]), R[:, 9:12].astype(np.float64),
                            R[:, 12].astype(np.float64), emulate_bf16=emulate,
                            pb=R[:, 20].astype(np.float64) if mixture else None)


def _oracle_lobes(params, f9):
    _, raw = G.forward(G.unflatten(params), G.features(f9), emulate_bf16=True)
    mu, kappa, w, _, _ = G.lobes(raw)
    return mu, kappa, w, raw


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [1, 127, 1000])
def test_guide_forward_matches_oracle(rows):
    rng = np.random.default_rng(rows)
    params = _params(3)
    f9 = _feats(rng, rows)
    got, sel = xb.guide_forward(params, f9, with_selection=True)
    mu, kappa, w, raw = _oracle_lobes(params, f9)
    assert np.abs(sel - G.selection(raw)).max() < 1e-2
    # BF16 operands on both sides; the remaining differences are FP32 vs FP64 accumulation and
    # activations that round to a neighbouring bf16 value
    assert np.abs(got[:, :, 0:3] - mu).max() < 2e-2
    assert np.median(np.abs(got[:, :, 0:3] - mu)) < 1e-3
    assert (np.abs(got[:, :, 3] - kappa) / kappa).max() < 2e-2
    assert np.abs(got[:, :, 4] - w).max() < 5e-3
    assert np.allclose(got[:, :, 4].sum(1), 1.0, atol=1e-5)
    assert np.allclose(np.linalg.norm(got[:, :, 0:3], axis=2), 1.0, atol=1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("n,mixture", [(128, False), (777, False), (128, True), (777, True)])
def test_guide_gradient_matches_oracle(n, mixture):
    rng = np.random.default_rng(n)
    params = _params(5)
    R = _records(rng, n, mixture)
    loss, grad = xb.guide_loss_grad(params, R)
    want_loss, GW, _ = _oracle_loss(params, R)
    want = G.flatten(GW)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss) + 1e-5, (loss, want_loss)
    # per layer: the backward MMAs take the error signal in BF16, so relative agreement ~1e-2
    for i, (o, k) in enumerate(G.LAYERS):
        sl = slice(i * 4160, i * 4160 + o * k + o)
        num = np.linalg.norm(grad[sl] - want[sl])
        den = np.linalg.norm(want[sl]) + 1e-12
        assert num / den < 3e-2, (i, num / den)


@pytest.mark.gpu
def test_guide_adam_steps_match_oracle():
    rng = np.random.default_rng(11)
    params = _params(7)
    R = _records(rng, 512)
    steps = 4
    got, losses = xb.guide_train(params, R, steps=steps, batch=512, lr=1e-3)
    P = G.unflatten(params)
    M = {k: np.zeros_like(v) for k, v in P.items()}
    V = {k: np.zeros_like(v) for k, v in P.items()}
    want_losses = []
    X = G.features(R[:, 0:9])
    for t in range(1, steps + 1):
        l, GW, _ = G.loss_and_grads(P, X, R[:, 9:12].astype(np.float64), R[:, 12].astype(np.float64), True,
                                    pb=R[:, 20].astype(np.float64))
        want_losses.append(l)
        G.adam(P, GW, M, V, t, lr=1e-3)
    want = G.flatten(P)
    d_got, d_want = got - params, want - params
    rel = np.linalg.norm(d_got - d_want) / np.linalg.norm(d_want)
    assert rel < 0.1, rel
    assert np.allclose(losses, want_losses, rtol=2e-3, atol=1e-5), (losses, want_losses)


@pytest.mark.gpu
def test_guide_training_learns_a_direction_field():
    """Records whose directions concentrate around a position-dependent axis: training must raise
    the learned density there far above uniform (1 / 4 pi)."""
    rng = np.random.default_rng(2)
    n = 16384
    R = _records(rng, n, mixture=False)
    axis = np.stack([np.cos(2 * np.pi * R[:, 0]), np.sin(2 * np.pi * R[:, 0]), 0.3 * np.ones(n)], 1)
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    om = axis + 0.15 * rng.normal(size=(n, 3))
    R[:, 9:12] = om / np.linalg.norm(om, axis=1, keepdims=True)
    R[:, 12] = 1.0
    params = xb.guide_init_params(1)
    trained, losses = xb.guide_train(params, R, steps=600, batch=4096, lr=5e-3)
    assert losses[-20:].mean() < losses[:5].mean() - 1.5, (losses[:5], losses[-20:])
    lob = xb.guide_forward(trained, R[:256, 0:9])
    q = xb.guide_mixture_pdf(lob, axis[:256].astype(np.float32))
    assert np.median(q) > 20 * (1 / (4 * np.pi)), np.median(q)


def _fibonacci(n):
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)


@pytest.mark.gpu
def test_guide_mixture_pdf_normalised_and_matches_oracle():
    rng = np.random.default_rng(4)
    params = _params(9, out_scale=30.0)      # concentrations up to e^6
    lob = xb.guide_forward(params, _feats(rng, 3))
    dirs = _fibonacci(300_000)
    for row in range(3):
        L = np.repeat(lob[row:row + 1].reshape(1, 40), len(dirs), 0)
        q = xb.guide_mixture_pdf(L, dirs.astype(np.float32)).astype(np.float64)
        integral = q.mean() * 4 * np.pi
        assert abs(integral - 1.0) < 3e-3, integral
        # the same lobes through the FP64 formula
        raw = np.zeros((len(dirs), 48))
        Lr = lob[row].astype(np.float64)
        raw5 = raw[:, :40].reshape(-1, 8, 5)
        kap = Lr[:, 3]
        raw5[..., 0:3] = Lr[:, 0:3]
        raw5[..., 3] = np.log(kap)
        raw5[..., 4] = np.log(Lr[:, 4])
        want = G.pdf(raw, dirs)
        assert np.max(np.abs(q - want) / (want + 1e-3)) < 1e-3


@pytest.mark.gpu
def test_guide_mixture_sampling_follows_the_pdf():
    rng = np.random.default_rng(6)
    params = _params(13, out_scale=20.0)
    lob = xb.guide_forward(params, _feats(rng, 1))
    n = 400_000
    L = np.repeat(lob.reshape(1, 40), n, 0)
    d, pdf = xb.guide_mixture_sample(L, rng.random((n, 3)).astype(np.float32))
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    again = xb.guide_mixture_pdf(L, d)
    assert np.allclose(pdf, again, rtol=1e-6)
    # E_q[g / q] = integral of g over the sphere for g = 1 + x (4 pi) and g = z^2 (4 pi / 3)
    for g, want in ((1.0 + d[:, 0], 4 * np.pi), (d[:, 2] ** 2, 4 * np.pi / 3)):
        est = np.mean(g / pdf)
        se = np.std(g / pdf) / np.sqrt(n)
        assert abs(est - want) < 5 * se + 1e-3 * want, (est, want, se)
    # the sample mean direction equals the pdf's first moment (quadrature in FP64)
    dirs = _fibonacci(300_000)
    q = xb.guide_mixture_pdf(np.repeat(lob.reshape(1, 40), len(dirs), 0), dirs.astype(np.float32))
    m1 = (dirs * q[:, None].astype(np.float64)).mean(0) * 4 * np.pi
    se = d.std(0) / np.sqrt(n)
    assert np.all(np.abs(d.mean(0) - m1) < 5 * se + 1e-3), (d.mean(0), m1, se)
