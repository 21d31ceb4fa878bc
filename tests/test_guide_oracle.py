"""The guiding network's FP64 oracle checked on its own: analytic gradients against finite
differences, the vMF mixture normalised over the sphere, sampling consistent with the pdf."""
import numpy as np
import pytest

from oracle import guide_ref as g


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    p = rng.random((n, 3))
    nn = rng.normal(size=(n, 3)); nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3)); wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    om = rng.normal(size=(n, 3)); om /= np.linalg.norm(om, axis=1, keepdims=True)
    c = rng.random(n) * 3.0
    return g.encode(p, nn, wo), om, c


def test_encoding_shape_and_range():
    X, _, _ = _batch(10, 0)
    assert X.shape == (10, 64)
    assert np.all(np.abs(X[:, :60]) <= 1.0) and np.all(X[:, 63] == 1.0)


@pytest.mark.parametrize("mixture", [False, True])
def test_gradients_match_finite_differences(mixture):
    P = g.init_params(3)
    for k in P:          # larger output layer so every lobe matters
        if k == "W3":
            P[k] = P[k] * 10
    P["b3"][g.SELECT] = 0.7
    X, om, c = _batch(16, 1)
    pb = np.random.default_rng(5).random(16) * 0.6 if mixture else None
    if mixture:
        pb[3] = 0.0                       # a direction the BSDF cannot sample
    loss, G, _ = g.loss_and_grads(P, X, om, c, pb=pb)
    rng = np.random.default_rng(7)
    checks = [(key, tuple(rng.integers(0, s) for s in P[key].shape))
              for key in ("W0", "b0", "W1", "W2", "W3", "b3") for _ in range(6)]
    checks += [("b3", (g.SELECT,)), ("W3", (g.SELECT, 5)), ("W3", (g.SELECT, 17))]
    for key, idx in checks:
        h = 1e-6
        Pp = {k: v.copy() for k, v in P.items()}
        Pm = {k: v.copy() for k, v in P.items()}
        Pp[key][idx] += h
        Pm[key][idx] -= h
        lp, _, _ = g.loss_and_grads(Pp, X, om, c, pb=pb)
        lm, _, _ = g.loss_and_grads(Pm, X, om, c, pb=pb)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - G[key][idx]) <= 1e-6 + 1e-4 * abs(fd), (key, idx, fd, G[key][idx])


def test_mixture_pdf_integrates_to_one():
    P = g.init_params(5)
    P["W3"] *= 30.0          # sharp lobes: kappa up to e^6
    X, _, _ = _batch(4, 2)
    _, raw = g.forward(P, X)
    # Fibonacci sphere quadrature
    n = 400_000
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    phi = np.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    for row in range(len(raw)):
        q = g.pdf(np.repeat(raw[row:row + 1], n, 0), dirs)
        integral = q.mean() * 4 * np.pi
        assert abs(integral - 1.0) < 2e-3, integral


def test_sampling_follows_the_pdf():
    P = g.init_params(9)
    P["W3"] *= 20.0
    X, _, _ = _batch(1, 4)
    _, raw = g.forward(P, X)
    rng = np.random.default_rng(1)
    n = 200_000
    R = np.repeat(raw, n, 0)
    d = g.sample(R, rng.random((n, 3)))
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-9)
    # E_q[f / q] = integral of f for f = 1 + x: Monte Carlo estimate of the sphere integral
    f = 1.0 + d[:, 0]
    est = np.mean(f / g.pdf(R, d))
    assert abs(est - 4 * np.pi) / (4 * np.pi) < 0.02, est
