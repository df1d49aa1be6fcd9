"""The CPU MLP oracle against finite differences (float64, no BF16 rounding).

The surrogate network has no reference counterpart, so its oracle is pinned by
calculus: analytic gradients and forward-mode tangents against central
differences of the oracle's own loss / output.
"""

import numpy as np
import pytest

from oracle import mlp_oracle as mo


def _net(rng, F=32, hidden=64, depth=2, outs=2):
    dims = [2 * F] + [hidden] * depth + [outs]
    Ws = [rng.normal(0, 1.0 / np.sqrt(dims[i]), (dims[i + 1], dims[i])) for i in range(len(dims) - 1)]
    bs = [rng.normal(0, 0.1, dims[i + 1]) for i in range(len(dims) - 1)]
    freq = np.zeros((F, 4), dtype=np.float32)
    freq[:, :3] = rng.normal(0, 2.0, (F, 3))
    return freq, Ws, bs


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1e-30], dtype=np.float64)
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even
    assert r[2] == 1.0 + 4 * 2 ** -8        # tie -> even (up)
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 1e-30) / 1e-30 < 2 ** -8


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    freq, Ws, bs = _net(rng)
    pts = rng.uniform(0, 6.28, (16, 3))
    feat = mo.features(pts, freq)
    target = rng.normal(0, 1, (16, 2))
    loss, gW, gb, _ = mo.loss_and_grads(feat, Ws, bs, target, 2, bf16_points=False)
    eps = 1e-6
    for l in range(len(Ws)):
        for (i, j) in [(0, 0), (1, 3), (Ws[l].shape[0] - 1, Ws[l].shape[1] - 1)]:
            Wp = [w.copy() for w in Ws]
            Wp[l][i, j] += eps
            Wm = [w.copy() for w in Ws]
            Wm[l][i, j] -= eps
            lp = mo.loss_and_grads(feat, Wp, bs, target, 2, bf16_points=False)[0]
            lm = mo.loss_and_grads(feat, Wm, bs, target, 2, bf16_points=False)[0]
            assert gW[l][i, j] == pytest.approx((lp - lm) / (2 * eps), rel=1e-5, abs=1e-9)
        bp = [b.copy() for b in bs]
        bp[l][0] += eps
        bm = [b.copy() for b in bs]
        bm[l][0] -= eps
        lp = mo.loss_and_grads(feat, Ws, bp, target, 2, bf16_points=False)[0]
        lm = mo.loss_and_grads(feat, Ws, bm, target, 2, bf16_points=False)[0]
        assert gb[l][0] == pytest.approx((lp - lm) / (2 * eps), rel=1e-5, abs=1e-9)


def test_tangents_match_finite_differences():
    rng = np.random.default_rng(2)
    freq, Ws, bs = _net(rng)
    pts = rng.uniform(0, 6.28, (8, 3))
    feat, tx, ty = mo.features(pts, freq, tangents=True)
    _, jx, jy = mo.jacobian(feat, tx, ty, Ws, bs, bf16_points=False)
    eps = 1e-6
    for axis, j in ((0, jx), (1, jy)):
        d = np.zeros(3)
        d[axis] = eps
        yp = mo.forward(mo.features(pts + d, freq), Ws, bs, bf16_points=False)["Y"]
        ym = mo.forward(mo.features(pts - d, freq), Ws, bs, bf16_points=False)["Y"]
        np.testing.assert_allclose(j, (yp - ym) / (2 * eps), rtol=1e-5, atol=1e-8)


def test_3d_tangents_and_ftle_match_finite_differences():
    rng = np.random.default_rng(3)
    F = 32
    freq = np.zeros((F, 8), dtype=np.float32)
    freq[:, :4] = rng.normal(0, 1.5, (F, 4))
    dims = [2 * F, 48, 48, 3]
    Ws = [rng.normal(0, 1.0 / np.sqrt(dims[i]), (dims[i + 1], dims[i])) for i in range(3)]
    bs = [rng.normal(0, 0.1, dims[i + 1]) for i in range(3)]
    pts = rng.uniform(0, 6.28, (6, 4))
    feat, *tan = mo.features(pts, freq, tangents=True)
    assert len(tan) == 3
    _, J = mo.jacobian_n(feat, tan, Ws, bs, bf16_points=False)
    eps = 1e-6
    for a in range(3):
        d = np.zeros(4)
        d[a] = eps
        yp = mo.forward(mo.features(pts + d, freq), Ws, bs, bf16_points=False)["Y"]
        ym = mo.forward(mo.features(pts - d, freq), Ws, bs, bf16_points=False)["Y"]
        np.testing.assert_allclose(J[a], (yp - ym) / (2 * eps), rtol=1e-5, atol=1e-8)
    # FTLE of the map x + s*y(x) against finite differences of the map itself
    s, T = 0.3, 2.0
    f = mo.ftle_from_tangents(J, s, T)
    h = 1e-6
    Fd = np.zeros((6, 3, 3))
    for a in range(3):
        d = np.zeros(4)
        d[a] = h
        xp = pts[:, :3] + d[:3] + s * mo.forward(mo.features(pts + d, freq), Ws, bs, False)["Y"]
        xm = pts[:, :3] - d[:3] + s * mo.forward(mo.features(pts - d, freq), Ws, bs, False)["Y"]
        Fd[:, :, a] = (xp - xm) / (2 * h)
    lam = np.linalg.eigvalsh(np.einsum("nra,nrb->nab", Fd, Fd))[:, -1]
    np.testing.assert_allclose(f, np.log(np.sqrt(lam)) / T, rtol=1e-6)
