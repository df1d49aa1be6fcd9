"""Surrogate MLP kernels (tcgen05 BF16 GEMMs, fused epilogues, loss, Adam,
tangents) against float64 references and the CPU MLP oracle."""

import math

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _lib():
    from pyftle_b200 import _lib
    return _lib


def _ptr(t):
    import ctypes
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    import ctypes
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _bf(shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen, dtype=torch.float32) * scale).to(
        torch.bfloat16).cuda()


@pytest.mark.parametrize("a_t,b_t", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K,splits", [(128, 16, 64, 1), (256, 256, 256, 1),
                                          (200, 64, 320, 1), (384, 264, 128, 1),
                                          (128, 96, 1024, 4)])
def test_gemm_matches_fp64(a_t, b_t, M, N, K, splits):
    L = _lib()
    g = torch.Generator().manual_seed(M * 7 + N + K)
    A = _bf((K, M) if a_t else (M, K), g)
    B = _bf((K, N) if b_t else (N, K), g)
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    if splits > 1:
        C.zero_()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("ftle_mlp_gemm", _ptr(A), A.shape[1], a_t, _ptr(B), B.shape[1], b_t, _ptr(C), N, M, N,
           K, splits, 0, _ptr(err), _stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    a = A.double().cpu()
    b = B.double().cpu()
    a = a.T if a_t else a
    b = b.T if b_t else b
    ref = a @ b.T
    bound = (a.abs() @ b.abs().T) * 2e-6 + 1e-6  # FP32 accumulation over K terms
    assert torch.all((C.double().cpu() - ref).abs() <= bound * math.sqrt(K))


def test_gemm_accumulates_into_c():
    L = _lib()
    g = torch.Generator().manual_seed(5)
    A, B = _bf((128, 64), g), _bf((32, 64), g)
    C = torch.ones(128, 32, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("ftle_mlp_gemm", _ptr(A), 64, 0, _ptr(B), 64, 0, _ptr(C), 32, 128, 32, 64, 1, 1,
           _ptr(err), _stream())
    ref = A.double().cpu() @ B.double().cpu().T + 1.0
    torch.testing.assert_close(C.double().cpu(), ref, rtol=1e-5, atol=1e-5)


def test_gemm_rejects_bad_shapes():
    L = _lib()
    A = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(128, 16, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(L.FTLEError, match="K must be a multiple of 64"):
        L.call("ftle_mlp_gemm", _ptr(A), 64, 0, _ptr(A), 64, 0, _ptr(C), 16, 128, 16, 48, 1, 0,
               _ptr(err), _stream())
    with pytest.raises(L.FTLEError, match="multiples of 8"):
        L.call("ftle_mlp_gemm", _ptr(A), 64, 0, _ptr(A), 64, 0, _ptr(C), 16, 100, 12, 64, 1, 0,
               _ptr(err), _stream())


def test_linear_silu_and_dsilu_epilogues():
    L = _lib()
    g = torch.Generator().manual_seed(9)
    M, N, K = 256, 128, 192
    X, W = _bf((M, K), g), _bf((N, K), g, 0.1)
    b = (torch.randn(N, generator=g) * 0.3).cuda()
    Z = torch.empty(M, N, dtype=torch.float32, device="cuda")
    H = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("ftle_mlp_linear", _ptr(X), K, _ptr(W), K, _ptr(b), M, N, K, 1, _ptr(Z), N, _ptr(H), N,
           _ptr(err), _stream())
    z_ref = X.double().cpu() @ W.double().cpu().T + b.double().cpu()
    torch.testing.assert_close(Z.double().cpu(), z_ref, rtol=1e-5, atol=1e-5)
    h_ref = mo.bf16(mo.silu(z_ref.numpy()))
    np.testing.assert_allclose(H.double().cpu().numpy(), h_ref, rtol=1e-2, atol=1e-3)
    # dsilu: G = (A B^T) * silu'(Z); colsum = column sums of the BF16 G
    A2 = _bf((M, 64), g)
    B2 = _bf((N, 64), g)
    G = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    cs = torch.zeros(N, dtype=torch.float32, device="cuda")
    L.call("ftle_mlp_gemm_dsilu", _ptr(A2), 64, 0, _ptr(B2), 64, 0, M, N, 64, _ptr(Z), N, _ptr(G),
           N, _ptr(cs), _ptr(err), _stream())
    acc = (A2.double().cpu() @ B2.double().cpu().T).numpy()
    g_ref = acc * mo.dsilu(Z.double().cpu().numpy())
    np.testing.assert_allclose(G.double().cpu().numpy(), g_ref, rtol=1e-2, atol=1e-3)
    np.testing.assert_allclose(cs.double().cpu().numpy(), G.double().cpu().numpy().sum(0),
                               rtol=1e-5, atol=1e-4)
    torch.cuda.synchronize()
    assert int(err.item()) == 0


def _small_net(hidden=256, depth=4, seed=3):
    from pyftle_b200.surrogate import FlowMapMLP, fourier_frequencies
    return FlowMapMLP(fourier_frequencies(32, seed=seed), hidden=hidden, depth=depth,
                      out_scale=0.1, seed=seed)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_gradients_match_oracle():
    net = _small_net()
    rng = np.random.default_rng(4)
    n = 1024
    pts = np.column_stack((rng.uniform(0, 2 * np.pi, (n, 2)), rng.uniform(0, 10, n)))
    target = rng.normal(0, 1, (n, 2)).astype(np.float32)
    P = torch.from_numpy(pts).cuda()
    T = torch.from_numpy(target).cuda()
    loss = net.loss_and_grads(P, T)
    torch.cuda.synchronize()
    net.check_errors()
    Ws = [net.weight(l, bf16=True).double().cpu().numpy()[:L.fan_out]
          for l, L in enumerate(net.layers)]
    bs = [net.bias(l).double().cpu().numpy()[:L.fan_out] for l, L in enumerate(net.layers)]
    feat = mo.features(pts, net.freq_np)
    ref_loss, gW, gb, _ = mo.loss_and_grads(feat, Ws, bs, target.astype(np.float64), 2)
    assert float(loss.item()) == pytest.approx(ref_loss, rel=1e-3)
    for l, L in enumerate(net.layers):
        gw = net.grad_weight(l).double().cpu().numpy()
        assert np.all(gw[L.fan_out:] == 0.0)  # padded output rows get no gradient
        # BF16 rounding points are shared with the oracle; what is left is FP32 vs
        # FP64 accumulation and rare rounding-boundary flips
        assert _rel(gw[:L.fan_out], gW[l]) < 2e-3, l
        assert _rel(net.grad_bias(l).double().cpu().numpy()[:L.fan_out], gb[l]) < 2e-3, l
    # and the BF16 network's gradient is close to the exact FP64 gradient
    _, gW64, _, _ = mo.loss_and_grads(feat, Ws, bs, target.astype(np.float64), 2,
                                      bf16_points=False)
    for l in range(len(Ws)):
        assert _rel(net.grad_weight(l).double().cpu().numpy()[:net.layers[l].fan_out],
                    gW64[l]) < 5e-2


def test_tangents_match_oracle():
    net = _small_net(seed=6)
    rng = np.random.default_rng(7)
    n = 512
    pts = np.column_stack((rng.uniform(0, 2 * np.pi, (n, 2)), rng.uniform(0, 10, n)))
    P = torch.from_numpy(pts).cuda()
    y, jx, jy = net.predict(P, jacobian=True)
    torch.cuda.synchronize()
    net.check_errors()
    Ws, bs = net.numpy_params()
    Ws = [mo.bf16(w) for w in Ws]
    feat, tx, ty = mo.features(pts, net.freq_np, tangents=True)
    y_ref, jx_ref, jy_ref = mo.jacobian(feat, tx, ty, Ws, bs)
    assert _rel(y.double().cpu().numpy()[:, :2], y_ref) < 2e-3
    assert _rel(jx.double().cpu().numpy()[:, :2], jx_ref) < 5e-3
    assert _rel(jy.double().cpu().numpy()[:, :2], jy_ref) < 5e-3


def test_training_reduces_loss():
    from pyftle_b200.surrogate import TrainConfig, train
    net = _small_net(seed=8)
    g = torch.Generator(device="cuda").manual_seed(0)
    n = 1 << 16
    pts = torch.rand(n, 3, generator=g, device="cuda", dtype=torch.float64)
    pts[:, :2] *= 2 * math.pi
    pts[:, 2] *= 10
    disp = 0.1 * torch.stack((torch.sin(pts[:, 1] + 0.3 * pts[:, 2]),
                              torch.cos(2 * pts[:, 0]) * torch.sin(pts[:, 1])), dim=1)
    log = train(net, pts, disp, TrainConfig(steps=400, batch=8192, lr=2e-3, warmup=20,
                                            log_every=50))
    assert log[-1][1] < 0.02 * log[0][1], log


def _ftle_from_tangents(jx, jy, scale, T):
    a = 1.0 + scale * jx[:, 0]
    b = scale * jy[:, 0]
    c = scale * jx[:, 1]
    d = 1.0 + scale * jy[:, 1]
    c11, c12, c22 = a * a + c * c, a * b + c * d, b * b + d * d
    lam = 0.5 * (c11 + c22) + np.sqrt((0.5 * (c11 - c22)) ** 2 + c12 ** 2)
    return np.log(np.sqrt(lam)) / abs(T)


@pytest.mark.parametrize("n", [1, 40, 1003, 20000])
def test_fused_inference_matches_layered_kernels(n):
    net = _small_net(seed=11)
    # a few training steps so the weights are not at their initial values
    g = torch.Generator(device="cuda").manual_seed(1)
    pts = torch.rand(8192, 3, generator=g, device="cuda", dtype=torch.float64) * 6
    disp = 0.05 * torch.sin(pts[:, :2] + pts[:, 2:])
    from pyftle_b200.surrogate import TrainConfig, train
    train(net, pts, disp, TrainConfig(steps=20, batch=4096, warmup=2))
    rng = np.random.default_rng(n)
    t0, T = 3.7, 5.0
    seeds = torch.from_numpy(rng.uniform(0, 2 * np.pi, (n, 2))).cuda()
    end = torch.empty(n, 2, dtype=torch.float64, device="cuda")
    f = net.ftle_fused(seeds, t0, T, end_positions=end)
    m = (n + 7) // 8 * 8
    P = torch.zeros(m, 3, dtype=torch.float64, device="cuda")
    P[:n, :2] = seeds
    P[:, 2] = t0
    f_ref = net.ftle(P, T)[:n]
    e_ref = net.end_positions(P)[:n]
    torch.cuda.synchronize()
    net.check_errors()
    torch.testing.assert_close(f, f_ref, rtol=1e-6, atol=1e-9)
    torch.testing.assert_close(end, e_ref, rtol=1e-9, atol=1e-9)
    if n <= 1003:
        # and the oracle's FP64 evaluation of the same BF16 network
        Ws, bs = net.numpy_params()
        Ws = [mo.bf16(w) for w in Ws]
        pts_np = np.column_stack((seeds.cpu().numpy(), np.full(n, t0)))
        feat, tx, ty = mo.features(pts_np, net.freq_np, tangents=True)
        _, jx, jy = mo.jacobian(feat, tx, ty, Ws, bs)
        f_or = _ftle_from_tangents(jx, jy, net.out_scale, T)
        # absolute: single-seed FTLEs can sit near 0, where a relative bound is
        # meaningless; BF16 tangents move log(sigma) by ~1e-4 here, FTLE by ~1e-4/T
        assert np.max(np.abs(f.cpu().numpy() - f_or)) < 1e-3


def test_fused_inference_empty_and_errors():
    net = _small_net(seed=12)
    seeds = torch.empty(0, 2, dtype=torch.float64, device="cuda")
    assert net.ftle_fused(seeds, 0.0, 5.0).numel() == 0
    from pyftle_b200.surrogate import FlowMapMLP, fourier_frequencies
    small = FlowMapMLP(fourier_frequencies(32), hidden=128, depth=2)
    with pytest.raises(ValueError, match="fused kernel"):
        small.ftle_fused(torch.zeros(8, 2, dtype=torch.float64, device="cuda"), 0.0, 5.0)


def _small_turbulence(kmax=8.0, urms=0.2, n=256, S=60, dt=0.05):
    from pyftle_b200 import SnapshotSeries, flows
    from pyftle_b200.interpolate import GridSpec
    turb = flows.FourierTurbulence2D(seed=3, num_modes=64, kmin=2, kmax=kmax, urms=urms)
    snaps = turb.snapshots_device(n, np.arange(S) * dt)
    ax = flows.periodic_axis(n)
    grid = GridSpec(shape=(n, n), origin=(0.0, 0.0), spacing=(ax[1], ax[1]), periodic=True)
    return (SnapshotSeries(grid, snaps, precision="fp64"),
            SnapshotSeries(grid, snaps, precision="fx15"))


def test_surrogate_judge_and_what_training_gains():
    """The judge keeps the field within tolerance whatever the network, and the
    trained network earns acceptance that the untrained one does not."""
    from pyftle_b200.surrogate import (FlowMapMLP, SurrogateFTLE, TrainConfig, fit_flow_map,
                                       fourier_frequencies)
    s64, sfx = _small_turbulence()
    dt, h, T = 0.05, 0.025, 1.0
    starts = np.arange(20) * dt
    freq = fourier_frequencies(32, space_sigma=3.0, time_sigma=0.5, seed=1)
    net, fit = fit_flow_map(s64, T=T, h=h, snapshot_dt=dt, t0_values=starts,
                            num_samples=1 << 21, freq=freq,
                            cfg=TrainConfig(steps=1500, batch=16384, lr=2e-3, warmup=50))
    untrained = FlowMapMLP(freq, out_scale=net.out_scale, seed=5)
    m = 128
    sp = 2 * np.pi / m
    kw = dict(nx=m, ny=m, origin=(0.5 * sp, 0.5 * sp), spacing=(sp, sp), T=T, h=h,
              snapshot_dt=dt, tile=16)
    judged = {}
    for name, nn in (("trained", net), ("untrained", untrained)):
        sur = SurrogateFTLE(nn, sfx, **kw)
        t0 = float(starts[7])
        ref = sur.reference_field(t0)
        fs, sref, rerr = sur.evaluate(t0)
        raw = float(torch.linalg.vector_norm(fs - ref) / torch.linalg.vector_norm(ref))
        f, rep = sur.field(t0, tol=1e-3)
        # sampled seeds and every rejected region carry the RK4 values exactly
        bad = torch.nonzero(torch.from_numpy(rep.region_errors).cuda() > 1e-3).squeeze(1)
        rejected = torch.isin(sur.region_of, bad)
        assert torch.equal(f[rejected], ref[rejected])
        assert torch.equal(f[sur.sample_idx], ref[sur.sample_idx])
        judged[name] = dict(raw=raw, rerr=rep.region_errors,
                            err=float(torch.linalg.vector_norm(f - ref) /
                                      torch.linalg.vector_norm(ref)))
    print({k: (v["raw"], v["err"], float(np.median(v["rerr"]))) for k, v in judged.items()})
    tr, un = judged["trained"], judged["untrained"]
    # what training gains: a far more accurate flow map ...
    assert tr["raw"] < 0.25 * un["raw"]
    # ... and regions the judge accepts at a tolerance the untrained network never meets
    loose = float(np.quantile(tr["rerr"], 0.5))
    assert np.mean(tr["rerr"] <= loose) >= 0.5
    assert np.mean(un["rerr"] <= loose) == 0.0


# ---- 3D surrogate (input (x0, y0, z0, t0), hidden 384) ----------------------------------

def _net3d(hidden=384, seed=21):
    from pyftle_b200.surrogate import FlowMapMLP, fourier_frequencies
    return FlowMapMLP(fourier_frequencies(32, dim=3, space_sigma=2.0, seed=seed),
                      hidden=hidden, depth=4, out_scale=0.2, seed=seed)


def test_3d_gradients_match_oracle():
    net = _net3d()
    rng = np.random.default_rng(22)
    n = 512
    pts = np.column_stack((rng.uniform(0, 2 * np.pi, (n, 3)), rng.uniform(0, 5, n)))
    target = rng.normal(0, 1, (n, 3)).astype(np.float32)
    loss = net.loss_and_grads(torch.from_numpy(pts).cuda(), torch.from_numpy(target).cuda())
    torch.cuda.synchronize()
    net.check_errors()
    Ws = [net.weight(l, bf16=True).double().cpu().numpy()[:L.fan_out]
          for l, L in enumerate(net.layers)]
    bs = [net.bias(l).double().cpu().numpy()[:L.fan_out] for l, L in enumerate(net.layers)]
    ref_loss, gW, gb, _ = mo.loss_and_grads(mo.features(pts, net.freq_np), Ws, bs,
                                            target.astype(np.float64), 3)
    assert float(loss.item()) == pytest.approx(ref_loss, rel=1e-3)
    # the oracle rounds to BF16 at the GPU's points; FP32 (GPU) and FP64 (oracle) sums
    # then land on different sides of a BF16 rounding boundary now and then (2^-8 each),
    # and those flips compound back through four 384-wide layers: 5e-3 here
    # (measured 2.3e-3 for the first layer) against 2e-3 for the 256-wide 2D network
    for l, L in enumerate(net.layers):
        assert _rel(net.grad_weight(l).double().cpu().numpy()[:L.fan_out], gW[l]) < 5e-3, l
        assert _rel(net.grad_bias(l).double().cpu().numpy()[:L.fan_out], gb[l]) < 5e-3, l


def test_3d_tangents_and_ftle_match_oracle():
    net = _net3d(seed=23)
    rng = np.random.default_rng(24)
    n = 1000
    pts = np.column_stack((rng.uniform(0, 2 * np.pi, (n, 3)), rng.uniform(0, 5, n)))
    P = torch.from_numpy(pts).cuda()
    y, jx, jy, jz = net.predict(P, jacobian=True)
    Ws, bs = net.numpy_params()
    Ws = [mo.bf16(w) for w in Ws]
    feat, *tan = mo.features(pts, net.freq_np, tangents=True)
    y_ref, J = mo.jacobian_n(feat, tan, Ws, bs)
    assert _rel(y.double().cpu().numpy()[:, :3], y_ref) < 2e-3
    for got, ref in zip((jx, jy, jz), J):
        assert _rel(got.double().cpu().numpy()[:, :3], ref) < 5e-3
    f = net.ftle(P, 2.0).cpu().numpy()
    f_ref = mo.ftle_from_tangents(J, net.out_scale, 2.0)
    assert _rel(f, f_ref) < 5e-3
    end = net.end_positions(P).cpu().numpy()
    np.testing.assert_allclose(end, pts[:, :3] + net.out_scale * y_ref, rtol=0, atol=2e-3)
    torch.cuda.synchronize()
    net.check_errors()


def test_3d_surrogate_judge_and_what_training_gains():
    from pyftle_b200 import SnapshotSeries, flows
    from pyftle_b200.interpolate import GridSpec
    from pyftle_b200.surrogate import FlowMapMLP, SurrogateFTLE, TrainConfig, fit_flow_map
    n = 32
    ax = flows.periodic_axis(n)
    S = 16
    dt = 2 * math.pi / S
    snaps = flows.abc_snapshots(ax, ax, ax, np.arange(S) * dt)
    grid = GridSpec.from_points(flows.grid_points_3d(ax, ax, ax), (n, n, n), periodic=True)
    s64 = SnapshotSeries(grid, snaps, precision="fp64", periodic_time=True)
    sfx = SnapshotSeries(grid, snaps, precision="fx15", periodic_time=True)
    h, T = 0.05, 1.0
    starts = np.arange(4) * dt
    from pyftle_b200.surrogate import fourier_frequencies
    # the ABC field has only |k| = 1 modes: low spatial frequencies suit its flow map
    freq = fourier_frequencies(32, dim=3, space_sigma=1.5, time_sigma=0.5, seed=2)
    net, _ = fit_flow_map(s64, T=T, h=h, snapshot_dt=dt, t0_values=starts,
                          num_samples=1 << 21, hidden=384, freq=freq,
                          cfg=TrainConfig(steps=3000, batch=16384, lr=2e-3, warmup=50))
    untrained = FlowMapMLP(net.freq_np, hidden=384, out_scale=net.out_scale, seed=9)
    m = 16
    sp = 2 * np.pi / m
    errs = {}
    for name, nn in (("trained", net), ("untrained", untrained)):
        sur = SurrogateFTLE(nn, sfx, nx=m, ny=m, nz=m, origin=(0.5 * sp,) * 3,
                            spacing=(sp,) * 3, T=T, h=h, snapshot_dt=dt, delta=1e-3, tile=8)
        t0 = float(starts[1])
        ref = sur.reference_field(t0)
        fs, _, rerr = sur.evaluate(t0)
        f, rep = sur.field(t0, tol=1e-3)
        bad = torch.nonzero(torch.from_numpy(rep.region_errors).cuda() > 1e-3).squeeze(1)
        rejected = torch.isin(sur.region_of, bad)
        assert torch.equal(f[rejected], ref[rejected])
        assert torch.equal(f[sur.sample_idx], ref[sur.sample_idx])
        errs[name] = float(torch.linalg.vector_norm(fs - ref) / torch.linalg.vector_norm(ref))
    print("3D raw FTLE error", errs)
    assert errs["trained"] < 0.5 * errs["untrained"]
