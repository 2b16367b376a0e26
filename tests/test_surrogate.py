"""The warm-start surrogate: its device kernels (include/lbm_surrogate.h)
against the numpy oracle (oracle/unet_oracle.py), the oracle's own backward
pass against finite differences, and the data plumbing of warmstart.py.

Tolerances: the device accumulates in FP32 in another order than the float64
oracle, and both round to bfloat16 at the same points, so FP32 outputs agree to
~1e-5 of their scale and bf16 outputs to one bf16 unit (2^-8 relative)."""
import numpy as np
import pytest

import unet_oracle as U


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
def test_layer_tables_agree(pkg):
    S = pkg.surrogate
    assert S.layer_table() == U.layer_table()
    assert (S.IN_CH, S.LEVELS, S.OUT_CH) == (U.IN_CH, U.LEVELS, U.OUT_CH)
    n = U.param_count()
    assert 1.8e6 < n < 2.2e6  # the ~2M-parameter 4-level U-Net


def test_bf16_round_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = U.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                       # tie rounds to even (1.0)
    assert r[2] == 1.0 + 2 ** -7             # above the tie rounds up
    assert r[3] == -2.5
    assert np.isfinite(r[4])


def test_oracle_backward_matches_finite_differences():
    # float64, no bf16 rounding: the oracle's analytic gradients of
    # L = sum(dy * y) against central differences on a 16x16 image
    rng = np.random.default_rng(0)
    params = U.init_params(1)
    params = {k: (w, rng.normal(0, 0.1, size=b.shape)) for k, (w, b) in params.items()}
    x = rng.normal(size=(1, 16, 16, U.IN_CH))
    y, cache = U.forward(params, x, bf16=False)
    dy = rng.normal(size=y.shape)
    grads = U.backward(cache, dy, bf16=False)

    def L(p):
        return float((U.forward(p, x, bf16=False)[0] * dy).sum())

    h = 1e-6
    for name in ("e1a", "e2b", "bb", "d3a", "d1b", "head"):
        w, b = params[name]
        for _ in range(3):
            idx = tuple(rng.integers(0, s) for s in w.shape)
            wp, wm = w.copy(), w.copy()
            wp[idx] += h
            wm[idx] -= h
            fd = (L({**params, name: (wp, b)}) - L({**params, name: (wm, b)})) / (2 * h)
            an = grads[name][0][idx]
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (name, idx, fd, an)
        j = int(rng.integers(0, b.shape[0]))
        bp, bm = b.copy(), b.copy()
        bp[j] += h
        bm[j] -= h
        fd = (L({**params, name: (w, bp)}) - L({**params, name: (w, bm)})) / (2 * h)
        assert abs(fd - grads[name][1][j]) <= 1e-5 * max(1.0, abs(fd)), (name, "bias")


def test_resample_round_trip(pkg):
    W = pkg.warmstart
    rng = np.random.default_rng(2)
    a = rng.normal(size=(24, 24))
    assert np.allclose(W.resample(a, (24, 24)), a)
    # linear fields in index space survive down- and up-sampling away from the ends
    yy, xx = np.meshgrid((np.arange(64) + 0.5) / 64, (np.arange(64) + 0.5) / 64, indexing="ij")
    lin = 2.0 * xx - 0.5 * yy
    back = W.resample(W.resample(lin, (32, 32)), (64, 64))
    assert np.abs(back - lin)[2:-2, 2:-2].max() < 1e-12


def test_features_encode_grid_and_parameters(pkg):
    W = pkg.warmstart
    case = W.sample_cases(1, seed=3, sizes=(96,))[0]
    f = W.features(case, 32)
    assert f.shape == (32, 32, W.NF) and W.NF <= pkg.surrogate.IN_CH
    assert np.all(np.diff(f[0, :, 0]) > 0) and np.all(np.diff(f[:, 0, 1]) > 0)   # X along x, Y along y
    assert 0.0 < f[0, 0, 0] < f[0, -1, 0] < 1.0
    assert np.allclose(f[..., 2], (np.log10(case["Ra"]) - 4.5) / 1.5)
    assert np.all(f[..., 5:] == 0)


# ---------------------------------------------------------------------------
# GPU: kernels against the oracle
# ---------------------------------------------------------------------------
def _dev():
    import torch
    return torch, torch.device("cuda", 0)


def _bf16(torch, dev, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev).to(torch.bfloat16)


def _f32(torch, dev, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _close(a, b, rel):
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= rel * scale


@pytest.mark.gpu
@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("Cin,Cout,xs,xo", [(32, 48, 32, 0), (64, 128, 96, 32), (96, 32, 96, 0)])
def test_conv3x3_forward_and_data_gradient(pkg, Cin, Cout, xs, xo, path):
    torch, dev = _dev()
    lib = pkg.surrogate.nn()
    pkg.surrogate.set_tensor_path(path)
    try:
        _conv_forward_and_data_gradient(torch, dev, lib, Cin, Cout, xs, xo)
    finally:
        pkg.surrogate.set_tensor_path(0)
    assert pkg.surrogate.timeouts(reset=True) == 0


def _conv_forward_and_data_gradient(torch, dev, lib, Cin, Cout, xs, xo):
    rng = np.random.default_rng(Cin + Cout)
    B, H, W = 2, 12, 20
    xfull = U.bf16_round(rng.normal(size=(B, H, W, xs)))
    x = xfull[..., xo:xo + Cin]
    w = U.bf16_round(rng.normal(0, 0.1, size=(Cout, 9, Cin)))
    bias = rng.normal(size=Cout).astype(np.float32).astype(np.float64)
    xd, wd, bd = _bf16(torch, dev, xfull), _bf16(torch, dev, w), _f32(torch, dev, bias)
    z = torch.zeros(B, H, W, Cout + 8, dtype=torch.float32, device=dev)
    a = torch.zeros(B, H, W, Cout, dtype=torch.bfloat16, device=dev)
    st = lib.lbm_nn_conv3x3(xd.data_ptr(), xs, xo, wd.data_ptr(), bd.data_ptr(), B, H, W, Cin, Cout,
                            z.data_ptr(), Cout + 8, 8, 0, a.data_ptr(), Cout, 0, 1, None)
    assert st == 0
    torch.cuda.synchronize()
    zr = U.conv3x3(x, w, bias)
    assert _close(_np(z)[..., 8:8 + Cout], zr, 1e-5)
    ar = U.bf16_round(U.silu(_np(z)[..., 8:8 + Cout]))
    assert np.abs(_np(a) - ar).max() <= 2 ** -7 * np.abs(ar).max()
    # data gradient through the flipped weights, accumulated onto a prefilled buffer
    dz = U.bf16_round(rng.normal(size=(B, H, W, Cout)))
    if Cout % 32 == 0:
        wt = torch.zeros(Cin * 9 * Cout, dtype=torch.bfloat16, device=dev)
        assert lib.lbm_nn_flip_weights(wd.data_ptr(), wt.data_ptr(), Cout, Cin, None) == 0
        assert np.array_equal(_np(wt).reshape(Cin, 9, Cout), U.flip_weights(w))
        dx = torch.ones(B, H, W, Cin, dtype=torch.float32, device=dev)
        dzd = _bf16(torch, dev, dz)
        st = lib.lbm_nn_conv3x3(dzd.data_ptr(), Cout, 0, wt.data_ptr(), None, B, H, W, Cout, Cin,
                                dx.data_ptr(), Cin, 0, 1, None, 0, 0, 0, None)
        assert st == 0
        torch.cuda.synchronize()
        assert _close(_np(dx) - 1.0, U.conv3x3_dgrad(dz, w), 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("Cin,Cout,H", [(32, 32, 16), (64, 96, 10), (128, 64, 34)])
def test_conv3x3_weight_gradient(pkg, Cin, Cout, H):
    torch, dev = _dev()
    lib = pkg.surrogate.nn()
    rng = np.random.default_rng(H)
    B = 3
    x = U.bf16_round(rng.normal(size=(B, H, H, Cin + 32)))
    dz = U.bf16_round(rng.normal(size=(B, H, H, Cout)))
    xd, dzd = _bf16(torch, dev, x), _bf16(torch, dev, dz)
    n = lib.lbm_nn_wgrad_workspace(B, H, H, Cin, Cout)
    ws = torch.zeros(n, dtype=torch.float32, device=dev)
    dw = torch.zeros(Cout * 9 * Cin, dtype=torch.float32, device=dev)
    st = lib.lbm_nn_conv3x3_wgrad(dzd.data_ptr(), xd.data_ptr(), Cin + 32, 32, B, H, H, Cin, Cout, ws.data_ptr(), n,
                                  dw.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    ref = U.conv3x3_wgrad(dz, x[..., 32:])
    assert _close(_np(dw).reshape(Cout, 9, Cin), ref, 1e-5)
    # deterministic: a second call gives the same bits
    dw2 = torch.zeros_like(dw)
    lib.lbm_nn_conv3x3_wgrad(dzd.data_ptr(), xd.data_ptr(), Cin + 32, 32, B, H, H, Cin, Cout, ws.data_ptr(), n,
                             dw2.data_ptr(), None)
    torch.cuda.synchronize()
    assert torch.equal(dw, dw2)


@pytest.mark.gpu
def test_elementwise_kernels(pkg):
    torch, dev = _dev()
    lib = pkg.surrogate.nn()
    rng = np.random.default_rng(5)
    B, H, C = 2, 8, 40
    # pool / up and their backwards, with channel offsets
    x = U.bf16_round(rng.normal(size=(B, H, H, C + 8)))
    xd = _bf16(torch, dev, x)
    y = torch.zeros(B, H // 2, H // 2, C, dtype=torch.bfloat16, device=dev)
    assert lib.lbm_nn_pool2(xd.data_ptr(), C + 8, 8, B, H, H, C, y.data_ptr(), C, 0, None) == 0
    u = torch.zeros(B, 2 * H, 2 * H, C, dtype=torch.bfloat16, device=dev)
    assert lib.lbm_nn_up2(xd.data_ptr(), C + 8, 8, B, H, H, C, u.data_ptr(), C, 0, None) == 0
    dy = rng.normal(size=(B, H // 2, H // 2, C))
    dx = torch.full((B, H, H, C), 0.5, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_pool2_backward(_f32(torch, dev, dy).data_ptr(), C, 0, B, H, H, C, dx.data_ptr(), C, 0, None) == 0
    dyu = rng.normal(size=(B, 2 * H, 2 * H, C))
    dxu = torch.zeros(B, H, H, C, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_up2_backward(_f32(torch, dev, dyu).data_ptr(), C, 0, B, H, H, C, dxu.data_ptr(), C, 0, 0,
                                   None) == 0
    # silu backward and column sums
    da = rng.normal(size=(B * H * H, C))
    z = rng.normal(size=(B * H * H, C))
    dz = torch.zeros(B * H * H, C, dtype=torch.bfloat16, device=dev)
    assert lib.lbm_nn_silu_backward(_f32(torch, dev, da).data_ptr(), C, 0, _f32(torch, dev, z).data_ptr(), B * H * H, C,
                                    dz.data_ptr(), None) == 0
    n = lib.lbm_nn_colsum_workspace(B * H * H, C)
    ws = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
    cs = torch.zeros(C, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_colsum(dz.data_ptr(), B * H * H, C, ws.data_ptr(), cs.data_ptr(), None) == 0
    torch.cuda.synchronize()
    xs = x[..., 8:]
    assert np.abs(_np(y) - U.bf16_round(U.pool2(xs))).max() <= 2 ** -7 * np.abs(xs).max()
    assert np.array_equal(_np(u), U.up2(xs))
    assert np.allclose(_np(dx), 0.5 + U.pool2_backward(dy), rtol=1e-6, atol=1e-6)
    assert np.allclose(_np(dxu), U.up2_backward(dyu), rtol=1e-5, atol=1e-5)
    dzr = U.bf16_round((da * U.silu_grad(z)).astype(np.float32))
    assert np.abs(_np(dz) - dzr).max() <= 2 ** -7 * np.abs(dzr).max()
    assert np.allclose(_np(cs), _np(dz).sum(0), rtol=1e-5, atol=1e-4)


@pytest.mark.gpu
def test_head_loss_and_adam(pkg):
    torch, dev = _dev()
    lib = pkg.surrogate.nn()
    rng = np.random.default_rng(6)
    P, C, J = 3000, 32, 3
    a = U.bf16_round(rng.normal(size=(P, C)))
    wh = U.bf16_round(rng.normal(size=(J, C)))
    bh = rng.normal(size=J).astype(np.float32).astype(np.float64)
    ad, whd = _bf16(torch, dev, a), _bf16(torch, dev, wh)
    y = torch.zeros(P, J, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_head(ad.data_ptr(), C, 0, whd.data_ptr(), _f32(torch, dev, bh).data_ptr(), P, C, J, y.data_ptr(),
                           None) == 0
    t = rng.normal(size=(P, J))
    cw = np.array([1.0, 2.0, 0.5])
    n = max(lib.lbm_nn_mse_workspace(P, J), lib.lbm_nn_head_workspace(P, C, J))
    ws = torch.zeros(n, dtype=torch.float32, device=dev)
    dy = torch.zeros(P, J, dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_mse(y.data_ptr(), _f32(torch, dev, t).data_ptr(), _f32(torch, dev, cw).data_ptr(), P, J,
                          dy.data_ptr(), ws.data_ptr(), n, loss.data_ptr(), None) == 0
    torch.cuda.synchronize()
    yr = U.head(a, wh, bh)
    assert _close(_np(y), yr, 1e-5)
    lr_, dyr = U.mse(_np(y), t, cw)
    assert abs(float(loss.item()) - lr_) <= 1e-5 * lr_
    assert _close(_np(dy), dyr, 1e-5)
    da = torch.zeros(P, C, dtype=torch.float32, device=dev)
    dwh = torch.zeros(J, C, dtype=torch.float32, device=dev)
    dbh = torch.zeros(J, dtype=torch.float32, device=dev)
    assert lib.lbm_nn_head_backward(dy.data_ptr(), ad.data_ptr(), C, 0, whd.data_ptr(), P, C, J, da.data_ptr(), C, 0,
                                    ws.data_ptr(), n, dwh.data_ptr(), dbh.data_ptr(), None) == 0
    torch.cuda.synchronize()
    dyh = _np(dy)
    assert _close(_np(da), dyh @ wh, 1e-5)
    assert _close(_np(dwh), dyh.T @ a, 1e-4)
    assert _close(_np(dbh), dyh.sum(0), 1e-4)
    # Adam against the textbook update
    m0 = rng.normal(size=50) * 0.01
    v0 = np.abs(rng.normal(size=50)) * 0.01
    p0, g = rng.normal(size=50), rng.normal(size=50)
    p, m, v = (_f32(torch, dev, q) for q in (p0, m0, v0))
    pb = torch.zeros(50, dtype=torch.bfloat16, device=dev)
    b1, b2, lr, eps, wd = 0.9, 0.999, 1e-2, 1e-8, 1e-3
    c1, c2 = 1 - b1 ** 3, 1 - b2 ** 3
    assert lib.lbm_nn_adam(p.data_ptr(), pb.data_ptr(), _f32(torch, dev, g).data_ptr(), m.data_ptr(), v.data_ptr(), 50,
                           lr, b1, b2, eps, c1, c2, wd, None) == 0
    torch.cuda.synchronize()
    mr = b1 * m0 + (1 - b1) * g
    vr = b2 * v0 + (1 - b2) * g * g
    pr = p0 - lr * ((mr / c1) / (np.sqrt(vr / c2) + eps) + wd * p0)
    assert np.allclose(_np(p), pr, rtol=1e-5, atol=1e-6)
    assert np.array_equal(_np(pb), U.bf16_round(_np(p)))


@pytest.mark.gpu
def test_network_forward_and_gradients_match_oracle(pkg):
    # the whole U-Net on the device (mma.sync convolutions) against the oracle
    # with the same bf16 rounding points: outputs and every parameter gradient
    torch, dev = _dev()
    S = pkg.surrogate
    rng = np.random.default_rng(7)
    params = U.init_params(3)
    params = {k: (w, rng.normal(0, 0.05, size=b.shape).astype(np.float32)) for k, (w, b) in params.items()}
    B = 2
    x = U.bf16_round(rng.normal(size=(B, 32, 32, U.IN_CH)))
    dy = rng.normal(size=(B * 32 * 32, U.OUT_CH)).astype(np.float32)
    S.set_tensor_path(0)
    try:
        net = S.Net(R=32, params=params)
        y = net.forward(_bf16(torch, dev, x))
        net.buffers(B)["dy"].copy_(_f32(torch, dev, dy))
        net.backward(B)
        torch.cuda.synchronize()
    finally:
        S.set_tensor_path(0)
    yr, cache = U.forward({k: (np.asarray(w, np.float64), np.asarray(b, np.float64)) for k, (w, b) in params.items()},
                          x, bf16=True)
    assert np.linalg.norm(_np(y) - yr.reshape(-1, 3)) <= 1e-2 * np.linalg.norm(yr)
    gr = U.backward(cache, dy.reshape(yr.shape).astype(np.float64), bf16=True)
    gd = net.get_params("grad")
    for name in list(gr):
        for k in range(2):
            ref, got = gr[name][k], gd[name][k]
            err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            assert err <= 2e-2, (name, k, err)


@pytest.mark.gpu
def test_training_reduces_loss(pkg):
    # fit four fixed smooth targets; the loss must fall well below its start
    W = pkg.warmstart
    rng = np.random.default_rng(8)
    R = 32
    X = np.zeros((4, R, R, pkg.surrogate.IN_CH), dtype=np.float32)
    yy, xx = np.meshgrid((np.arange(R) + 0.5) / R, (np.arange(R) + 0.5) / R, indexing="ij")
    Y = np.zeros((4, R, R, 3), dtype=np.float32)
    for i in range(4):
        X[i, ..., 0], X[i, ..., 1], X[i, ..., 2] = xx, yy, i / 3.0
        Y[i, ..., 0] = np.sin(np.pi * xx) * np.sin(2 * np.pi * yy) * (1 + i)
        Y[i, ..., 1] = -np.sin(2 * np.pi * xx) * np.sin(np.pi * yy) * (1 + i)
        Y[i, ..., 2] = 1 - xx + 0.1 * i * np.sin(np.pi * xx)
    ws = W.WarmStart(R=R, seed=0)
    hist = ws.fit(X, Y, steps=300, batch=4, lr=2e-3, warmup=20, log_every=50, seed=rng.integers(1 << 30))
    assert hist[-1][1] < 0.1 * hist[0][1]
    pred = ws.predict_images(X)
    assert np.sqrt(((pred - Y) ** 2).mean()) < 0.3 * Y.std()


@pytest.mark.gpu
@pytest.mark.parametrize("Cin,Cout,H,W", [(32, 32, 16, 24), (64, 64, 12, 20), (96, 128, 8, 40), (128, 256, 9, 15),
                                          (32, 48, 17, 13)])
def test_tcgen05_convolution_matches_oracle(pkg, Cin, Cout, H, W):
    # the tcgen05 path (accumulators in tensor memory) against the oracle and
    # against the mma.sync path, forward with bias + SiLU and accumulate mode
    torch, dev = _dev()
    S = pkg.surrogate
    lib = S.nn()
    rng = np.random.default_rng(Cin * Cout + H)
    B = 2
    x = U.bf16_round(rng.normal(size=(B, H, W, Cin)))
    w = U.bf16_round(rng.normal(0, 0.1, size=(Cout, 9, Cin)))
    bias = rng.normal(size=Cout).astype(np.float32).astype(np.float64)
    xd, wd, bd = _bf16(torch, dev, x), _bf16(torch, dev, w), _f32(torch, dev, bias)
    outs = {}
    S.timeouts(reset=True)
    try:
        for path in (0, 1):
            S.set_tensor_path(path)
            z = torch.zeros(B, H, W, Cout, dtype=torch.float32, device=dev)
            a = torch.zeros(B, H, W, Cout, dtype=torch.bfloat16, device=dev)
            assert lib.lbm_nn_conv3x3(xd.data_ptr(), Cin, 0, wd.data_ptr(), bd.data_ptr(), B, H, W, Cin, Cout,
                                      z.data_ptr(), Cout, 0, 0, a.data_ptr(), Cout, 0, 1, None) == 0
            acc = torch.ones(B, H, W, Cout, dtype=torch.float32, device=dev)
            assert lib.lbm_nn_conv3x3(xd.data_ptr(), Cin, 0, wd.data_ptr(), None, B, H, W, Cin, Cout,
                                      acc.data_ptr(), Cout, 0, 1, None, 0, 0, 0, None) == 0
            torch.cuda.synchronize()
            outs[path] = (_np(z), _np(a), _np(acc))
    finally:
        S.set_tensor_path(0)
    assert S.timeouts(reset=True) == 0
    zr = U.conv3x3(x, w, bias)
    z1, a1, acc1 = outs[1]
    assert _close(z1, zr, 1e-5)
    assert np.abs(a1 - U.bf16_round(U.silu(z1))).max() <= 2 ** -7 * np.abs(a1).max()
    assert _close(acc1 - 1.0, zr - bias, 1e-5)
    assert _close(z1, outs[0][0], 1e-5)


@pytest.mark.gpu
def test_network_gradients_on_tcgen05_path(pkg):
    # the whole U-Net's gradients with the tcgen05 convolutions, against the oracle
    torch, dev = _dev()
    S = pkg.surrogate
    rng = np.random.default_rng(9)
    params = {k: (w, rng.normal(0, 0.05, size=b.shape).astype(np.float32)) for k, (w, b) in U.init_params(4).items()}
    S.set_tensor_path(1)
    try:
        net = S.Net(R=32, params=params)
        x = U.bf16_round(rng.normal(size=(2, 32, 32, U.IN_CH)))
        y = net.forward(_bf16(torch, dev, x))
        dy = rng.normal(size=(2 * 32 * 32, U.OUT_CH)).astype(np.float32)
        net.buffers(2)["dy"].copy_(_f32(torch, dev, dy))
        net.backward(2)
        torch.cuda.synchronize()
    finally:
        S.set_tensor_path(0)
    assert S.timeouts(reset=True) == 0
    yr, cache = U.forward({k: (np.asarray(w, np.float64), np.asarray(b, np.float64)) for k, (w, b) in params.items()},
                          x)
    assert np.linalg.norm(_np(y) - yr.reshape(-1, 3)) <= 1e-2 * np.linalg.norm(yr)
    gr = U.backward(cache, dy.reshape(yr.shape).astype(np.float64))
    gd = net.get_params("grad")
    for name in gr:
        for k in range(2):
            err = np.linalg.norm(gd[name][k] - gr[name][k]) / max(np.linalg.norm(gr[name][k]), 1e-30)
            assert err <= 2e-2, (name, k, err)


def test_centro_symmetrize_is_a_projection(pkg):
    # the projection keeps symmetric fields, removes antisymmetric ones, and is idempotent
    W = pkg.warmstart
    rng = np.random.default_rng(4)
    u, v, T = rng.normal(size=(3, 12, 9))
    su, sv, sT = W.centro_symmetrize(u, v, T, 1.0, 0.0)
    assert np.allclose(su, -su[::-1, ::-1]) and np.allclose(sv, -sv[::-1, ::-1])
    assert np.allclose(sT, 1.0 - sT[::-1, ::-1])
    again = W.centro_symmetrize(su, sv, sT, 1.0, 0.0)
    assert all(np.allclose(a, b) for a, b in zip(again, (su, sv, sT)))
    # the mesh the projection relies on: node i mirrors node n+1-i about the centre
    m = pkg.mesh_box(24, 24, 0, 1.0, 1.0, 1.0, "tanh", 1.7)
    lo, hi = m.x[1] - 0.5 * m.dt, m.x[24] + 0.5 * m.dt
    assert np.allclose(m.x[1:25] - lo, hi - m.x[24:0:-1], atol=1e-9)


def test_surrogate_entry_points_reject_bad_arguments_without_a_gpu(pkg):
    # argument checks come before any device work, so they hold on a machine
    # without a GPU; fake (never dereferenced) but aligned addresses stand in
    # for device buffers
    lib = pkg.surrogate.nn()
    P = pkg.lib()
    x, w, o = 1 << 20, 2 << 20, 3 << 20
    ERR_PARAM = -1
    # Cin not a multiple of 32
    assert lib.lbm_nn_conv3x3(x, 16, 0, w, None, 1, 8, 8, 16, 32, o, 32, 0, 0, None, 0, 0, 1, None) == ERR_PARAM
    # input channel window outside the stride
    assert lib.lbm_nn_conv3x3(x, 32, 8, w, None, 1, 8, 8, 32, 32, o, 32, 0, 0, None, 0, 0, 1, None) == ERR_PARAM
    # misaligned input
    assert lib.lbm_nn_conv3x3(x + 2, 32, 0, w, None, 1, 8, 8, 32, 32, o, 32, 0, 0, None, 0, 0, 1, None) == ERR_PARAM
    # accumulate with a bias
    assert lib.lbm_nn_conv3x3(x, 32, 0, w, o, 1, 8, 8, 32, 32, o, 32, 0, 1, None, 0, 0, 0, None) == ERR_PARAM
    # no output at all
    assert lib.lbm_nn_conv3x3(x, 32, 0, w, None, 1, 8, 8, 32, 32, None, 0, 0, 0, None, 0, 0, 1, None) == ERR_PARAM
    # weight gradient: Cout not a multiple of 8, workspace too small
    assert lib.lbm_nn_conv3x3_wgrad(x, w, 32, 0, 1, 8, 8, 32, 12, o, 1 << 20, o, None) == ERR_PARAM
    need = lib.lbm_nn_wgrad_workspace(1, 8, 8, 32, 32)
    assert need > 0
    assert lib.lbm_nn_conv3x3_wgrad(x, w, 32, 0, 1, 8, 8, 32, 32, o, need - 1, o, None) == ERR_PARAM
    # pooling needs even sizes; the head at most 8 outputs; Adam needs positive bias corrections
    assert lib.lbm_nn_pool2(x, 32, 0, 1, 7, 8, 32, o, 32, 0, None) == ERR_PARAM
    assert lib.lbm_nn_head(x, 32, 0, w, None, 64, 32, 9, o, None) == ERR_PARAM
    assert lib.lbm_nn_adam(x, None, w, o, o, 10, 1e-3, 0.9, 0.999, 1e-8, 0.0, 1.0, 0.0, None) == ERR_PARAM
    assert lib.lbm_nn_set_tensor_path(3) == ERR_PARAM
    assert lib.lbm_nn_set_tensor_path(2) == ERR_PARAM
    assert "path" in P.lbm_last_error().decode()
    assert lib.lbm_nn_get_tensor_path() in (0, 1)


def test_masked_batch_run_rejects_a_null_batch(pkg):
    import ctypes
    conv = (ctypes.c_int32 * 1)()
    done = (ctypes.c_int64 * 1)()
    assert pkg.lib().lbm_batch_run_masked(None, None, 10, 2, 1e-6, conv, done) == -1
