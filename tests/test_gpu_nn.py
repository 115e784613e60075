"""The warm-start network's CUDA kernels (pty_nn_*, pty_warm_*) through the C ABI against the float64 numpy
restatement in oracle/nn_ref.py, layer by layer and for the whole network's forward and backward pass."""
import ctypes
import os
import sys

import numpy as np
import pytest

from conftest import rel_err

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import nn_ref  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 2e-5


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.float64)


def _lib():
    from ptychopy_b200 import abi

    return abi, abi.lib()


@pytest.mark.parametrize("B,Cin,Cout,H,W,relu", [(2, 3, 5, 8, 8, 0), (2, 1, 16, 16, 16, 1), (3, 9, 40, 13, 13, 0),
                                                  (1, 17, 33, 11, 20, 1), (2, 64, 130, 8, 8, 1),
                                                  (1, 20, 7, 35, 33, 0)])
def test_conv3x3_forward_and_gradients(B, Cin, Cout, H, W, relu):
    import torch

    abi, L = _lib()
    rng = np.random.default_rng(B * 1000 + Cin * 10 + Cout)
    x = rng.standard_normal((B, Cin, H, W))
    w = rng.standard_normal((Cout, Cin, 3, 3)) / np.sqrt(Cin * 9)
    b = rng.standard_normal(Cout)
    dy = rng.standard_normal((B, Cout, H, W))
    xd, wd, bd, dyd = _dev(x), _dev(w), _dev(b), _dev(dy)
    y = torch.empty((B, Cout, H, W), device="cuda")
    abi.check(L.pty_nn_conv3x3(_p(xd), _p(wd), _p(bd), _p(y), B, Cin, Cout, H, W, relu, None))
    ref = nn_ref.conv3x3(x, w, b)
    if relu:
        ref = nn_ref.relu(ref)
    assert rel_err(_host(y), ref) < TOL
    dx = torch.empty_like(xd)
    dw = torch.full_like(wd, 7.0)  # overwritten, not accumulated
    db = torch.full_like(bd, 7.0)
    abi.check(L.pty_nn_conv3x3_bwd(_p(xd), _p(wd), _p(dyd), _p(dx), _p(dw), _p(db), B, Cin, Cout, H, W, None))
    rdx, rdw, rdb = nn_ref.conv3x3_bwd(x, w, dy)
    assert rel_err(_host(dx), rdx) < TOL
    assert rel_err(_host(dw), rdw) < TOL
    assert rel_err(_host(db), rdb) < TOL
    # without dx and db
    abi.check(L.pty_nn_conv3x3_bwd(_p(xd), _p(wd), _p(dyd), None, _p(dw), None, B, Cin, Cout, H, W, None))
    assert rel_err(_host(dw), rdw) < TOL


def test_elementwise_layers():
    import torch

    abi, L = _lib()
    rng = np.random.default_rng(5)
    x = rng.standard_normal((2, 3, 12, 10)).astype(np.float32).astype(np.float64)  # exact in float32
    xd = _dev(x)
    pooled = torch.empty((2, 3, 6, 5), device="cuda")
    abi.check(L.pty_nn_pool2(_p(xd), _p(pooled), 6, 6, 5, None))
    assert rel_err(_host(pooled), nn_ref.pool2(x)) < 1e-6
    g = rng.standard_normal((2, 3, 6, 5))
    gx = torch.empty_like(xd)
    gd = _dev(g)  # every device buffer stays referenced until the kernel has run
    abi.check(L.pty_nn_pool2_bwd(_p(gd), _p(gx), 6, 6, 5, None))
    assert rel_err(_host(gx), nn_ref.pool2_bwd(g)) < 1e-6
    up = torch.empty((2, 3, 24, 20), device="cuda")
    abi.check(L.pty_nn_up2(_p(xd), _p(up), 6, 12, 10, None))
    assert rel_err(_host(up), nn_ref.up2(x)) == 0
    g2 = rng.standard_normal((2, 3, 24, 20))
    gu = torch.empty_like(xd)
    g2d = _dev(g2)
    abi.check(L.pty_nn_up2_bwd(_p(g2d), _p(gu), 6, 12, 10, None))
    assert rel_err(_host(gu), nn_ref.up2_bwd(g2)) < 1e-6
    r = xd.clone()
    abi.check(L.pty_nn_relu(_p(r), r.numel(), None))
    assert rel_err(_host(r), nn_ref.relu(x)) == 0
    gr = _dev(x[::-1].copy())
    abi.check(L.pty_nn_relu_bwd(_p(r), _p(gr), r.numel(), None))
    assert rel_err(_host(gr), nn_ref.relu_bwd(nn_ref.relu(x), x[::-1])) == 0


def test_weighted_mse_and_adam():
    import torch

    abi, L = _lib()
    rng = np.random.default_rng(6)
    p, t = rng.standard_normal((4, 3, 8, 8)), rng.standard_normal((4, 3, 8, 8))
    w = rng.uniform(0.1, 2.0, (8, 8))
    g = torch.empty((4, 3, 8, 8), device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    pd_, td_, wd_ = _dev(p), _dev(t), _dev(w)
    abi.check(L.pty_nn_mse(_p(pd_), _p(td_), _p(wd_), 64, _p(g), p.size, _p(loss), None))
    d = p - t
    n = p.size
    assert abs(float(loss.cpu()) - float((w * d * d).sum() / n)) < 1e-6 * float((w * d * d).sum() / n)
    assert rel_err(_host(g), 2 * w * d / n) < 1e-6
    abi.check(L.pty_nn_mse(_p(pd_), _p(td_), None, 0, _p(g), p.size, _p(loss), None))
    assert abs(float(loss.cpu()) - float((d * d).mean())) < 1e-6 * float((d * d).mean())
    # Adam: three steps
    prm, gr = rng.standard_normal(1000), rng.standard_normal(1000)
    pd, gd = _dev(prm), _dev(gr)
    md, vd = torch.zeros_like(pd), torch.zeros_like(pd)
    m, v = np.zeros(1000), np.zeros(1000)
    for s in range(1, 4):
        abi.check(L.pty_nn_adam(_p(pd), _p(gd), _p(md), _p(vd), 1000, 1e-2, 0.9, 0.999, 1e-8, s, None))
        prm, m, v = nn_ref.adam(prm, gr, m, v, s, lr=1e-2)
    assert rel_err(_host(pd), prm) < 1e-6


def _np_net(plan, params, x, g_out):
    """Forward and backward of the warm-start network in numpy (float64) from nn_ref layers."""
    acts, a = [], x
    off = 0
    ws = []
    for cin, cout, H, relu, after in plan:
        w = params[off:off + cout * cin * 9].reshape(cout, cin, 3, 3)
        b = params[off + cout * cin * 9:off + cout * cin * 9 + cout]
        off += cout * cin * 9 + cout
        ws.append((w, b))
        y = nn_ref.conv3x3(a, w, b)
        if relu:
            y = nn_ref.relu(y)
        post = nn_ref.pool2(y) if after == "pool" else (nn_ref.up2(y) if after == "up" else y)
        acts.append((a, y))
        a = post
    out = a
    grads = []
    g = g_out
    for l in range(len(plan) - 1, -1, -1):
        cin, cout, H, relu, after = plan[l]
        a_in, y = acts[l]
        gy = nn_ref.pool2_bwd(g) if after == "pool" else (nn_ref.up2_bwd(g) if after == "up" else g)
        if relu:
            gy = nn_ref.relu_bwd(y, gy)
        dx, dw, db = nn_ref.conv3x3_bwd(a_in, ws[l][0], gy)
        grads.append((dw, db))
        g = dx
    flat = np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads[::-1]])
    return out, flat


def test_network_forward_backward_matches_numpy():
    import torch

    from ptychopy_b200 import warmstart

    net = warmstart.Net(N=32, width=2, seed=3)
    rng = np.random.default_rng(8)
    B = 3
    x = rng.standard_normal((B, 1, 32, 32))
    xd = _dev(x)
    out = net.forward(xd, B)
    g = rng.standard_normal((B, 3, 8, 8))
    ref_out, ref_grads = _np_net(net.plan, net.state().astype(np.float64), x, g)
    assert rel_err(_host(out), ref_out) < 1e-4
    net.backward(_dev(g), B)
    assert rel_err(_host(net.grads), ref_grads) < 1e-4
    # the same buffers at a smaller batch
    out1 = net.forward(xd[:1], 1)
    assert rel_err(_host(out1), ref_out[:1]) < 1e-4
    torch.cuda.synchronize()


def test_warm_assembly_matches_numpy():
    import torch

    from ptychopy_b200 import abi, synth, warmstart

    L = abi.lib()
    rng = np.random.default_rng(9)
    N, S = 64, 16
    dx_s = synth.sample_pixel(2.48e-10, 1.0, 172e-6, N)
    pos, X, Y = synth.raster_positions(6, 5, 40e-9, 40e-9, dx_s, N)
    P = pos.shape[0]
    probe = synth.make_probe(N, dx_s, K=1, fwhm=8 * dx_s)[0]
    amp = rng.uniform(0, 3, (P, N, N)).astype(np.float32)
    ampd = _dev(amp)
    # network input
    xin = torch.empty((P, 1, N, N), device="cuda")
    abi.check(L.pty_warm_input(_p(ampd), _p(xin), P, N, 0.25, None))
    assert rel_err(_host(xin)[:, 0], nn_ref.warm_input(amp, 0.25)) < 1e-6
    # stitching and assembly
    out = rng.standard_normal((P, 3, S, S)).astype(np.float32) * 0.5
    weight = warmstart.stitch_weight(probe, S)
    ref_acc = nn_ref.warm_stitch(out, pos, weight, N, X, Y, warmstart.AMP_MEAN, warmstart.AMP_SCALE,
                                 warmstart.GRAD_SCALE)
    acc = torch.empty((4, X, Y), device="cuda")
    outd, posd, wd = _dev(out), _dev(pos), _dev(weight)
    abi.check(L.pty_warm_stitch(_p(outd), _p(posd), P, _p(wd), S, N, warmstart.AMP_MEAN,
                                warmstart.AMP_SCALE, warmstart.GRAD_SCALE, _p(acc), X, Y, None))
    assert rel_err(_host(acc), ref_acc) < 1e-5
    obj = warmstart.assemble(outd, pos, probe, X, Y, ampd)
    ref_obj = nn_ref.warm_object(ref_acc, 1e-3, warmstart.AMP_MEAN, probe, pos, amp)
    got = obj.cpu().numpy().view(np.complex64)[..., 0]
    assert got.shape == (X, Y)
    assert rel_err(got, ref_obj) < 1e-4
