"""Tensor-core (tcgen05, BF16 in, FP32 accumulate) convolution of the warm-start network's inference path against
float64 numpy on the same BF16-rounded inputs and weights, and the whole BF16 network against the FP32 one."""
import ctypes
import os
import sys

import numpy as np
import pytest

from conftest import rel_err

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import nn_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _bf16_round(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def _run_conv(x_dev, w, b, B, Cin, Cout, H, W, relu, in_mode, out_mode, in_scale=1.0):
    import torch

    from ptychopy_b200 import abi

    L = abi.lib()
    wd = torch.from_numpy(w.astype(np.float32)).cuda()
    bd = torch.from_numpy(b.astype(np.float32)).cuda()
    wpk = torch.empty(L.pty_tc_weights_size(Cin, Cout), dtype=torch.bfloat16, device="cuda")
    abi.check(L.pty_tc_pack_weights(_p(wd), Cin, Cout, _p(wpk), None))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    if out_mode == 1:
        y = torch.full((B, Cout, H, W), 12345.0, device="cuda")
    elif out_mode == 2:
        y = torch.zeros((B, H // 2, W // 2, Cout), dtype=torch.bfloat16, device="cuda")
    else:
        y = torch.zeros((B, H, W, Cout), dtype=torch.bfloat16, device="cuda")
    abi.check(L.pty_tc_conv3x3(_p(x_dev), _p(wpk), _p(bd), _p(y), B, Cin, Cout, H, W, relu, in_mode, out_mode,
                               in_scale, _p(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    if out_mode == 1:
        return y.cpu().numpy().astype(np.float64)
    return y.float().cpu().numpy().astype(np.float64).transpose(0, 3, 1, 2)


def _nhwc_bf16(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x.transpose(0, 2, 3, 1), np.float32)).cuda().to(torch.bfloat16)


@pytest.mark.parametrize("B,Cin,Cout,H,W,relu,out_mode", [
    (2, 1, 16, 16, 16, 0, 1),     # thin input (element gather), one K stage of 16
    (3, 16, 32, 13, 13, 1, 1),    # ragged pixel count (507: last CTA partly empty), K = 144 over 3 stages
    (2, 64, 256, 8, 8, 0, 1),     # N = 256, K = 576
    (1, 32, 3, 32, 32, 0, 1),     # N padded 3 -> 16, FP32 NCHW output (the output layer)
    (2, 256, 64, 16, 16, 1, 0),   # K = 2304 (36 stages), NHWC BF16 output
    (1, 8, 24, 12, 20, 1, 0),     # Cin = 8, Cout = 24 (N padded to 32), non-square
    (2, 16, 32, 8, 32, 1, 2),     # pooled output, W = 32 (two column blocks per row pair)
    (3, 32, 64, 6, 16, 0, 2),     # pooled output, W = 16, tiles spanning images
])
def test_tc_conv_matches_numpy(B, Cin, Cout, H, W, relu, out_mode):
    rng = np.random.default_rng(B * 7919 + Cin * 31 + Cout + out_mode)
    x = _bf16_round(rng.standard_normal((B, Cin, H, W)))
    w = _bf16_round(rng.standard_normal((Cout, Cin, 3, 3)) / np.sqrt(Cin * 9))
    b = rng.standard_normal(Cout).astype(np.float32).astype(np.float64)
    ref = nn_ref.conv3x3(x, w, b)
    if relu:
        ref = nn_ref.relu(ref)
    if out_mode == 2:
        ref = nn_ref.pool2(ref)
    xd = _nhwc_bf16(x)
    got = _run_conv(xd, w, b, B, Cin, Cout, H, W, relu, 0, out_mode)
    if out_mode == 1:
        assert rel_err(got, ref) < 1e-5  # exact BF16 products, FP32 sums
    else:
        assert rel_err(got, ref) < 6e-3  # plus the BF16 rounding of the stored output


@pytest.mark.parametrize("B,Cin,Cout,H,W,relu,in_mode,out_mode", [
    (2, 16, 32, 32, 16, 1, 0, 0),   # shifted-GEMM form: Cin = 16, NHWC output, tiles across two images
    (3, 32, 64, 16, 24, 0, 0, 2),   # Cin = 32, pooled output, three tile columns per row block
    (2, 64, 32, 32, 32, 1, 1, 0),   # Cin = 64 read from an upsampled 16 x 16 input (the decoder layer)
    (1, 16, 16, 48, 8, 1, 0, 2),    # one tile column, three tile rows, N = 16
    (2, 16, 32, 64, 64, 1, 0, 2),   # the encoder's second layer at its size
    (2, 32, 3, 32, 32, 0, 0, 1),    # the output layer: N padded 3 -> 16, FP32 NCHW output
    (1, 16, 24, 16, 8, 1, 0, 0),    # Cout = 24 (N padded to 32), NHWC output
    (2, 64, 128, 16, 16, 1, 0, 2),  # 147 KB of weights: one CTA per SM (the encoder's 64 -> 128 layer)
    (2, 256, 64, 16, 16, 1, 1, 0),  # four 64-channel groups streamed per tile, upsampled input (the decoder's first)
    (3, 128, 48, 32, 8, 0, 0, 2),   # two groups, N padded 48, pooled, tiles across images
])
def test_tc_conv_shifted_gemm_form(B, Cin, Cout, H, W, relu, in_mode, out_mode):
    """Thin layers (Cin <= 64, weights resident in shared memory, 16 x 8 pixel tiles) run as nine shifted GEMMs over
    an input halo in shared memory (k_conv_tap); same bounds as the im2col form."""
    rng = np.random.default_rng(B * 131 + Cin * 7 + Cout + 3 * in_mode + out_mode)
    hs, ws = (H // 2, W // 2) if in_mode == 1 else (H, W)
    x = _bf16_round(rng.standard_normal((B, Cin, hs, ws)))
    w = _bf16_round(rng.standard_normal((Cout, Cin, 3, 3)) / np.sqrt(Cin * 9))
    b = rng.standard_normal(Cout).astype(np.float32).astype(np.float64)
    ref = nn_ref.conv3x3(nn_ref.up2(x) if in_mode == 1 else x, w, b)
    if relu:
        ref = nn_ref.relu(ref)
    if out_mode == 2:
        ref = nn_ref.pool2(ref)
    got = _run_conv(_nhwc_bf16(x), w, b, B, Cin, Cout, H, W, relu, in_mode, out_mode)
    # exact BF16 products with FP32 sums; NHWC outputs are also rounded to BF16
    assert rel_err(got, ref) < (1e-5 if out_mode == 1 else 6e-3)


def test_tc_conv_upsampled_input():
    rng = np.random.default_rng(11)
    B, Cin, Cout, h, w_ = 2, 16, 24, 5, 7
    x = _bf16_round(rng.standard_normal((B, Cin, h, w_)))
    w = _bf16_round(rng.standard_normal((Cout, Cin, 3, 3)) / np.sqrt(Cin * 9))
    b = rng.standard_normal(Cout).astype(np.float32).astype(np.float64)
    ref = nn_ref.conv3x3(nn_ref.up2(x), w, b)
    got = _run_conv(_nhwc_bf16(x), w, b, B, Cin, Cout, 2 * h, 2 * w_, 0, 1, 1)
    assert rel_err(got, ref) < 1e-5


def test_tc_conv_amplitude_input():
    import torch

    rng = np.random.default_rng(12)
    B, Cout, H, W = 3, 16, 32, 32
    amp = rng.uniform(0, 50, (B, H, W)).astype(np.float32)
    w = _bf16_round(rng.standard_normal((Cout, 1, 3, 3)) / 3)
    b = rng.standard_normal(Cout).astype(np.float32).astype(np.float64)
    xin = _bf16_round(nn_ref.warm_input(amp, 0.25))[:, None]
    ref = nn_ref.pool2(nn_ref.relu(nn_ref.conv3x3(xin, w, b)))
    got = _run_conv(torch.from_numpy(amp).cuda(), w, b, B, 1, Cout, H, W, 1, 2, 2, 0.25)
    assert rel_err(got, ref) < 6e-3


def test_cuda_core_first_and_last_layers():
    import torch

    from ptychopy_b200 import abi

    L = abi.lib()
    rng = np.random.default_rng(13)
    B, H, W = 2, 40, 36
    amp = rng.uniform(0, 50, (B, H, W)).astype(np.float32)
    w = rng.standard_normal((16, 1, 3, 3)).astype(np.float32) / 3
    b = rng.standard_normal(16).astype(np.float32)
    xin = _bf16_round(nn_ref.warm_input(amp, 0.25))[:, None]
    ref = nn_ref.pool2(nn_ref.relu(nn_ref.conv3x3(xin, _bf16_round(w), b.astype(np.float64))))
    y = torch.zeros((B, H // 2, W // 2, 16), dtype=torch.bfloat16, device="cuda")
    ampd, wd, bd = torch.from_numpy(amp).cuda(), torch.from_numpy(w).cuda(), torch.from_numpy(b).cuda()
    abi.check(L.pty_tc_first_layer(_p(ampd), _p(wd), _p(bd), _p(y), B, 16, H, W, 0.25, None))
    torch.cuda.synchronize()
    assert rel_err(y.float().cpu().numpy().transpose(0, 3, 1, 2), ref) < 6e-3
    # output layer: NHWC BF16 32 channels -> NCHW FP32 3 planes
    x = _bf16_round(rng.standard_normal((B, 32, 12, 10)))
    w3 = rng.standard_normal((3, 32, 3, 3)).astype(np.float32) / 17
    b3 = rng.standard_normal(3).astype(np.float32)
    ref3 = nn_ref.conv3x3(x, _bf16_round(w3), b3.astype(np.float64))
    y3 = torch.zeros((B, 3, 12, 10), device="cuda")
    xd, w3d, b3d = _nhwc_bf16(x), torch.from_numpy(w3).cuda(), torch.from_numpy(b3).cuda()
    abi.check(L.pty_tc_last_layer(_p(xd), _p(w3d), _p(b3d), _p(y3), B, 32, 3, 12, 10, None))
    torch.cuda.synchronize()
    assert rel_err(y3.cpu().numpy(), ref3) < 1e-5


def test_tc_pool_up_match_numpy():
    import torch

    from ptychopy_b200 import abi

    L = abi.lib()
    rng = np.random.default_rng(3)
    x = _bf16_round(rng.standard_normal((2, 8, 6, 16)))  # B, H, W, C (NHWC)
    xd = torch.from_numpy(x.astype(np.float32)).cuda().to(torch.bfloat16)
    p = torch.empty((2, 4, 3, 16), dtype=torch.bfloat16, device="cuda")
    abi.check(L.pty_tc_pool2(_p(xd), _p(p), 2, 4, 3, 16, None))
    u = torch.empty((2, 16, 12, 16), dtype=torch.bfloat16, device="cuda")
    abi.check(L.pty_tc_up2(_p(xd), _p(u), 2, 8, 6, 16, None))
    torch.cuda.synchronize()
    ref_p = nn_ref.pool2(x.transpose(0, 3, 1, 2)).transpose(0, 2, 3, 1)
    assert rel_err(p.float().cpu().numpy(), ref_p) < 6e-3
    ref_u = nn_ref.up2(x.transpose(0, 3, 1, 2)).transpose(0, 2, 3, 1)
    assert rel_err(u.float().cpu().numpy(), ref_u) == 0


def test_tc_network_matches_fp32_network():
    import torch

    from ptychopy_b200 import synth, warmstart

    N = 128
    net = warmstart.Net(N=N, width=16, seed=4)
    dx_s = synth.sample_pixel(2.48e-10, 1.0, 172e-6, N)
    probe = synth.make_probe(N, dx_s, K=1)[0]
    rng = np.random.default_rng(5)
    pos, X, Y = synth.raster_positions(4, 4, 50e-9, 50e-9, dx_s, N)
    obj = synth.make_object(X, Y, rng)
    amp = synth.make_patterns_torch(obj, probe[None], pos, N, 1e5, seed=5)
    ref = warmstart.predict(net, amp, chunk=7)
    tc = warmstart.TcNet(net)
    got = warmstart.predict(tc, amp, chunk=7)
    torch.cuda.synchronize()
    assert rel_err(got.cpu().numpy(), ref.cpu().numpy()) < 3e-2
