"""Learned warm start end to end on the GPU: training on patterns from the library's forward model, inference,
assembly, and what the trained network gains over a flat start for ePIE and DM; plus the DM exit-wave start from a
given object (pty_dm_psi_from_object)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _session(alg, amp, probe, cfg, nx, obj=None):
    import torch

    from ptychopy_b200 import abi, synth

    N = probe.shape[-1]
    s = abi.Session(size=N, scanDimsx=nx, scanDimsy=nx, stepx=cfg["step"], stepy=cfg["step"], lambd=cfg["lambd"],
                    z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1, algorithm=alg)
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    s.set_patterns_ptr(amp.data_ptr(), amp.shape[0], N)
    s.set_probe(probe[None])
    if obj is not None:
        s.set_object(obj)
    s.init()
    return s


def test_dm_psi_from_object_keeps_a_consistent_object():
    import torch

    from ptychopy_b200 import synth

    cfg = dict(synth.CONFIGS["warm128"])
    N, nx = 64, 6
    rng = np.random.default_rng(21)
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = synth.raster_positions(nx, nx, cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=1, fwhm=8 * dx_s)[0]
    starts = np.rint(pos).astype(int)  # DM windows start at the rounded positions
    amp = np.stack([np.abs(np.fft.fft2(probe * obj[r:r + N, c:c + N])) for r, c in starts]).astype(np.float32)
    ampd = torch.from_numpy(amp).cuda()
    kept = _session("DM", ampd, probe, cfg, nx, obj=obj)
    kept.psi_from_object()
    kept.step()
    zero = _session("DM", ampd, probe, cfg, nx, obj=obj)
    zero.step()
    inner = (slice(N // 2, X - N // 2), slice(N // 2, Y - N // 2))
    ref = obj[inner]
    e_kept = np.linalg.norm(kept.object()[inner] - ref) / np.linalg.norm(ref)
    e_zero = np.linalg.norm(zero.object()[inner] - ref) / np.linalg.norm(ref)
    kept.close()
    zero.close()
    assert e_kept < 1e-3, e_kept
    assert e_zero > 0.3, e_zero  # the zero exit-wave start (the reference's) discards the given object


def test_warm_start_training_and_gain():
    import torch

    from ptychopy_b200 import synth, warmstart

    cfg = dict(synth.CONFIGS["warm128"])
    N = cfg["N"]
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    probe = synth.make_probe(N, dx_s, K=1)[0]
    torch.manual_seed(0)
    x, t = warmstart.training_set(probe, n_patterns=8192, N=N, seed=500)
    net = warmstart.Net(N=N, width=16, seed=1)
    hist = warmstart.train(net, x, t, warmstart.loss_weight(probe, N // 4), epochs=3, batch=64)
    del x, t
    assert hist[-1] < hist[0]
    # a test scan: fresh object seed, 24 x 24 raster, 1e5 photons per pattern
    nx = 24
    rng = np.random.default_rng(77)
    pos, X, Y = synth.raster_positions(nx, nx, cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    amp = synth.make_patterns_torch(obj, probe[None], pos, N, cfg["photons"], seed=77)
    mask = np.zeros((X, Y), bool)
    mask[N // 2:X - N // 2, N // 2:Y - N // 2] = True
    s = _session("ePIE", amp, probe, cfg, nx)
    spos = s.positions()
    flat = []
    for _ in range(2):
        s.step()
        flat.append(synth.phase_nrmse(s.object(), obj, mask))
    s.close()
    o0 = warmstart.initial_object(net, amp, spos, probe, X, Y)
    warm0 = synth.phase_nrmse(o0, obj, mask)
    assert warm0 < 0.08, warm0
    assert warm0 < flat[1], (warm0, flat)
    s = _session("ePIE", amp, probe, cfg, nx, obj=o0)
    for _ in range(2):
        s.step()
    warm_epie = synth.phase_nrmse(s.object(), obj, mask)
    s.close()
    assert warm_epie < flat[1], (warm_epie, flat)
    # DM: flat start vs the warm object with its exit waves
    res = {}
    for name, init in (("flat", None), ("warm", o0)):
        s = _session("DM", amp, probe, cfg, nx, obj=init)
        if init is not None:
            s.psi_from_object()
        for _ in range(5):
            s.step()
        res[name] = synth.phase_nrmse(s.object(), obj, mask)
        s.close()
    assert res["warm"] < res["flat"], res


def test_native_warm_start_matches_python_path():
    """pty_set_warm_start + pty_init (C++ inference and assembly inside the session) against warmstart.py on the
    same network, patterns, probe and positions; also through the ptychopy module's warmStart keyword."""
    import torch

    from conftest import rel_err
    from ptychopy_b200 import abi, synth, warmstart

    cfg = dict(synth.CONFIGS["warm128"])
    N, nx = cfg["N"], 12
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    probe = synth.make_probe(N, dx_s, K=1)[0]
    rng = np.random.default_rng(31)
    pos, X, Y = synth.raster_positions(nx, nx, cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    amp = synth.make_patterns_torch(obj, probe[None], pos, N, cfg["photons"], seed=31)
    net = warmstart.Net(N=N, width=16, seed=9)
    params = net.state()
    s = _session("ePIE", amp, probe, cfg, nx)
    spos = s.positions()
    s.close()
    ref = warmstart.initial_object(warmstart.TcNet(net), amp, spos, probe, X, Y)
    for alg in ("ePIE", "DM"):
        kw = dict(size=N, scanDimsx=nx, scanDimsy=nx, stepx=cfg["step"], stepy=cfg["step"], lambd=cfg["lambd"],
                  z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1, algorithm=alg)
        s = abi.Session(**kw)
        s.set_stream(torch.cuda.current_stream().cuda_stream)
        s.set_patterns_ptr(amp.data_ptr(), amp.shape[0], N)
        s.set_probe(probe[None])
        s.set_warm_start(params, 16)
        s.init()
        got = s.object()
        s.close()
        assert rel_err(got, ref) < 1e-5, alg
    # a parameter count that does not match the network is refused at pty_init
    s = abi.Session(size=N, scanDimsx=nx, scanDimsy=nx, stepx=cfg["step"], stepy=cfg["step"], lambd=cfg["lambd"],
                    z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1, algorithm="ePIE")
    s.set_patterns(amp.cpu().numpy())
    s.set_warm_start(params[:-1], 16)
    with pytest.raises(abi.PtyError):
        s.init()
    s.close()
    # the reference-facing module: epienpinit(..., warmStart=params) starts from the same object
    import ptychopy_b200

    ptychopy = ptychopy_b200.import_ptychopy()
    ptychopy.epienpinit(jobID="warm", diffractionNP=amp.cpu().numpy(), probeNP=probe, size=N, scanDimsx=nx,
                        scanDimsy=nx, stepx=cfg["step"], stepy=cfg["step"], lambd=cfg["lambd"], z=cfg["z"],
                        dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, iter=5, warmStart=params, warmStartWidth=16)
    got = ptychopy.epieresobj()
    ptychopy.epiepost()
    assert rel_err(got, ref) < 1e-5
