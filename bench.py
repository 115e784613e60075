#!/usr/bin/env python
"""Benchmark: reference DM at 512^2 over a 30x30 raster (900 positions), patterns/s.

One step = one DM iteration over all 900 patterns (forward propagation, modulus projection, back-propagation,
object/probe update).  `value` is measured with the inputs resident in HBM, CUDA events on the session's
stream, after `--warmup` untimed steps; `e2e` times the public API call (ptychopy.dmnp) end to end with the
patterns in pinned host memory.  Multi-GPU runs (torchrun) are independent replicas, one per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

`--shard` (with torchrun, N GPUs) splits the DM scan's positions over the ranks: each rank steps its share, the
object / probe increments are summed with one NCCL all-reduce per iteration, and every rank applies the sum
(strong scaling: the whole job is the 900-pattern iteration).

`--algo batch` measures the batched configuration: 16 independent scans of uneven sizes (8 DM, 8 MLs; detectors
128-512, rasters 10x10-40x40, steps 30-100 nm), `--steps` iterations each, interleaved by pty_batch_run against
the same scans run one after another; each DM scan's wave size is chosen first by the autotuner (pty_autotune,
reported; `--no-autotune` keeps the defaults).

`--algo mls` measures MLs on one scan of the batched configuration's MLs range (256^2, 20x20 raster, 400 positions,
groups of 4): the reference's default path with every part active (variable probe and intensity, sub-pixel probe
shift, position search), the fixed-probe core beside it, and the FP64 oracle on a bounded sample as the CPU
reference.

`--algo nrmse` measures the plain half of the warm-start comparison: ePIE from a flat (zero) object on the
warm-start workload (64x64 raster at 128^2, 1e5 photons/pattern), iterations and GPU time until the phase NRMSE
(after phase-ramp removal, central region) reaches 0.05.

`--algo warm` measures the whole warm-start comparison on that workload: the encoder-decoder is trained first
(20480 patterns from the forward model on objects of fresh seeds, 6 epochs; reported, not part of the timed
comparison), then plain ePIE from a flat start against the warm start (inference over all 4096 patterns, stitching,
phase integration, energy match, then ePIE iterations only if the warm object is still above 0.05), each as GPU time
to phase NRMSE <= 0.05 checked after every iteration; DM from a flat start and from the warm object (exit waves
P * O) are reported beside them.

`--algo infer` measures the warm-start network's BF16 tensor-core inference alone (the width-16 encoder-decoder,
seeded random weights, on the 4096 patterns of the warm-start workload): patterns/s per forward pass, the FP32
CUDA-core forward beside it, and the roofline of the dominant tcgen05 convolution against the measured BF16 peak.

`--algo fft` measures the precision pattern: the batched 2-D FFT of 900 patterns of 256^2 as split-BF16 tensor-core
GEMM stages (pty_fft2_tc) against the engine's FP32 FFT (pty_fft2_dev), each with its error against numpy's FP64
FFT on a sample.

`--algo epie --cfg epie128|epie256k5|dm512` measures the ePIE configurations instead (10x10 raster at 128^2 with one
probe mode; 51x51 raster at 256^2 with 5 modes; ePIE on the 30x30 raster at 512^2 of the DM configuration): one step = one ePIE iteration over all positions, after enough warm-up
iterations that the probe (iteration 10) and the modes (iteration 20) are being updated.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DM/ePIE patterns/s at 512² (HBM roofline %); time to NRMSE≤0.05 warm vs plain"
UNIT = "patterns/s"
WORKLOAD = ("reference DM, 512x512 detector, 30x30 raster (900 positions), 50 nm step, lambda 2.48e-10 m, "
            "z 1 m, dx_d 172 um, 1 probe mode, object 1027x1027, 1e7 photons/pattern")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=30)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--e2e-iters", type=int, default=100, help="iterations per public-API call (the config's 100)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="--algo batch / epie: keep the default launch variants")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the ePIE 512^2 and warm-start parts of the headline after the DM line")
    ap.add_argument("--batch-scans", default="all", choices=["all", "DM", "MLs"],
                    help="--algo batch: the 16 mixed scans, or only their DM or MLs members")
    ap.add_argument("--nx", type=int, default=30, help="raster size (30 = the DM configuration; smaller for profiling)")
    ap.add_argument("--wave", type=int, default=0, help="DM patterns per pipeline wave (0 = automatic)")
    ap.add_argument("--algo", default="dm", choices=["dm", "epie", "batch", "nrmse", "mls", "warm", "infer", "fft"])
    ap.add_argument("--shard", action="store_true",
                    help="N>1: split the 900 positions over the GPUs (one NCCL all-reduce of the DM increments per "
                         "iteration, strong scaling) instead of independent replicas")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1],
                    help="--algo epie: 1 runs the transforms as split-BF16 tensor-core stages (256^2); --algo dm: "
                         "1 runs the column pass's 32-point DFT stages as split-FP16 tensor-core GEMMs (512^2)")
    ap.add_argument("--cfg", default="epie128", choices=["epie128", "epie256k5", "dm512"],
                    help="ePIE configuration (dm512: ePIE on the 512^2 DM configuration's scan)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """SM clock and throttle-reason samples (NVML) taken while the timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index, interval=0.02):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.ok = False
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            return
        self.interval = interval
        self.stop_ev = threading.Event()
        self.th = threading.Thread(target=self._run, daemon=True)

    def _sample(self):
        try:
            self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
            r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            for bit, name in self.REASONS.items():
                if r & bit:
                    self.reasons.add(name)
        except Exception:
            pass

    def _run(self):
        while not self.stop_ev.is_set():
            self._sample()
            time.sleep(self.interval)

    def start(self):
        if self.ok:
            self._sample()
            self.th.start()

    def stop(self):
        if not self.ok:
            return None
        self.stop_ev.set()
        self.th.join()
        self._sample()
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """DRAM bytes per DM iteration from the committed ncu summary (line `traffic_bytes_per_step: <int>`)."""
    path = os.path.join(ROOT, "profiles", "dm_pipeline_512.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_step:"):
            try:
                return int(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def dataset(device, nx=30):
    """Seeded synthetic DM workload; patterns generated on `device` (torch) to keep set-up short."""
    import numpy as np

    from ptychopy_b200 import synth

    cfg = dict(synth.CONFIGS["dm512"], nx=nx, ny=nx)
    rng = np.random.default_rng(20261204)
    N = cfg["N"]
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=1)
    amp = synth.make_patterns_torch(obj, probe, pos, N, cfg["photons"], seed=20261204, device=device)
    kwargs = dict(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
                  lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1)
    return dict(amp=amp, pos=pos, X=X, Y=Y, probe=probe, kwargs=kwargs, N=N, P=pos.shape[0])


def cpu_port_rate(amp_np, ds, budget_s=15.0, threads=None):
    """The oracle's FP32 multithreaded DM on a bounded sample: returns (patterns/s, threads, sample text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = threads or os.cpu_count() or 1
    pos, X, Y, probe = ds["pos"], ds["X"], ds["Y"], ds["probe"]
    n0 = min(ds["P"], 4 * threads)
    t0, _ = pyoracle.dm_baseline_f32(amp_np[:n0], pos[:n0], probe, X, Y, 1, threads)
    n = int(min(ds["P"], max(n0, budget_s / max(t0 / n0, 1e-9))))
    t, _ = pyoracle.dm_baseline_f32(amp_np[:n], pos[:n], probe, X, Y, 1, threads)
    return n / t, threads, f"1 DM iteration over {n} of the 900 patterns (512^2, FP32, {threads} threads)"


def run_reference(args, rank):
    if rank != 0:
        return
    import numpy as np

    try:
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
    except Exception:
        dev = None
    if dev is None:
        print(json.dumps({"impl": "reference", "unavailable": "torch is required to generate the dataset"}))
        return
    ds = dataset(dev)
    amp_np = ds["amp"].cpu().numpy().astype(np.float32)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle

    threads = os.cpu_count() or 1
    # calibrate the per-step sample so the whole run stays within a few minutes
    n0 = min(ds["P"], 4 * threads)
    t0, _ = pyoracle.dm_baseline_f32(amp_np[:n0], ds["pos"][:n0], ds["probe"], ds["X"], ds["Y"], 1, threads)
    per = t0 / n0
    budget = max(1.0, 150.0 / max(args.steps + args.warmup, 1))
    n = int(min(ds["P"], max(n0, budget / per)))
    rates = []
    for i in range(args.warmup + args.steps):
        t, _ = pyoracle.dm_baseline_f32(amp_np[:n], ds["pos"][:n], ds["probe"], ds["X"], ds["Y"], 1, threads)
        if i >= args.warmup:
            rates.append(n / t)
    value = statistics.median(rates)
    sample = f"1 DM iteration over {n} of the 900 patterns per step (512^2, FP32 C++ port, {threads} threads)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * n / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "N": 512, "positions": 900, "object": [ds["X"], ds["Y"]],
                   "step": "one DM iteration over all 900 patterns",
                   "l2": "inputs larger than L2 (exit waves 1.89 GB + amplitudes 0.94 GB per step)",
                   "parallelism": "replicas" if args.gpus > 1 else "single GPU"},  # as the GPU arm's config
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's CUDA sources do not build with CUDA 12.9; its DM is restated as a multithreaded "
                "FP32 C++ port of the same equations",
    }))


class _DeviceBuf:
    """A float32 view of a complex64 device buffer (length 2n) for torch, through __cuda_array_interface__."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (2 * n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def _device_view(ptr, n):
    import torch

    return torch.as_tensor(_DeviceBuf(ptr, n), device="cuda")


def run_b200(args, rank, world, local):
    import numpy as np
    import torch

    from ptychopy_b200 import abi

    torch.cuda.set_device(local)
    dist = None
    if world > 1 or args.shard:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    ds = dataset("cuda", args.nx)
    N, P = ds["N"], ds["P"]
    stream = torch.cuda.Stream()
    shard = args.shard
    s = abi.Session(**dict(ds["kwargs"], algorithm="DM", device=local, wave=args.wave, precision=args.precision))
    s.set_stream(stream.cuda_stream)
    if shard:
        bounds = [P * r // world for r in range(world + 1)]
        first, count = bounds[rank], bounds[rank + 1] - bounds[rank]
        s.set_shard(first, P)
        s.set_patterns_ptr(ds["amp"][first:first + count].data_ptr(), count, N)
        s.set_probe(ds["probe"])
        dO_ptr, n_obj, dP_ptr, n_probe = None, 0, None, 0
    else:
        s.set_patterns_ptr(ds["amp"].data_ptr(), P, N)
    s.init()
    if shard:
        dO_ptr, n_obj, dP_ptr, n_probe = s.increments()
        t_dO, t_dP = _device_view(dO_ptr, n_obj), _device_view(dP_ptr, n_probe)

        def step():
            s.step_local()
            with torch.cuda.stream(stream):
                dist.all_reduce(t_dO)
                dist.all_reduce(t_dP)
            s.step_finish()
    else:
        step = s.step
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    l0 = s.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.start()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
    stream.synchronize()
    ck = clocks.stop()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = s.launches() - l0
    obj = s.object()
    finite = bool(np.isfinite(obj).all())
    s.close()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = P * args.steps * (1 if shard else world) / (ms_max / 1000.0)
    ms_step = ms_max / args.steps

    if args.no_e2e or shard:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms_step, "steps": args.steps,
                              "positions": P, "gpu_launches": int(launches), "finite": finite, "clocks": ck,
                              "n_gpus": world, "scaling": "strong" if shard else "weak",
                              "note": "partial run (--no-e2e)" if not shard else
                                      "positions sharded over the GPUs, one NCCL all-reduce of the increments "
                                      "per iteration"}), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    # end to end through the public API: pinned host patterns -> dmnp(iter=...) -> object/probe on the host
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    host = torch.empty((P, N, N), dtype=torch.float32, pin_memory=True)
    host.copy_(ds["amp"])
    amp_host = host.numpy()
    del ds["amp"]
    torch.cuda.empty_cache()
    kw = dict(ds["kwargs"], iter=args.e2e_iters, returnResults=1, writeResults=0, device=local, wave=args.wave,
              precision=args.precision)
    pt.dmnp(diffractionNP=amp_host, **dict(kw, iter=2))  # warm-up call
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    res = None
    for _ in range(args.e2e_calls):
        res = pt.dmnp(diffractionNP=amp_host, **kw)
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = P * args.e2e_iters * args.e2e_calls * world / float(t.item())
    d2h = res[0].nbytes + res[1].nbytes

    if rank == 0:
        peak, kind = peaks()
        XY = ds["X"] * ds["Y"]
        bytes_step = 20 * N * N * P + 16 * XY + 16 * N * N  # psi r+w, A r; object/probe pass
        achieved = bytes_step / (ms_step / 1000.0) / 1e9
        traffic = profiled_traffic()
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (column DFT stages split-FP16 on tensor cores)" if args.precision else "f32",
            "data": "synthetic (seeded; object GRF phase, 110 nm probe, Poisson)",
            "config": {"workload": WORKLOAD if args.nx == 30 else f"{WORKLOAD} (raster {args.nx}x{args.nx})",
                       "N": N, "positions": P, "object": [ds["X"], ds["Y"]],
                       "step": "one DM iteration over all 900 patterns",
                       "l2": "inputs larger than L2 (exit waves 1.89 GB + amplitudes 0.94 GB per step)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": kind,
                         "kernel": "DM iteration graph (k_dm_rows, %s, k_dm_inv per wave + finalize)"
                                   % ("k_dm_cols_tc" if args.precision else "k_dm_cols"),
                         "algorithmic_bytes_per_step": bytes_step},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(amp_host.nbytes) // args.e2e_iters,
                    "d2h_bytes_per_step": int(d2h) // args.e2e_iters,
                    "h2d_bytes_per_call": int(amp_host.nbytes), "d2h_bytes_per_call": int(d2h),
                    "step": f"one DM iteration; each ptychopy.dmnp(iter={args.e2e_iters}) call uploads the patterns "
                            "from pinned host memory once and returns object and probe to the host, so the per-step "
                            "copies are the call's divided by its iterations"},
            "gpu_launches": int(launches), "clocks": ck, "finite": finite,
        }
        if world == 1 and not args.no_cpu:
            rate, cores, sample = cpu_port_rate(amp_host, ds)
            out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
        if world == 1 and not args.no_extras:
            out["headline_parts"] = headline_parts(args, rank, local)
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def headline_parts(args, rank, local):
    """The other two parts of the headline metric, measured after the DM line at N = 1: ePIE at 512^2 (the DM
    configuration's scan) and the time to phase NRMSE <= 0.05 with the learned warm start vs plain ePIE.  Each is
    the summary of its own bench mode (--algo epie --cfg dm512, --algo warm); a failure is reported, not raised."""
    parts = {}
    try:
        a = argparse.Namespace(**dict(vars(args), cfg="dm512", steps=3, warmup=21, no_cpu=True))
        r = run_epie(a, rank, local, emit=False)
        parts["epie_512"] = {"value": round(r["value"], 1), "unit": r["unit"], "ms_per_step": round(r["ms_per_step"], 3),
                             "roofline_frac": round(r["roofline"]["frac"], 4), "command": "bench.py --algo epie --cfg dm512"}
    except Exception as e:  # noqa: BLE001
        parts["epie_512"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        import torch

        torch.cuda.empty_cache()
        a = argparse.Namespace(**dict(vars(args), steps=300))
        r = run_warm(a, rank, local, emit=False)
        parts["warm_vs_plain"] = {
            "metric": "GPU time to phase NRMSE <= 0.05", "unit": "ms", "warm": r["value"],
            "plain": r["plain"]["reached"]["gpu_ms"] if r["plain"]["reached"] else None,
            "plain_iterations": r["plain"]["reached"]["iterations"] if r["plain"]["reached"] else None,
            "warm_object_nrmse": r["warm"]["warm_object_nrmse"],
            "e2e_ms": {"warm": r["e2e"]["value"], "plain": r["e2e"]["plain_ms"]} if r.get("e2e") else None,
            "command": "bench.py --algo warm"}
    except Exception as e:  # noqa: BLE001
        parts["warm_vs_plain"] = {"error": f"{type(e).__name__}: {e}"}
    return parts


def run_epie(args, rank, local, emit=True):
    """ePIE throughput on one of the ePIE configurations (device-timed steps, oracle FP32 port as CPU baseline)."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth

    torch.cuda.set_device(local)
    cfg = dict(synth.CONFIGS[args.cfg])
    N, K = cfg["N"], cfg["K"]
    rng = np.random.default_rng(20261205)
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=K)
    amp = synth.make_patterns_torch(obj, probe, pos, N, cfg["photons"], seed=20261205, device="cuda")
    P = pos.shape[0]
    kwargs = dict(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
                  lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=K,
                  algorithm="ePIE", device=local, precision=args.precision)
    stream = torch.cuda.Stream()
    s = abi.Session(**kwargs)
    s.set_stream(stream.cuda_stream)
    s.set_patterns_ptr(amp.data_ptr(), P, N)
    tuning = None
    if not args.no_autotune and not args.precision:  # pick the launch variant (pty_autotune), reported
        t0 = time.perf_counter()
        tuning = {"choice": s.autotune(iters=1), "seconds": round(time.perf_counter() - t0, 3)}
    s.init()
    warm = max(args.warmup, 21)
    for _ in range(warm):
        s.step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    l0 = s.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.start()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            s.step()
        e1.record(stream)
    stream.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = s.launches() - l0
    finite = bool(np.isfinite(s.object()).all())
    s.close()
    value = P * args.steps / (ms / 1000.0)
    peak, kind = peaks()
    bytes_pattern = 4 * N * N + 16 * N * N * (1 + K)  # A; object patch r+w; probe modes r+w (probe updating)
    achieved = bytes_pattern * value / 1e9
    out = {"metric": "ePIE patterns/s", "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": warm, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "dtype": "f32 (transforms split-BF16 on tensor cores)" if args.precision else "f32",
           "data": "synthetic (seeded)",
           "config": {"workload": f"ePIE {args.cfg}: {cfg['nx']}x{cfg['ny']} raster ({P} positions), {N}x{N} "
                                  f"detector, {K} probe mode(s), object {X}x{Y}", "N": N, "positions": P, "modes": K},
           "roofline": {"bound": "latency (serial positions)", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "peak_kind": kind, "kernel": ("per-position kernel chain with tensor-core transforms" if args.precision
                                                           else "the autotuned ePIE launch variant"),
                        "algorithmic_bytes_per_pattern": bytes_pattern},
           "gpu_launches": int(launches), "clocks": ck, "finite": finite,
           "autotune": tuning if tuning else ("tensor-core chain (precision=1)" if args.precision else "off")}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        amp_np = amp.cpu().numpy()
        threads = 1  # the port's ePIE is serial over positions, like the method
        n = min(P, 16)
        o = pyoracle.OracleSession("ePIE", amp_np[:n], pos[:n], np.zeros((X, Y)), probe, probe_guess_path=False,
                                   modes_given=K > 1, nthreads=threads, fp32=True)
        t0 = time.perf_counter()
        o.step()
        per = (time.perf_counter() - t0) / n
        n = int(min(P, max(n, 15.0 / max(per, 1e-9))))
        o = pyoracle.OracleSession("ePIE", amp_np[:n], pos[:n], np.zeros((X, Y)), probe, probe_guess_path=False,
                                   modes_given=K > 1, nthreads=threads, fp32=True)
        t0 = time.perf_counter()
        o.step()
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / t, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"iteration 1 of ePIE over {n} of the {P} positions (FP32 C++ port, "
                                         "no probe update yet)"}
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_mls(args, rank, local):
    """MLs throughput on a 256^2, 20x20 scan (device-timed iterations): the reference's default path (variable probe
    and intensity, sub-pixel probe shift, position search) with every part active, the fixed-probe core beside it;
    the FP64 oracle's default path on a sample as CPU reference."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth

    torch.cuda.set_device(local)
    N, nx, step = 256, 20, 60e-9
    lambd, z, dx_d = 2.48e-10, 1.0, 172e-6
    rng = np.random.default_rng(20261208)
    dx_s = synth.sample_pixel(lambd, z, dx_d, N)
    pos, X, Y = synth.raster_positions(nx, nx, step, step, dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=1)
    intens = synth.make_patterns_torch(obj, probe, pos, N, 1e6, seed=20261208, device="cuda", intensities=True)
    P = pos.shape[0]
    stream = torch.cuda.Stream()
    pps = 3  # position search from iteration 3: with >= 3 warm-up iterations every timed one runs all parts

    def timed(core):
        s = abi.Session(size=N, scanDimsx=nx, scanDimsy=nx, stepx=step, stepy=step, lambd=lambd, z=z, dx_d=dx_d,
                        beamSize=synth.BEAM_FWHM, probeModes=1, algorithm="MLs", delta_p=0.1, device=local,
                        mlsCore=core, PPS=pps)
        s.set_stream(stream.cuda_stream)
        s.set_patterns_ptr(intens.data_ptr(), P, N)
        s.set_probe(probe)
        s.init()
        for _ in range(max(args.warmup, 3)):
            s.run(1)
        torch.cuda.synchronize()
        clocks = Clocks(local)
        l0 = s.launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks.start()
        with torch.cuda.stream(stream):
            e0.record(stream)
            s.run(args.steps)
            e1.record(stream)
        stream.synchronize()
        ck = clocks.stop()
        ms = e0.elapsed_time(e1)
        launches = s.launches() - l0
        finite = bool(np.isfinite(s.object()).all())
        s.close()
        return ms, launches, ck, finite

    ms, launches, ck, finite = timed(0)
    ms_core, _, _, _ = timed(1)
    G = max(1, P // 100)
    out = {"metric": "MLs patterns/s", "value": P * args.steps / (ms / 1000.0), "unit": UNIT, "n_gpus": 1,
           "steps": args.steps, "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f32",
           "data": "synthetic (seeded)",
           "config": {"workload": f"MLs, the reference's default path (variable probe and intensity, sub-pixel probe "
                                  f"shift, position search from iteration {pps}), {N}^2, {nx}x{nx} raster ({P} "
                                  f"positions, groups of {G}), delta_p 0.1", "N": N, "positions": P},
           "core": {"value": P * args.steps / (ms_core / 1000.0), "ms_per_step": ms_core / args.steps,
                    "path": "fixed-probe core (mlsCore=1)"},
           "gpu_launches": int(launches), "clocks": ck, "finite": finite,
           "timing": "CUDA events around pty_run (the host builds each iteration's group tables while the GPU runs)"}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        raw = pyoracle.mls_raw_positions(nx, nx, step, step, dx_s)
        n = 16
        sub = intens[:n].cpu().numpy().astype(np.float64)
        o = pyoracle.OracleMls(raw[:n], sub, probe[0], variable=1, PPS=1)
        t0 = time.perf_counter()
        o.step()
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / t, "unit": UNIT, "cores": 1, "kind": "port",
                               "sample": f"1 MLs iteration of the FP64 oracle's default path (position search on) "
                                         f"over {n} of the {P} positions"}
    print(json.dumps(out), flush=True)


def run_nrmse(args, rank, local):
    """Plain ePIE from a flat start on the warm-start workload: iterations and GPU time to phase NRMSE <= 0.05."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth

    torch.cuda.set_device(local)
    cfg = dict(synth.CONFIGS["warm128"])
    N = cfg["N"]
    rng = np.random.default_rng(20261207)
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    obj = synth.make_object(X, Y, rng)
    probe = synth.make_probe(N, dx_s, K=1)
    amp = synth.make_patterns_torch(obj, probe, pos, N, cfg["photons"], seed=20261207, device="cuda")
    P = pos.shape[0]
    stream = torch.cuda.Stream()
    s = abi.Session(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
                    lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1,
                    algorithm="ePIE", device=local)
    s.set_stream(stream.cuda_stream)
    s.set_patterns_ptr(amp.data_ptr(), P, N)
    s.set_probe(probe)
    s.init()
    mask = np.zeros((X, Y), bool)
    mask[N // 2:X - N // 2, N // 2:Y - N // 2] = True
    gpu_ms, history, reached = 0.0, [], None
    max_iters, chunk = max(args.steps, 5), 5
    it = 0
    while it < max_iters:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(chunk):
                s.step()
            e1.record(stream)
        stream.synchronize()
        gpu_ms += e0.elapsed_time(e1)
        it += chunk
        err = synth.phase_nrmse(s.object(), obj, mask)
        history.append([it, round(gpu_ms, 3), err])
        if err <= 0.05 and reached is None:
            reached = {"iterations": it, "gpu_ms": gpu_ms}
            break
    s.close()
    print(json.dumps({"metric": "time to phase NRMSE <= 0.05, plain ePIE from a flat start", "unit": "ms",
                      "value": reached["gpu_ms"] if reached else None, "higher_is_better": False,
                      "reached": reached, "history": history, "positions": P,
                      "config": {"workload": f"warm-start workload without the warm start: {cfg['nx']}x{cfg['ny']} "
                                             f"raster ({P} positions), {N}^2, 1e5 photons/pattern, object {X}x{Y}, "
                                             "true probe given, zero object",
                                 "nrmse": "phase NRMSE after offset and linear-ramp removal over the central region "
                                          "(N/2 margin), checked every 5 iterations"},
                      "note": "the plain half of the comparison; bench.py --algo warm measures both halves"}),
          flush=True)


def run_warm(args, rank, local, emit=True):
    """Time to phase NRMSE <= 0.05 on the warm-start workload: learned warm start vs plain ePIE from a flat start."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth, warmstart

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    cfg = dict(synth.CONFIGS["warm128"])
    N, target = cfg["N"], 0.05
    max_iters = max(args.steps, 10) if args.steps != 300 else 40
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    probe = synth.make_probe(N, dx_s, K=1)[0]
    clocks = Clocks(local)
    with torch.cuda.stream(stream):
        # ---- training (one-off; wall clock) ----
        t0 = time.time()
        x, t = warmstart.training_set(probe, n_patterns=20480, N=N, seed=1000)
        net = warmstart.Net(N=N, width=16, seed=0)
        hist = warmstart.train(net, x, t, warmstart.loss_weight(probe, N // 4), epochs=6, batch=64)
        stream.synchronize()
        train_s = time.time() - t0
        del x, t
        # ---- the scan (same data as --algo nrmse) ----
        rng = np.random.default_rng(20261207)
        pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
        obj = synth.make_object(X, Y, rng)
        amp = synth.make_patterns_torch(obj, probe[None], pos, N, cfg["photons"], seed=20261207, device="cuda")
        P = pos.shape[0]
    mask = np.zeros((X, Y), bool)
    mask[N // 2:X - N // 2, N // 2:Y - N // 2] = True

    def session(alg, init=None):
        s = abi.Session(size=N, scanDimsx=cfg["nx"], scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"],
                        lambd=cfg["lambd"], z=cfg["z"], dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1,
                        algorithm=alg, device=local)
        s.set_stream(stream.cuda_stream)
        s.set_patterns_ptr(amp.data_ptr(), P, N)
        s.set_probe(probe[None])
        if init is not None:
            s.set_object(init)
        s.init()
        return s

    def iterate(s, gpu_ms, it0):
        """Step until the phase NRMSE reaches the target (checked after every iteration) or max_iters."""
        history, it = [], it0
        while it < max_iters:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                s.step()
            e1.record(stream)
            stream.synchronize()
            gpu_ms += e0.elapsed_time(e1)
            it += 1
            err = synth.phase_nrmse(s.object(), obj, mask)
            history.append([it, round(gpu_ms, 3), round(err, 5)])
            if err <= target:
                return {"iterations": it, "gpu_ms": round(gpu_ms, 3)}, history
        return None, history

    out = {"metric": "time to phase NRMSE <= 0.05: learned warm start vs plain ePIE from a flat start", "unit": "ms",
           "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
           "positions": P}
    clocks.start()
    # plain ePIE from a flat start
    s = session("ePIE")
    spos = s.positions()
    plain, plain_hist = iterate(s, 0.0, 0)
    s.close()
    # warm start: inference + assembly timed on the stream, then ePIE only while above the target.  Inference runs
    # on the BF16 tensor-core copy of the network (all 4096 patterns in one batch); the FP32 CUDA-core network is
    # timed beside it for reference.
    with torch.cuda.stream(stream):
        tc = warmstart.TcNet(net)

        def warm_object(model, chunk):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record(stream)
            net_out = warmstart.predict(model, amp, chunk=chunk)
            ev[1].record(stream)
            o = warmstart.assemble(net_out, spos, probe, X, Y, amp)
            ev[2].record(stream)
            stream.synchronize()
            return o, ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

        for _ in range(3):  # warm-up
            warm_object(tc, P)
            warm_object(net, 256)
        o32, infer32_ms, _ = warm_object(net, 256)
        err32 = synth.phase_nrmse(o32.cpu().numpy().view(np.complex64)[..., 0], obj, mask)
        o, infer_ms, assemble_ms = warm_object(tc, P)
        t0 = time.time()
        o0 = o.cpu().numpy().view(np.complex64)[..., 0].copy()
        handoff_ms = (time.time() - t0) * 1e3
    warm_err = synth.phase_nrmse(o0, obj, mask)
    warm_ms = infer_ms + assemble_ms
    if warm_err <= target:
        warm = {"iterations": 0, "gpu_ms": round(warm_ms, 3)}
        s = session("ePIE", o0)
        _, warm_hist = iterate(s, warm_ms, 0)  # refinement trajectory, for the record
        warm_hist = warm_hist[:10]
    else:
        s = session("ePIE", o0)
        warm, warm_hist = iterate(s, warm_ms, 0)
    s.close()
    # DM beside them: flat start, and the warm object with exit waves P * O
    dm = {}
    for name, init in (("flat", None), ("warm", o0)):
        s = session("DM", init)
        if init is not None:
            s.psi_from_object()
        r, h = iterate(s, warm_ms if init is not None else 0.0, 0)
        dm[name] = {"reached": r, "history": h if len(h) <= 8 else h[:5] + h[-3:]}
        s.close()
    # end to end through the reference-facing module with host arrays: plain epienp for the iterations the plain
    # arm needed vs epienpinit(warmStart=...) + epieresobj; host wall clock, one untimed call of each first
    e2e = None
    if plain and warm:
        import ptychopy_b200

        ptychopy = ptychopy_b200.import_ptychopy()
        amp_h = amp.cpu().numpy()
        params = net.state()
        common = dict(jobID="warm_e2e", diffractionNP=amp_h, probeNP=probe, size=N, scanDimsx=cfg["nx"],
                      scanDimsy=cfg["ny"], stepx=cfg["step"], stepy=cfg["step"], lambd=cfg["lambd"], z=cfg["z"],
                      dx_d=cfg["dx_d"], beamSize=synth.BEAM_FWHM, probeModes=1, device=local)

        def plain_call():
            o, _ = ptychopy.epienp(iter=plain["iterations"], returnResults=1, writeResults=0, **common)
            return o

        def warm_call():
            ptychopy.epienpinit(iter=max(warm["iterations"], 1), warmStart=params, warmStartWidth=16, writeResults=0,
                                **common)
            for _ in range(warm["iterations"]):
                ptychopy.epiestep()
            o = ptychopy.epieresobj()
            ptychopy.epiepost(writeResults=0)
            return o

        times = {}
        for name, fn in (("plain", plain_call), ("warm", warm_call)):
            fn()
            torch.cuda.synchronize()
            t0 = time.time()
            o = fn()
            torch.cuda.synchronize()
            times[name] = ((time.time() - t0) * 1e3, synth.phase_nrmse(o, obj, mask))
        e2e = {"value": round(times["warm"][0], 2), "unit": "ms", "plain_ms": round(times["plain"][0], 2),
               "warm_nrmse": round(times["warm"][1], 5), "plain_nrmse": round(times["plain"][1], 5),
               "h2d_bytes_per_step": int(amp_h.nbytes), "d2h_bytes_per_step": int(X * Y * 8),
               "call": "ptychopy.epienp(iter=plain iterations) vs ptychopy.epienpinit(warmStart=...) + epieresobj, "
                       "host arrays, session set-up included"}
    clk = clocks.stop()
    if plain and not args.no_cpu:
        # the reference's method on the host: the oracle's FP32 ePIE port over a bounded sample of the positions,
        # scaled to the positions x iterations the plain GPU arm needed to reach the target
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle

        amp_np = amp.cpu().numpy()
        n = min(P, 16)
        for _ in range(2):
            o = pyoracle.OracleSession("ePIE", amp_np[:n], pos[:n], np.zeros((X, Y)), probe[None],
                                       probe_guess_path=False, modes_given=False, nthreads=1, fp32=True)
            t0 = time.perf_counter()
            o.step()
            t = time.perf_counter() - t0
            if t > 10.0 or n == P:
                break
            n = int(min(P, max(n, 15.0 * n / max(t, 1e-9))))
        cpu_ms = t / n * P * plain["iterations"] * 1e3
        out["cpu_baseline"] = {"value": round(cpu_ms, 1), "unit": "ms", "cores": 1, "kind": "port",
                               "sample": f"iteration 1 of ePIE over {n} of the {P} positions (FP32 C++ port), "
                                         f"scaled to {P} positions x the {plain['iterations']} iterations plain "
                                         "ePIE needs to reach the target"}
    out.update({
        "e2e": e2e,
        "value": warm["gpu_ms"] if warm else None,
        "plain": {"reached": plain, "history": plain_hist},
        "warm": {"reached": warm, "infer_ms": round(infer_ms, 3), "assemble_ms": round(assemble_ms, 3),
                 "inference": "BF16 tcgen05 implicit-GEMM convolutions, FP32 accumulation, 4096 patterns per batch",
                 "warm_object_nrmse": round(warm_err, 5), "handoff_d2h_ms": round(handoff_ms, 3),
                 "fp32_cuda_core_infer_ms": round(infer32_ms, 3), "fp32_warm_object_nrmse": round(err32, 5),
                 "refinement_history": warm_hist},
        "dm": dm,
        "training": {"patterns": 20480, "epochs": 6, "batch": 64, "wall_s": round(train_s, 2),
                     "loss_per_epoch": [round(v, 5) for v in hist], "parameters": net.n_params,
                     "data": "pty_simulate at integer positions on objects of seeds 1000-1004, Poisson 1e5"},
        "clocks": clk,
        "config": {"workload": f"learned warm start: {cfg['nx']}x{cfg['ny']} raster ({P} positions), {N}^2, 50 nm "
                               f"step, 1e5 photons/pattern, object {X}x{Y}, true probe given",
                   "nrmse": "phase NRMSE after offset and linear-ramp removal over the central region (N/2 margin), "
                            "after every iteration",
                   "timing": "GPU time (CUDA events on the session's stream) of inference + assembly and of each "
                             "iteration; session set-up and the object hand-off (host copy, reported) excluded in "
                             "both arms"},
    })
    if emit:
        print(json.dumps(out), flush=True)
    return out


def run_infer(args, rank, local):
    """Warm-start network inference throughput: BF16 tcgen05 convolutions vs the FP32 CUDA-core network."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth, warmstart

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    cfg = dict(synth.CONFIGS["warm128"])
    N = cfg["N"]
    steps, warmup = max(args.steps if args.steps != 300 else 20, 1), max(args.warmup if args.warmup != 30 else 3, 1)
    dx_s = synth.sample_pixel(cfg["lambd"], cfg["z"], cfg["dx_d"], N)
    probe = synth.make_probe(N, dx_s, K=1)
    rng = np.random.default_rng(20261207)
    pos, X, Y = synth.raster_positions(cfg["nx"], cfg["ny"], cfg["step"], cfg["step"], dx_s, N)
    with torch.cuda.stream(stream):
        amp = synth.make_patterns_torch(synth.make_object(X, Y, rng), probe, pos, N, cfg["photons"], seed=20261207)
        P = amp.shape[0]
        net = warmstart.Net(N=N, width=16, seed=0)
        tc = warmstart.TcNet(net)
        out = torch.empty((P, 3, N // 4, N // 4), device="cuda")
        for _ in range(warmup):
            warmstart.predict(tc, amp, chunk=P, out=out)
        stream.synchronize()
        clocks = Clocks(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            tc.forward_amp(amp, P, out)
        e1.record(stream)
        stream.synchronize()
        clk = clocks.stop()
        tc.check()
        ms = e0.elapsed_time(e1) / steps
        # the dominant tensor-core layer (256 -> 256 channels at 8 x 8) timed alone for the roofline
        L = abi.lib()
        l5 = 5
        cin, cout, H = net.plan[l5][0], net.plan[l5][1], net.plan[l5][2]
        xin = torch.zeros((P, H, H, cin), dtype=torch.bfloat16, device="cuda")
        y = torch.empty((P, H, H, cout), dtype=torch.bfloat16, device="cuda")

        def layer():
            abi.check(L.pty_tc_conv3x3(warmstart._p(xin), warmstart._p(tc.wpk[l5]),
                                       warmstart._p(net._b(net.params, l5)), warmstart._p(y), P, cin, cout, H, H, 1,
                                       0, 0, 1.0, warmstart._p(tc.err), warmstart._stream()))

        for _ in range(3):
            layer()
        e0.record(stream)
        for _ in range(10):
            layer()
        e1.record(stream)
        stream.synchronize()
        layer_ms = e0.elapsed_time(e1) / 10
        flops = 2.0 * P * H * H * cout * cin * 9
        e0.record(stream)
        warmstart.predict(net, amp, chunk=256, out=out)
        e1.record(stream)
        stream.synchronize()
        fp32_ms = e0.elapsed_time(e1)
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    pk = {"bf16_tflops": 1590.0, "source": "fallback"}
    if os.path.exists(path):
        with open(path) as f:
            pk = {"bf16_tflops": float(json.load(f)["bf16_tflops"]), "source": "measured (burst)"}
    achieved = flops / (layer_ms * 1e-3) / 1e12
    total_flops = sum(2.0 * P * h * h * co * ci * 9 for ci, co, h, _r, _a in net.plan)
    print(json.dumps({
        "metric": "warm-start network inference, patterns/s (BF16 tcgen05)", "value": round(P / (ms * 1e-3), 1),
        "unit": "patterns/s", "higher_is_better": True, "n_gpus": 1, "steps": steps, "warmup": warmup,
        "ms_per_step": round(ms, 4), "dtype": "bf16", "data": "synthetic", "scaling": "weak", "vs_baseline": None,
        "network_tflops": round(total_flops / (ms * 1e-3) / 1e12, 1),
        "fp32_cuda_core_ms_per_step": round(fp32_ms, 3),
        "roofline": {"bound": "tensor", "kernel": "k_conv_tc (256 -> 256 channels, 8 x 8, 4096 patterns)",
                     "achieved": round(achieved, 1), "peak": pk["bf16_tflops"], "peak_source": pk["source"],
                     "unit": "TFLOP/s", "frac": round(achieved / pk["bf16_tflops"], 4), "layer_ms": round(layer_ms, 4),
                     "traffic": None},
        "clocks": clk,
        "config": {"workload": f"width-16 encoder-decoder (1.15 M parameters), {P} patterns of {N}^2, one batch",
                   "timing": "CUDA events over one forward pass of all patterns, inputs resident in HBM"},
    }), flush=True)


def run_fft(args, rank, local):
    """Split-BF16 tensor-core 2-D FFT vs the FP32 FFT: time per batch and error vs FP64."""
    if rank != 0:
        return
    import ctypes

    import numpy as np
    import torch

    from ptychopy_b200 import abi

    torch.cuda.set_device(local)
    L = abi.lib()
    B, N = 900, 256
    steps = args.steps if args.steps != 300 else 20
    g = torch.Generator(device="cuda")
    g.manual_seed(20261209)
    base = torch.randn((B, N, N, 2), generator=g, device="cuda")
    d = base.clone()
    w = torch.empty_like(d)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def tc():
        abi.check(L.pty_fft2_tc(p(d), p(w), B, N, 0, p(err), ctypes.c_void_p(stream)))

    def fp32():
        abi.check(L.pty_fft2_dev(p(d), p(w), B, N, 0, ctypes.c_void_p(stream)))

    res = {}
    for name, fn in (("tensor_core_split_bf16", tc), ("fp32", fp32)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # error on a 2-pattern sample against numpy's FP64 FFT
        d.copy_(base)
        fn()
        torch.cuda.synchronize()
        got = d[:2].cpu().numpy().view(np.complex64)[..., 0].astype(np.complex128)
        src = base[:2].cpu().numpy().view(np.complex64)[..., 0].astype(np.complex128)
        exact = np.fft.fft2(src)
        rel = float(np.linalg.norm(got - exact) / np.linalg.norm(exact))
        algo_bytes = 2 * 16.0 * N * N * B  # two passes, each reading and writing every element once
        res[name] = {"ms_per_batch": round(ms, 4), "patterns_per_s": round(B / (ms * 1e-3), 1),
                     "algorithmic_GBps": round(algo_bytes / (ms * 1e-3) / 1e9, 1), "rel_err_vs_fp64": rel}
        d.copy_(base)
    assert int(err.item()) == 0, "tensor-core FFT wait timed out"
    print(json.dumps({"metric": "batched 2-D FFT, patterns/s (split-BF16 tensor cores vs FP32)",
                      "value": res["tensor_core_split_bf16"]["patterns_per_s"], "unit": "patterns/s",
                      "higher_is_better": True, "n_gpus": 1, "steps": steps, "dtype": "bf16x3 / f32",
                      "data": "synthetic (seeded normal)", "results": res,
                      "config": {"workload": f"{B} patterns of {N}^2 complex64, forward, unnormalised",
                                 "timing": "CUDA events over repeated calls; pty_fft2_dev includes its twiddle "
                                           "table set-up per call"}}), flush=True)


BATCH_SCANS = [  # (algorithm, N, raster, step m)
    ("DM", 128, 10, 30e-9), ("DM", 128, 20, 50e-9), ("DM", 256, 15, 60e-9), ("DM", 256, 25, 80e-9),
    ("DM", 512, 10, 50e-9), ("DM", 512, 20, 100e-9), ("DM", 128, 40, 40e-9), ("DM", 256, 30, 70e-9),
    ("MLs", 128, 12, 50e-9), ("MLs", 128, 24, 30e-9), ("MLs", 256, 10, 100e-9), ("MLs", 256, 20, 60e-9),
    ("MLs", 512, 12, 80e-9), ("MLs", 128, 35, 40e-9), ("MLs", 256, 16, 50e-9), ("MLs", 512, 10, 100e-9),
]


def run_batch(args, rank, local):
    """Aggregate patterns/s of 16 uneven scans run through pty_batch_run vs one after another."""
    if rank != 0:
        return
    import numpy as np
    import torch

    from ptychopy_b200 import abi, synth

    torch.cuda.set_device(local)
    lambd, z, dx_d = 2.48e-10, 1.0, 172e-6
    sessions, total_p, keep, tuning = [], 0, [], []
    scans = [(i, sc) for i, sc in enumerate(BATCH_SCANS) if args.batch_scans in ("all", sc[0])]
    for i, (algo, N, nx, step) in scans:
        rng = np.random.default_rng(20261206 + i)
        dx_s = synth.sample_pixel(lambd, z, dx_d, N)
        pos, X, Y = synth.raster_positions(nx, nx, step, step, dx_s, N)
        obj = synth.make_object(X, Y, rng)
        probe = synth.make_probe(N, dx_s, K=1)
        amp = synth.make_patterns_torch(obj, probe, pos, N, 1e6, seed=20261206 + i, device="cuda",
                                        intensities=(algo == "MLs"))
        s = abi.Session(size=N, scanDimsx=nx, scanDimsy=nx, stepx=step, stepy=step, lambd=lambd, z=z, dx_d=dx_d,
                        beamSize=synth.BEAM_FWHM, probeModes=1, algorithm=algo, delta_p=0.1, PPS=20, device=local)
        s.set_patterns_ptr(amp.data_ptr(), pos.shape[0], N)
        s.set_probe(probe)
        if not args.no_autotune and algo != "MLs":
            t0 = time.perf_counter()
            tuning.append({"scan": f"{algo} {N}^2 {nx}x{nx}", "choice": s.autotune(iters=1),
                           "seconds": round(time.perf_counter() - t0, 3)})
        s.init()
        keep.append(amp)
        sessions.append(s)
        total_p += pos.shape[0]
    abi.batch_run(sessions, 2)  # graph capture and warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in sessions:
        s.run(args.steps)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    clocks = Clocks(local)
    clocks.start()
    t0 = time.perf_counter()
    abi.batch_run(sessions, args.steps)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    ck = clocks.stop()
    finite = all(bool(np.isfinite(s.object()).all()) for s in sessions)
    work = total_p * args.steps
    out = {"metric": "batched reconstructions, aggregate patterns/s", "value": work / t_batch, "unit": UNIT,
           "n_gpus": 1, "steps": args.steps, "warmup": 2, "higher_is_better": True, "dtype": "f32",
           "data": "synthetic (seeded)",
           "config": {"workload": ("16 scans: 8 DM + 8 MLs (delta_p 0.1), detectors 128-512, rasters 10x10-40x40, "
                                   "steps 30-100 nm, 1e6 photons/pattern") if args.batch_scans == "all" else
                                  f"the {args.batch_scans} scans of the 16-scan batch", "positions": total_p,
                      "scans": [f"{a} {n}^2 {r}x{r} {st * 1e9:.0f} nm" for _, (a, n, r, st) in scans]},
           "sequential": {"value": work / t_seq, "unit": UNIT, "seconds": t_seq},
           "batched_seconds": t_batch, "speedup_vs_sequential": t_seq / t_batch, "clocks": ck, "finite": finite,
           "timing": "host wall clock around synchronised regions (includes each scan's host-side scheduling)",
           "autotune": tuning if tuning else "off (--no-autotune)",
           "note": "MLs runs the reference's default path: variable probe and intensity, sub-pixel probe shift, "
                   "position search from iteration PPS = 20 (the first 2 of the timed iterations run without it at "
                   "--steps 50 after 2 warm-up ones: iterations 3-19 do not search, 20-52 do)"}
    for s in sessions:
        s.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.algo == "epie" and args.impl == "b200":
        run_epie(args, rank, local)
    elif args.algo == "batch" and args.impl == "b200":
        run_batch(args, rank, local)
    elif args.algo == "nrmse" and args.impl == "b200":
        run_nrmse(args, rank, local)
    elif args.algo == "mls" and args.impl == "b200":
        run_mls(args, rank, local)
    elif args.algo == "warm" and args.impl == "b200":
        run_warm(args, rank, local)
    elif args.algo == "infer" and args.impl == "b200":
        run_infer(args, rank, local)
    elif args.algo == "fft" and args.impl == "b200":
        run_fft(args, rank, local)
    elif args.impl == "reference":
        run_reference(args, rank)
    else:
        run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
