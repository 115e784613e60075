"""DM position shards across two processes (gloo, CPU): each rank runs the FP64 oracle on its share of the
positions and all-reduces the iteration's object / probe increments; the result equals one process holding the
whole scan.  This is the decomposition the GPU shards use (pty_set_shard / pty_dm_step_local / pty_dm_step_finish)
with NCCL in place of gloo."""
import os
import socket
import tempfile

import numpy as np
import pytest

from conftest import rel_err

ITERS = 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _data():
    from gpu_helpers import dataset

    return dataset(N=32, nx=5, algorithm="DM")


def _worker(rank, world, port, out):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
    import pyoracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = _data()
    P = d["amp"].shape[0]
    bounds = np.linspace(0, P, world + 1).astype(int)
    a, b = bounds[rank], bounds[rank + 1]
    o = pyoracle.OracleSession("DM", d["amp"][a:b], d["pos"][a:b], np.zeros((d["X"], d["Y"])), d["probe"],
                               probe_guess_path=False, updateProbe=2)

    def reduce(dO, dP):
        for arr in (dO, dP):
            t = torch.from_numpy(arr.view(np.float64))
            dist.all_reduce(t)

    o.set_dm_reduce(reduce)
    for _ in range(ITERS):
        o.step()
    ob, pr, _ = o.state()
    np.savez(os.path.join(out, f"rank{rank}.npz"), obj=ob, probe=pr)
    dist.destroy_process_group()


def test_two_shards_equal_the_whole_scan(oracle):
    import torch.multiprocessing as mp

    d = _data()
    full = oracle.OracleSession("DM", d["amp"], d["pos"], np.zeros((d["X"], d["Y"])), d["probe"],
                                probe_guess_path=False, updateProbe=2)
    for _ in range(ITERS):
        full.step()
    ob, pr, _ = full.state()
    with tempfile.TemporaryDirectory() as out:
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        for r in range(2):
            z = np.load(os.path.join(out, f"rank{r}.npz"))
            assert rel_err(z["obj"], ob) < 1e-12
            assert rel_err(z["probe"], pr) < 1e-12
