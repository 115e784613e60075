"""DM position shards on one GPU: two shard sessions whose increments are summed between the local step and the
finish give the same object and probe as one session holding the whole scan."""
import numpy as np
import pytest
import torch

from conftest import rel_err
from gpu_helpers import dataset
from ptychopy_b200 import abi

pytestmark = pytest.mark.gpu


class _Dev:
    """A complex64 device buffer as a torch tensor (through __cuda_array_interface__)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (2 * n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def _tensor(ptr, n):
    return torch.as_tensor(_Dev(ptr, n), device="cuda")


def _shard(d, first, count, total):
    s = abi.Session(**dict(d["kw"], updateProbe=2))
    s.set_shard(first, total)
    s.set_patterns(np.ascontiguousarray(d["amp"][first:first + count]))
    s.set_probe(d["probe"])
    s.init()
    return s


def test_two_shards_equal_the_whole_scan():
    d = dataset(N=64, nx=5, algorithm="DM")
    P = d["amp"].shape[0]
    whole = abi.Session(**dict(d["kw"], updateProbe=2))
    whole.set_patterns(d["amp"])
    whole.set_probe(d["probe"])
    whole.init()
    a, b = _shard(d, 0, 13, P), _shard(d, 13, P - 13, P)
    assert np.array_equal(np.concatenate([a.positions(), b.positions()]), whole.positions())
    assert a.dims()["X"] == whole.dims()["X"] and b.dims()["Y"] == whole.dims()["Y"]
    for _ in range(4):
        whole.step()
        a.step_local()
        b.step_local()
        torch.cuda.synchronize()
        ia, ib = a.increments(), b.increments()
        for pa, pb, n in ((ia[0], ib[0], ia[1]), (ia[2], ib[2], ia[3])):
            ta, tb = _tensor(pa, n), _tensor(pb, n)
            ta += tb
            tb.copy_(ta)
        torch.cuda.synchronize()
        a.step_finish()
        b.step_finish()
    for s in (a, b):
        assert rel_err(s.object(), whole.object()) < 1e-5
        assert rel_err(s.probe(), whole.probe()) < 1e-5


def test_shard_rules():
    d = dataset(N=32, nx=3, algorithm="DM")
    s = abi.Session(**d["kw"])
    s.set_shard(0, 9)
    s.set_patterns(np.ascontiguousarray(d["amp"][:4]))
    with pytest.raises(abi.PtyError):  # no probe given: the guess needs every pattern
        s.init()
    s2 = abi.Session(**d["kw"])
    s2.set_shard(0, 9)
    s2.set_patterns(np.ascontiguousarray(d["amp"][:4]))
    s2.set_probe(d["probe"])
    s2.init()
    with pytest.raises(abi.PtyError):  # shards step in two halves around the reduction
        s2.step()
    with pytest.raises(abi.PtyError):
        s2.step_finish()
