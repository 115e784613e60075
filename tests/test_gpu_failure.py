"""Failure detection of the bounded device waits without a GPU fault: waits whose condition nothing satisfies must
give up, report through their device flag and let the kernel return (pty_selftest_bounded_waits); the controls,
whose conditions are met, must not."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_bounded_waits_time_out_and_report():
    from ptychopy_b200 import abi

    codes = (ctypes.c_int * 4)(-1, -1, -1, -1)
    abi.check(abi.lib().pty_selftest_bounded_waits(codes))
    # mbarrier wait with no arrival gave up; after one arrival it completed; 64 grid barriers that reach their count
    # completed; a grid barrier expecting one arrival too many gave up and every CTA returned
    assert list(codes) == [1, 0, 0, 1]


def test_session_usable_after_the_timeouts():
    """The context survives the timed-out waits: a small ePIE session still runs."""
    import numpy as np

    from gpu_helpers import dataset, gpu_session
    from ptychopy_b200 import abi

    codes = (ctypes.c_int * 4)()
    abi.check(abi.lib().pty_selftest_bounded_waits(codes))
    d = dataset(N=64, nx=3)
    s = gpu_session(d, probe=d["probe"])
    s.step()
    assert np.isfinite(s.object()).all()
    s.close()
