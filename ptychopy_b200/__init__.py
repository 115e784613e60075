"""B200 ptychographic reconstruction engine.

`ptychopy_b200.ptychopy` is the CPython module with the reference package's API (epienp, dmnp, mlsnp, the step
calls ...); `import_ptychopy()` also registers it under the top-level name `ptychopy` so existing scripts run
unchanged.  `ptychopy_b200.abi` binds the C ABI directly.
"""
import importlib
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def import_ptychopy():
    """Import the native `ptychopy` module and make `import ptychopy` resolve to it."""
    mod = importlib.import_module("ptychopy_b200.ptychopy")
    sys.modules.setdefault("ptychopy", mod)
    return mod
