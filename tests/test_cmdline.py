"""Command-line strings of the reference's `ptycho` program (pty_params_from_cmdline): the options its parser
reads (src/Parameters.cpp:66-375), the command line's own defaults (src/Parameters.h:67-170), the program name
skipped (src/ptychopy.c:543-576), and the refusals.  Host code only: no GPU needed."""
import ctypes

import pytest

# The command strings of the reference's own examples (example/epie.py, example/mls.py), the second with the
# backslash-newline continuation that Python folds into white space.
SIMSTR = ("./ptycho -jobID=sim256rDM -algorithm=DM -beamSize=110e-9 -scanDims=30,30 -step=50e-9,50e-9 -i=100 "
          "-size=256 -lambda=2.4796837508399954e-10 -dx_d=172e-6 -z=1 -simulate=1")
REALSTR = ("./ptycho -jobID=IOTes256MLs5 -algorithm=MLs -fp=/data/scan152/scan152_data_#06d.h5 -fs=1 "
           "-hdf5path=/entry/data/data -beamSize=100e-6 \
         -qxy=276,616 -scanDims=51,51 -step=100e-9,100e-9 -i=30 -size=256 -lambda=1.408911284090909e-10 "
           "-dx_d=75e-6 -z=1.92 -dpf=51 -probeModes=2 -delta_p=0.1 -PPS=20")


def parse(cmd):
    from ptychopy_b200 import abi

    p = abi.PtyParams()
    rc = abi.lib().pty_params_from_cmdline(cmd.encode(), ctypes.byref(p))
    return rc, p


def ok(cmd):
    from ptychopy_b200 import abi

    rc, p = parse(cmd)
    assert rc == abi.PTY_OK, abi.lib().pty_last_error().decode()
    return p


def test_reference_simulation_string():
    p = ok(SIMSTR)
    assert p.jobID == b"sim256rDM" and p.algorithm == b"DM"
    assert (p.beamSize, p.stepx, p.stepy) == (110e-9, 50e-9, 50e-9)
    assert (p.scanDimsx, p.scanDimsy, p.iter, p.size, p.simulate) == (30, 30, 100, 256, 1)
    assert (p.lambd, p.dx_d, p.z) == (2.4796837508399954e-10, 172e-6, 1.0)


def test_reference_file_string():
    p = ok(REALSTR)
    assert p.fp == b"/data/scan152/scan152_data_#06d.h5" and p.hdf5path == b"/entry/data/data"
    assert (p.fs, p.dpf, p.qx, p.qy, p.scanDimsx, p.scanDimsy) == (1, 51, 276, 616, 51, 51)
    assert (p.iter, p.size, p.probeModes, p.PPS) == (30, 256, 2, 20)
    assert (p.beamSize, p.lambd, p.dx_d, p.z) == (100e-6, 1.408911284090909e-10, 75e-6, 1.92)


def test_command_line_defaults():
    """Options absent from the string keep the command line's defaults, which are not the Python keywords'."""
    p = ok("./ptycho")
    assert (p.beamSize, p.lambd, p.dx_d, p.z) == (1e-7, 2.48e-10, 172e-6, 1.0)
    assert (p.scanDimsx, p.scanDimsy, p.stepx, p.stepy) == (12, 12, 40e-9, 40e-9)
    assert (p.size, p.qx, p.qy, p.nx, p.ny, p.fs, p.dpf) == (256, 128, 128, 256, 256, 0, 1)
    assert (p.iter, p.probeModes, p.updateProbe, p.updateModes, p.phaseConstraint, p.PPS) == (100, 1, 10, 20, 1, 5)
    assert (p.jitterRadius, p.threshold, p.rotate90, p.sqrtData, p.fftShiftData, p.simulate) == (0, 0, 0, 0, 0, 0)
    assert (p.save, p.T, p.delta_p) == (0, 0, 0.1)
    assert p.hdf5path == b"/entry/data/data" and p.fp == b"" and p.jobID == b""


def test_program_name_is_skipped():
    assert ok("-size=64").size == 256
    assert ok("prog -size=64").size == 64


def test_flags_and_integer_options():
    p = ok("x -sqrtData -fftShiftData -rotate90=1 -threshold=5 -RMS=1 -binaryOutput=1 -flipScanAxis=1 "
           "-mirror1stScanAxis=1 -mirror2ndScanAxis=2 -spiralScan=1 -jitterRadius=3 -save=10 -T=60.5 -lf=pos.csv "
           "-probeGuess=pg.csv -objectGuess=og.csv -nxy=512,400 -updateProbe=0 -updateModes=5 -phaseConstraint=0")
    assert (p.sqrtData, p.fftShiftData, p.rotate90, p.threshold, p.calculateRMS, p.binaryOutput) == (1, 1, 1, 5, 1, 1)
    assert (p.flipScanAxis, p.mirror1stScanAxis, p.mirror2ndScanAxis, p.spiralScan) == (1, 1, 1, 1)
    assert (p.jitterRadius, p.save, p.T, p.nx, p.ny) == (3, 10, 60, 512, 400)
    assert (p.updateProbe, p.updateModes, p.phaseConstraint) == (0, 5, 0)
    assert (p.lf, p.probeGuess, p.objectGuess) == (b"pos.csv", b"pg.csv", b"og.csv")
    # a bare integer option reads as 0, as the reference's integer lookup does
    assert ok("x -simulate").simulate == 0


def test_drift():
    p = ok("x -drift=3e-9,-1.5e-9")
    assert (p.driftx, p.drifty) == (3e-9, -1.5e-9)
    assert (ok("x").driftx, ok("x").drifty) == (0.0, 0.0)


def test_single_values_fill_both_components():
    """Without a comma the reference reads the second component from the start of the value again
    (substr(npos + 1)): drift, qxy, nxy and step take one value for both; scanDims sets the second to 1."""
    p = ok("x -drift=2e-9 -qxy=300 -nxy=640 -step=25e-9 -scanDims=9")
    assert (p.driftx, p.drifty, p.qx, p.qy, p.nx, p.ny) == (2e-9, 2e-9, 300, 300, 640, 640)
    assert (p.stepx, p.stepy, p.scanDimsx, p.scanDimsy) == (25e-9, 25e-9, 9, 1)


def test_numbers_read_like_atoi_and_atof():
    """Integers are read up to the first non-digit (atoi), out-of-range ones clamp; reals as atof."""
    p = ok("x -size=128px -i=1e3 -fs= -dpf=99999999999999999999 -T=1e30 -z=2.5m -jitterRadius=-3")
    assert (p.size, p.iter, p.fs, p.dpf, p.T, p.z) == (128, 1, 0, 2147483647, 2147483647, 2.5)
    assert p.jitterRadius == 0  # negative: out of the option's range, the default stays


def test_range_checks_keep_the_default():
    p = ok("x -size=16 -i=-1 -dpf=0 -probeModes=0 -PPS=0 -save=0 -fs=-2")
    assert (p.size, p.iter, p.dpf, p.probeModes, p.PPS, p.save, p.fs) == (256, 100, 1, 1, 5, 0, 0)


def test_pairs_names_and_repeats():
    p = ok("x --SIZE=128 -scanDims=7 -step=30e-9 -size=64 -qxy=10,20")
    assert p.size == 64  # last occurrence wins; names ignore case and the number of dashes
    assert (p.scanDimsx, p.scanDimsy) == (7, 1)  # one value: the second dimension is 1
    assert (p.stepx, p.stepy) == (30e-9, 30e-9)  # one value fills both (read as a real number)
    assert (p.qx, p.qy) == (10, 20)
    # an exact name: -threshold does not reset -T, and options this engine ignores are accepted
    p = ok("x -T=60 -threshold=5 -blind=0 -threads=8 -angles=2 -overlap=1 -shareFrequency=3 -updateVis=2 "
           "-wsServerUrl=ws://h -delta_p=0.3 -notanoption=1")
    assert (p.T, p.threshold, p.delta_p) == (60, 5, 0.1)  # delta_p is not a command-line option


def test_refusals_leave_the_parameters_unchanged():
    from ptychopy_b200 import abi

    L = abi.lib()
    p = abi.PtyParams()
    L.pty_params_init(ctypes.byref(p))
    p.size = 77
    for cmd, code in [("x -bitDepth=40", abi.PTY_ERR_INVALID), ("x -fp=" + "a" * 300, abi.PTY_ERR_INVALID),
                      ("x -algorithm=TOOLONGNAME", abi.PTY_ERR_INVALID)]:
        assert L.pty_params_from_cmdline(cmd.encode(), ctypes.byref(p)) == code, cmd
        assert L.pty_last_error()
        assert p.size == 77
    assert (ok("x -bitDepth=16").bitDepth, ok("x -bitDepth=0").bitDepth, ok("x").bitDepth) == (16, 0, 0)
    assert L.pty_params_from_cmdline(None, ctypes.byref(p)) == abi.PTY_ERR_INVALID


def test_module_entry_points_check_the_string():
    import ptychopy_b200

    pt = ptychopy_b200.import_ptychopy()
    with pytest.raises(ValueError):  # neither data files nor simulation
        pt.dmcmdstr("./ptycho -jobID=x -size=64")
    with pytest.raises(ValueError):
        pt.epieinit(cmdstr="./ptycho -i=3")
    with pytest.raises(NotImplementedError):  # the reference's own MLs example reads HDF5 files
        pt.mlsinit(REALSTR)
    with pytest.raises(ValueError):
        pt.epiecmdstr("./ptycho -simulate=1 -bitDepth=40")
    with pytest.raises(TypeError):
        pt.dmcmdstr(cmdstr="./ptycho", size=64)
