// CPython extension `ptychopy`: the reference's module surface (src/ptychopy.c:117-162) over the engine's C ABI.
//
// Same method names, keyword names and defaults.  Differences from the reference, all deliberate:
//   * errors raise Python exceptions instead of printing and returning None/True or exiting the process;
//   * result arrays are owned numpy arrays (the reference wraps leaked buffers, src/ptychopy.c:964-990);
//   * objectNP/probeNP accept any complex or real dtype (the reference misreads complex64, src/ptychopy.c:383-471);
//   * extra keywords: seed, calculateRMS, device, wave, returnResults, writeResults, outputDir, warmStart (trained
//     warm-start network parameters, float32) and warmStartWidth (its width, default 16), precision (0 FP32 FFT,
//     1 tensor-core FFT stages: MLs and ePIE at 256 x 256, DM at 512 x 512), mlsCore (1: MLs without the reference's variable
//     probe, sub-pixel shift and position search), save (write the results every `save` iterations, like the
//     reference's command-line option);
//     probeNP may be (K, N, N) to supply all probe modes.
// Whole-mode runs from data files (epie / dm / mls with fp) read .bin and .csv files; .h5 files (hdf5path) need the
// HDF5 library, which this build does not link, and raise NotImplementedError.  Command-line strings (epiecmdstr,
// dmcmdstr, mlscmdstr, epieinit, mlsinit) are parsed by pty_params_from_cmdline over the command line's defaults.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>

#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "../../include/ptychopy_b200.h"

namespace {

pty_session* g_session = nullptr;  // step-mode session (the reference's static IPhaser* phaser)
int g_binary_output = 0;           // its result-file format (binaryOutput), for epiepost / mlspost

PyObject* raise_status(int rc) {
  const char* msg = pty_last_error();
  PyObject* type = PyExc_RuntimeError;
  if (rc == PTY_ERR_INVALID) type = PyExc_ValueError;
  else if (rc == PTY_ERR_OOM) type = PyExc_MemoryError;
  else if (rc == PTY_ERR_UNSUPPORTED) type = PyExc_NotImplementedError;
  else if (rc == PTY_ERR_IO) type = PyExc_OSError;
  else if (rc == PTY_ERR_TIMEOUT) type = PyExc_TimeoutError;
  PyErr_SetString(type, (msg && *msg) ? msg : "ptychopy engine error");
  return nullptr;
}

void copy_str(char* dst, size_t cap, const char* src) {
  if (!src) src = "";
  std::strncpy(dst, src, cap - 1);
  dst[cap - 1] = 0;
}

struct Parsed {
  pty_params p;
  PyObject *diff = nullptr, *pos = nullptr, *obj = nullptr, *probe = nullptr, *warm = nullptr;
  int returnResults = 0, writeResults = 1, warmWidth = 16;
  const char* outputDir = "data";
};

// Keyword parsing identical to ptychopy_algorithmnp (src/ptychopy.c:282-342) plus the additions.
bool parse_kwargs(PyObject* args, PyObject* kw, const char* algorithm, bool np, Parsed& out) {
  pty_params_init(&out.p);
  copy_str(out.p.algorithm, sizeof(out.p.algorithm), algorithm);
  const char *jobID = "", *fp = "", *hdf5path = "", *probeGuess = "", *objectGuess = "", *lf = "";
  int fs = 0, dpf = 1, size = 512, qx = 128, qy = 128, nx = 256, ny = 256, scanDimsx = 26, scanDimsy = 26;
  int spiralScan = 0, flipScanAxis = 0, mirror1 = 0, mirror2 = 0, probeModes = 1, iter = 100, T = 0, jitter = 0;
  int threshold = 0, rotate90 = 0, sqrtData = 0, fftShiftData = 0, binaryOutput = 0, simulate = 0;
  int phaseConstraint = 1, updateProbe = 10, updateModes = 20, beamstopMask = 0, PPS = 20;
  double beamSize = 400e-9, stepx = 40e-9, stepy = 40e-9, lambd = 2.3843e-10, dx_d = 172e-6, z = 2.2, delta_p = 0.1;
  unsigned long long seed = out.p.seed;
  int calculateRMS = 0, device = 0, wave = 0, precision = 0, mlsCore = 0, save = 0;
  static const char* kw_np[] = {"jobID", "diffractionNP", "positionNP", "objectNP", "probeNP", "fp", "fs",
                                "hdf5path", "dpf", "beamSize", "probeGuess", "objectGuess", "size", "qx", "qy", "nx",
                                "ny", "scanDimsx", "scanDimsy", "spiralScan", "flipScanAxis", "mirror1stScanAxis",
                                "mirror2ndScanAxis", "stepx", "stepy", "probeModes", "lambd", "dx_d", "z", "iter",
                                "T", "jitterRadius", "delta_p", "threshold", "rotate90", "sqrtData", "fftShiftData",
                                "binaryOutput", "simulate", "phaseConstraint", "updateProbe", "updateModes",
                                "beamstopMask", "lf", "PPS", "seed", "calculateRMS", "device", "wave",
                                "returnResults", "writeResults", "outputDir", "warmStart", "warmStartWidth",
                                "precision", "mlsCore", "save", nullptr};
  static const char* kw_file[] = {"jobID", "fp", "fs", "hdf5path", "dpf", "beamSize", "probeGuess", "objectGuess",
                                  "size", "qx", "qy", "nx", "ny", "scanDimsx", "scanDimsy", "spiralScan",
                                  "flipScanAxis", "mirror1stScanAxis", "mirror2ndScanAxis", "stepx", "stepy",
                                  "probeModes", "lambd", "dx_d", "z", "iter", "T", "jitterRadius", "delta_p",
                                  "threshold", "rotate90", "sqrtData", "fftShiftData", "binaryOutput", "simulate",
                                  "phaseConstraint", "updateProbe", "updateModes", "beamstopMask", "lf", "PPS",
                                  "seed", "calculateRMS", "device", "wave", "returnResults", "writeResults",
                                  "outputDir", "precision", "mlsCore", "save", nullptr};
  int ok;
  if (np) {
    ok = PyArg_ParseTupleAndKeywords(
        args, kw, "|sOOOOsisidssiiiiiiiiiiiddidddiiidiiiiiiiiiisiKiiiiisOiiii", const_cast<char**>(kw_np), &jobID,
        &out.diff, &out.pos, &out.obj, &out.probe, &fp, &fs, &hdf5path, &dpf, &beamSize, &probeGuess, &objectGuess,
        &size, &qx, &qy, &nx, &ny, &scanDimsx, &scanDimsy, &spiralScan, &flipScanAxis, &mirror1, &mirror2, &stepx,
        &stepy, &probeModes, &lambd, &dx_d, &z, &iter, &T, &jitter, &delta_p, &threshold, &rotate90, &sqrtData,
        &fftShiftData, &binaryOutput, &simulate, &phaseConstraint, &updateProbe, &updateModes, &beamstopMask, &lf,
        &PPS, &seed, &calculateRMS, &device, &wave, &out.returnResults, &out.writeResults, &out.outputDir, &out.warm,
        &out.warmWidth, &precision, &mlsCore, &save);
  } else {
    ok = PyArg_ParseTupleAndKeywords(args, kw, "|ssisidssiiiiiiiiiiiddidddiiidiiiiiiiiiisiKiiiiisiii",
                                     const_cast<char**>(kw_file), &jobID, &fp, &fs, &hdf5path, &dpf, &beamSize,
                                     &probeGuess, &objectGuess, &size, &qx, &qy, &nx, &ny, &scanDimsx, &scanDimsy,
                                     &spiralScan, &flipScanAxis, &mirror1, &mirror2, &stepx, &stepy, &probeModes,
                                     &lambd, &dx_d, &z, &iter, &T, &jitter, &delta_p, &threshold, &rotate90,
                                     &sqrtData, &fftShiftData, &binaryOutput, &simulate, &phaseConstraint,
                                     &updateProbe, &updateModes, &beamstopMask, &lf, &PPS, &seed, &calculateRMS,
                                     &device, &wave, &out.returnResults, &out.writeResults, &out.outputDir,
                                     &precision, &mlsCore, &save);
  }
  if (!ok) return false;
  pty_params& p = out.p;
  copy_str(p.jobID, sizeof(p.jobID), jobID);
  copy_str(p.fp, sizeof(p.fp), fp);
  copy_str(p.hdf5path, sizeof(p.hdf5path), hdf5path);
  copy_str(p.probeGuess, sizeof(p.probeGuess), probeGuess);
  copy_str(p.objectGuess, sizeof(p.objectGuess), objectGuess);
  copy_str(p.lf, sizeof(p.lf), lf);
  p.fs = fs; p.dpf = dpf; p.beamSize = beamSize; p.size = size; p.qx = qx; p.qy = qy; p.nx = nx; p.ny = ny;
  p.scanDimsx = scanDimsx; p.scanDimsy = scanDimsy; p.spiralScan = spiralScan; p.flipScanAxis = flipScanAxis;
  p.mirror1stScanAxis = mirror1; p.mirror2ndScanAxis = mirror2; p.stepx = stepx; p.stepy = stepy;
  p.probeModes = probeModes; p.lambd = lambd; p.dx_d = dx_d; p.z = z; p.iter = iter; p.T = T;
  p.jitterRadius = jitter; p.delta_p = delta_p; p.threshold = threshold; p.rotate90 = rotate90;
  p.sqrtData = sqrtData; p.fftShiftData = fftShiftData; p.binaryOutput = binaryOutput; p.simulate = simulate;
  p.phaseConstraint = phaseConstraint; p.updateProbe = updateProbe; p.updateModes = updateModes;
  p.beamstopMask = beamstopMask; p.PPS = PPS; p.seed = seed; p.calculateRMS = calculateRMS; p.device = device;
  p.wave = wave;
  p.precision = precision;
  p.mlsCore = mlsCore;
  p.save = save;
  copy_str(p.outputDir, sizeof(p.outputDir), out.outputDir);
  return true;
}

// Builds a session from parsed numpy inputs and runs pty_init.  Returns nullptr with a Python error set.
pty_session* make_session(Parsed& a) {
  const bool from_files = (!a.diff || a.diff == Py_None) && (a.p.fp[0] || a.p.simulate);
  if (from_files) {  // whole-mode run: pty_init reads the patterns from the files of fp (or simulates them)
    pty_session* s = nullptr;
    int rc = pty_session_create(&a.p, &s);
    if (rc != PTY_OK) {
      raise_status(rc);
      return nullptr;
    }
    Py_BEGIN_ALLOW_THREADS rc = pty_init(s);
    Py_END_ALLOW_THREADS if (rc != PTY_OK) {
      raise_status(rc);
      pty_session_destroy(s);
      return nullptr;
    }
    return s;
  }
  if (!a.diff || a.diff == Py_None) {
    PyErr_SetString(PyExc_ValueError, "diffractionNP (or a data file pattern fp) is required");
    return nullptr;
  }
  PyArrayObject* d = nullptr;
  PyArray_Descr* in_descr = PyArray_DescrFromObject(a.diff, nullptr);
  const int want = (in_descr && in_descr->type_num == NPY_FLOAT32) ? NPY_FLOAT32 : NPY_FLOAT64;
  Py_XDECREF(in_descr);
  d = reinterpret_cast<PyArrayObject*>(PyArray_FROM_OTF(a.diff, want, NPY_ARRAY_IN_ARRAY));
  if (!d) return nullptr;
  if (PyArray_NDIM(d) != 3 || PyArray_DIM(d, 1) != PyArray_DIM(d, 2)) {
    Py_DECREF(d);
    PyErr_SetString(PyExc_ValueError, "diffractionNP must have shape (P, N, N)");
    return nullptr;
  }
  pty_session* s = nullptr;
  int rc = pty_session_create(&a.p, &s);
  if (rc != PTY_OK) {
    Py_DECREF(d);
    raise_status(rc);
    return nullptr;
  }
  const int P = int(PyArray_DIM(d, 0)), N = int(PyArray_DIM(d, 1));
  Py_BEGIN_ALLOW_THREADS rc = pty_set_patterns(s, PyArray_DATA(d), want == NPY_FLOAT32 ? PTY_F32 : PTY_F64, P, N);
  Py_END_ALLOW_THREADS Py_DECREF(d);
  auto bail = [&](int code) -> pty_session* {
    if (code != PTY_OK) raise_status(code);
    pty_session_destroy(s);
    return nullptr;
  };
  if (rc != PTY_OK) return bail(rc);
  if (a.pos && a.pos != Py_None) {
    PyArrayObject* q = reinterpret_cast<PyArrayObject*>(PyArray_FROM_OTF(a.pos, NPY_FLOAT64, NPY_ARRAY_IN_ARRAY));
    if (!q) return bail(PTY_OK);
    if (PyArray_NDIM(q) != 2 || PyArray_DIM(q, 1) != 2) {
      Py_DECREF(q);
      PyErr_SetString(PyExc_ValueError, "positionNP must have shape (P, 2)");
      return bail(PTY_OK);
    }
    rc = pty_set_positions(s, static_cast<const double*>(PyArray_DATA(q)), int(PyArray_DIM(q, 0)));
    Py_DECREF(q);
    if (rc != PTY_OK) return bail(rc);
  }
  if (a.obj && a.obj != Py_None) {
    PyArrayObject* o = reinterpret_cast<PyArrayObject*>(PyArray_FROM_OTF(a.obj, NPY_COMPLEX64, NPY_ARRAY_IN_ARRAY));
    if (!o) return bail(PTY_OK);
    if (PyArray_NDIM(o) != 2) {
      Py_DECREF(o);
      PyErr_SetString(PyExc_ValueError, "Expected 2 dimensional object array");
      return bail(PTY_OK);
    }
    rc = pty_set_object(s, static_cast<const float*>(PyArray_DATA(o)), int(PyArray_DIM(o, 0)), int(PyArray_DIM(o, 1)));
    Py_DECREF(o);
    if (rc != PTY_OK) return bail(rc);
  }
  if (a.probe && a.probe != Py_None) {
    PyArrayObject* pr =
        reinterpret_cast<PyArrayObject*>(PyArray_FROM_OTF(a.probe, NPY_COMPLEX64, NPY_ARRAY_IN_ARRAY));
    if (!pr) return bail(PTY_OK);
    const int nd = PyArray_NDIM(pr);
    if (nd != 2 && nd != 3) {
      Py_DECREF(pr);
      PyErr_SetString(PyExc_ValueError, "Expected 2 dimensional probe array (or K x N x N modes)");
      return bail(PTY_OK);
    }
    const int K = nd == 3 ? int(PyArray_DIM(pr, 0)) : 1, pn = int(PyArray_DIM(pr, nd - 1));
    if (PyArray_DIM(pr, nd - 2) != pn) {
      Py_DECREF(pr);
      PyErr_SetString(PyExc_ValueError, "probe must be square");
      return bail(PTY_OK);
    }
    rc = pty_set_probe(s, static_cast<const float*>(PyArray_DATA(pr)), K, pn);
    Py_DECREF(pr);
    if (rc != PTY_OK) return bail(rc);
  }
  if (a.warm && a.warm != Py_None) {
    PyArrayObject* wa = reinterpret_cast<PyArrayObject*>(PyArray_FROM_OTF(a.warm, NPY_FLOAT32, NPY_ARRAY_IN_ARRAY));
    if (!wa) return bail(PTY_OK);
    rc = pty_set_warm_start(s, static_cast<const float*>(PyArray_DATA(wa)), size_t(PyArray_SIZE(wa)), a.warmWidth);
    Py_DECREF(wa);
    if (rc != PTY_OK) return bail(rc);
  }
  Py_BEGIN_ALLOW_THREADS rc = pty_init(s);
  Py_END_ALLOW_THREADS if (rc != PTY_OK) return bail(rc);
  return s;
}

PyObject* object_array(pty_session* s) {
  int X = 0, Y = 0;
  pty_get_dims(s, &X, &Y, nullptr, nullptr, nullptr, nullptr);
  npy_intp dims[2] = {X, Y};
  PyObject* arr = PyArray_SimpleNew(2, dims, NPY_COMPLEX64);
  if (!arr) return nullptr;
  int rc = pty_get_object(s, static_cast<float*>(PyArray_DATA(reinterpret_cast<PyArrayObject*>(arr))), X, Y);
  if (rc != PTY_OK) {
    Py_DECREF(arr);
    return raise_status(rc);
  }
  return arr;
}

// The reference returns the probe stack as (K*N, N) (src/ptychopy.c:978-990).
PyObject* probe_array(pty_session* s) {
  int K = 0, N = 0;
  pty_get_dims(s, nullptr, nullptr, &K, &N, nullptr, nullptr);
  npy_intp dims[2] = {npy_intp(K) * N, N};
  PyObject* arr = PyArray_SimpleNew(2, dims, NPY_COMPLEX64);
  if (!arr) return nullptr;
  int rc = pty_get_probe(s, static_cast<float*>(PyArray_DATA(reinterpret_cast<PyArrayObject*>(arr))), K, N);
  if (rc != PTY_OK) {
    Py_DECREF(arr);
    return raise_status(rc);
  }
  return arr;
}

bool write_results(pty_session* s, const Parsed& a, int r) {
  struct stat st;
  if (stat(a.outputDir, &st) != 0) mkdir(a.outputDir, 0755);
  int rc = pty_write_results(s, a.outputDir, r, a.p.binaryOutput);
  if (rc != PTY_OK) {
    raise_status(rc);
    return false;
  }
  return true;
}

// Whole-mode run: IPhaser::init + phase + writeResultsToDisk (src/ptychopy.c:474-487); np selects the numpy keyword
// list (epienp, ...) or the file one (epie, ...: patterns from the data files of fp).
PyObject* run_np(PyObject* args, PyObject* kw, const char* algorithm, bool np = true) {
  Parsed a;
  if (!parse_kwargs(args, kw, algorithm, np, a)) return nullptr;
  if (!np && !a.p.fp[0] && !a.p.simulate) {
    PyErr_SetString(PyExc_ValueError, "fp (the data file pattern) or simulate=1 is required");
    return nullptr;
  }
  pty_session* s = make_session(a);
  if (!s) return nullptr;
  int rc;
  const int iters = a.p.iter;
  Py_BEGIN_ALLOW_THREADS rc = pty_run(s, iters, nullptr);
  Py_END_ALLOW_THREADS if (rc != PTY_OK) {
    raise_status(rc);
    pty_session_destroy(s);
    return nullptr;
  }
  PyObject* result = nullptr;
  if (a.writeResults && !write_results(s, a, 0)) {
    pty_session_destroy(s);
    return nullptr;
  }
  if (a.returnResults) {
    PyObject* o = object_array(s);
    PyObject* p = o ? probe_array(s) : nullptr;
    if (!o || !p) {
      Py_XDECREF(o);
      pty_session_destroy(s);
      return nullptr;
    }
    result = PyTuple_Pack(2, o, p);
    Py_DECREF(o);
    Py_DECREF(p);
  } else {
    result = Py_True;
    Py_INCREF(result);
  }
  pty_session_destroy(s);
  return result;
}

// The single keyword `cmdstr` of the command-string entry points, parsed into `out` for `algorithm` (the entry
// point's own: the reference's epiecmdstr runs ePIE whatever -algorithm says, src/ptychopy.c:578-612).
bool parse_cmdstr(PyObject* args, PyObject* kw, const char* algorithm, Parsed& out) {
  const char* cmdstr = "";
  static const char* kwl[] = {"cmdstr", nullptr};
  if (!PyArg_ParseTupleAndKeywords(args, kw, "|s", const_cast<char**>(kwl), &cmdstr)) return false;
  const int rc = pty_params_from_cmdline(cmdstr, &out.p);
  if (rc != PTY_OK) {
    raise_status(rc);
    return false;
  }
  copy_str(out.p.algorithm, sizeof(out.p.algorithm), algorithm);
  if (!out.p.fp[0] && !out.p.simulate) {
    PyErr_SetString(PyExc_ValueError, "the command string names no data files (-fp=...) and no -simulate=1");
    return false;
  }
  return true;
}

// epiecmdstr / dmcmdstr / mlscmdstr (src/ptychopy.c:578-689): a whole run from a command string; the results are
// written to data/ and the object is returned, complex64 (X, Y).
PyObject* run_cmdstr(PyObject* args, PyObject* kw, const char* algorithm) {
  Parsed a;
  if (!parse_cmdstr(args, kw, algorithm, a)) return nullptr;
  pty_session* s = make_session(a);
  if (!s) return nullptr;
  int rc;
  const int iters = a.p.iter;
  Py_BEGIN_ALLOW_THREADS rc = pty_run(s, iters, nullptr);
  Py_END_ALLOW_THREADS if (rc != PTY_OK) {
    raise_status(rc);
    pty_session_destroy(s);
    return nullptr;
  }
  PyObject* o = write_results(s, a, 0) ? object_array(s) : nullptr;
  pty_session_destroy(s);
  return o;
}

PyObject* m_helloworld(PyObject*, PyObject* args) {
  PyObject *a, *b, *c;
  if (!PyArg_ParseTuple(args, "OOO", &a, &b, &c)) return nullptr;
  Py_RETURN_NONE;
}

PyObject* m_epie(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "ePIE", false); }
PyObject* m_dm(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "DM", false); }
PyObject* m_mls(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "MLs", false); }
PyObject* m_epienp(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "ePIE"); }
PyObject* m_dmnp(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "DM"); }
PyObject* m_mlsnp(PyObject*, PyObject* args, PyObject* kw) { return run_np(args, kw, "MLs"); }
PyObject* m_epiecmdstr(PyObject*, PyObject* args, PyObject* kw) { return run_cmdstr(args, kw, "ePIE"); }
PyObject* m_dmcmdstr(PyObject*, PyObject* args, PyObject* kw) { return run_cmdstr(args, kw, "DM"); }
PyObject* m_mlscmdstr(PyObject*, PyObject* args, PyObject* kw) { return run_cmdstr(args, kw, "MLs"); }

void drop_session() {
  if (g_session) pty_session_destroy(g_session);
  g_session = nullptr;
}

// Step mode: ptychopy_algorithmnpinit (src/ptychopy.c:691-900) keeps one module-level session.
PyObject* npinit(PyObject* args, PyObject* kw, const char* algorithm) {
  Parsed a;
  if (!parse_kwargs(args, kw, algorithm, true, a)) return nullptr;
  drop_session();
  g_session = make_session(a);
  if (!g_session) return nullptr;
  g_binary_output = a.p.binaryOutput;
  Py_RETURN_TRUE;
}
PyObject* m_epienpinit(PyObject*, PyObject* args, PyObject* kw) { return npinit(args, kw, "ePIE"); }
PyObject* m_dmnpinit(PyObject*, PyObject* args, PyObject* kw) { return npinit(args, kw, "DM"); }
PyObject* m_mlsnpinit(PyObject*, PyObject* args, PyObject* kw) { return npinit(args, kw, "MLs"); }
// epieinit / mlsinit (src/ptychopy.c:902-937,994-1024): step mode from a command string.
PyObject* cmdinit(PyObject* args, PyObject* kw, const char* algorithm) {
  Parsed a;
  if (!parse_cmdstr(args, kw, algorithm, a)) return nullptr;
  drop_session();
  g_session = make_session(a);
  if (!g_session) return nullptr;
  g_binary_output = a.p.binaryOutput;
  Py_RETURN_TRUE;
}
PyObject* m_epieinit(PyObject*, PyObject* args, PyObject* kw) { return cmdinit(args, kw, "ePIE"); }
PyObject* m_mlsinit(PyObject*, PyObject* args, PyObject* kw) { return cmdinit(args, kw, "MLs"); }

PyObject* need_session() {
  PyErr_SetString(PyExc_RuntimeError, "no step-mode session: call epienpinit first");
  return nullptr;
}

// epiestep / mlsstep (src/ptychopy.c:955-962): one iteration; returns the iteration's error metric.
PyObject* m_step(PyObject*, PyObject*, PyObject*) {
  if (!g_session) return need_session();
  double err = 0;
  int rc;
  Py_BEGIN_ALLOW_THREADS rc = pty_step(g_session, &err);
  Py_END_ALLOW_THREADS if (rc != PTY_OK) return raise_status(rc);
  return PyFloat_FromDouble(err);
}
PyObject* m_resobj(PyObject*, PyObject*, PyObject*) {
  if (!g_session) return need_session();
  return object_array(g_session);
}
PyObject* m_resprobe(PyObject*, PyObject*, PyObject*) {
  if (!g_session) return need_session();
  return probe_array(g_session);
}
// epiepost / mlspost: write results (in the session's binaryOutput format) and release the session
// (src/ptychopy.c:944-953, IPhaser::writeResultsToDisk src/IPhaser.cpp:417-428).
PyObject* m_post(PyObject*, PyObject* args, PyObject* kw) {
  if (!g_session) return need_session();
  int writeResults = 1;
  const char* outputDir = "data";
  static const char* kwl[] = {"writeResults", "outputDir", nullptr};
  if (!PyArg_ParseTupleAndKeywords(args, kw, "|is", const_cast<char**>(kwl), &writeResults, &outputDir))
    return nullptr;
  if (writeResults) {
    struct stat st;
    if (stat(outputDir, &st) != 0) mkdir(outputDir, 0755);
    int rc = pty_write_results(g_session, outputDir, 0, g_binary_output);
    if (rc != PTY_OK) {
      drop_session();
      return raise_status(rc);
    }
  }
  drop_session();
  Py_RETURN_TRUE;
}

#define KW(f) reinterpret_cast<PyCFunction>(reinterpret_cast<void (*)(void)>(f)), METH_VARARGS | METH_KEYWORDS
PyMethodDef methods[] = {
    {"helloworld", m_helloworld, METH_VARARGS, "Argument round-trip check."},
    {"epie", KW(m_epie), "ePIE reconstruction from data files (fp: .bin or .csv)."},
    {"dm", KW(m_dm), "DM reconstruction from data files (fp: .bin or .csv)."},
    {"mls", KW(m_mls), "MLs reconstruction from data files (fp: .bin or .csv)."},
    {"epienp", KW(m_epienp), "ePIE reconstruction from numpy arrays."},
    {"dmnp", KW(m_dmnp), "DM reconstruction from numpy arrays."},
    {"mlsnp", KW(m_mlsnp), "MLs reconstruction from numpy arrays."},
    {"epiecmdstr", KW(m_epiecmdstr), "ePIE from a command-line string; returns the object."},
    {"dmcmdstr", KW(m_dmcmdstr), "DM from a command-line string; returns the object."},
    {"mlscmdstr", KW(m_mlscmdstr), "MLs from a command-line string; returns the object."},
    {"epieinit", KW(m_epieinit), "Step-mode ePIE init from a command-line string."},
    {"epiepost", KW(m_post), "Write results and end the step-mode session."},
    {"epiestep", KW(m_step), "One step-mode iteration; returns the error metric."},
    {"epieresobj", KW(m_resobj), "Current object, complex64 (X, Y)."},
    {"epieresprobe", KW(m_resprobe), "Current probe modes, complex64 (K*N, N)."},
    {"epienpinit", KW(m_epienpinit), "Step-mode ePIE init from numpy arrays."},
    {"mlsinit", KW(m_mlsinit), "Step-mode MLs init from a command-line string."},
    {"mlspost", KW(m_post), "Write results and end the step-mode session."},
    {"mlsstep", KW(m_step), "One step-mode iteration; returns the error metric."},
    {"mlsresobj", KW(m_resobj), "Current object, complex64 (X, Y)."},
    {"mlsresprobe", KW(m_resprobe), "Current probe modes, complex64 (K*N, N)."},
    {"dmnpinit", KW(m_dmnpinit), "Step-mode DM init from numpy arrays (addition)."},
    {"mlsnpinit", KW(m_mlsnpinit), "Step-mode MLs init from numpy arrays (addition)."},
    {nullptr, nullptr, 0, nullptr}};

PyModuleDef module_def = {PyModuleDef_HEAD_INIT, "ptychopy",
                          "B200 ptychographic reconstruction engine (ptychopy-compatible API).", -1, methods};

}  // namespace

PyMODINIT_FUNC PyInit_ptychopy(void) {
  import_array();
  return PyModule_Create(&module_def);
}
