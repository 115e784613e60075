/* ptychopy_b200 — C ABI of the B200 ptychographic reconstruction engine.
 *
 * This is the drop-in boundary underneath the CPython module `ptychopy` (same 20 method names and keyword
 * arguments as the reference's extension, src/ptychopy.c:117-140).  The reference has no C ABI of its own: its
 * CPython functions drive the C++ class IPhaser directly.  Each entry point below names the reference
 * interface whose behaviour it replaces.  All buffers are host buffers owned by the caller unless a name says
 * `dev`; complex arrays are interleaved (re, im) float32 ("complex64"), row-major, first index = x (row).
 *
 * Every function returns an int status: PTY_OK (0) or a negative PTY_ERR_* code; pty_last_error() gives the
 * message of the last failure on the calling thread.  No function calls exit(); the reference exits the
 * process on any CUDA error (src/utilities.h:73-92) and on a negative scan position (src/ePIE.cpp:100-105).
 */
#ifndef PTYCHOPY_B200_H_
#define PTYCHOPY_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PTY_OK 0
#define PTY_ERR_INVALID (-1)   /* bad argument, shape or dtype */
#define PTY_ERR_OOM (-2)       /* device or host allocation failed */
#define PTY_ERR_CUDA (-3)      /* CUDA runtime error (message in pty_last_error) */
#define PTY_ERR_STATE (-4)     /* call out of order (e.g. pty_step before pty_init) */
#define PTY_ERR_UNSUPPORTED (-5) /* valid request this build does not implement */
#define PTY_ERR_TIMEOUT (-6)   /* a bounded device-side wait gave up */
#define PTY_ERR_IO (-7)        /* file could not be written */

#define PTY_F32 0
#define PTY_F64 1

/* Reconstruction parameters.  Field names and meanings follow the reference's keyword arguments
 * (src/ptychopy.c:242-246, mapped to CXParams at src/Parameters.cpp:380-653); defaults (pty_params_init) are
 * the reference's C defaults (src/ptychopy.c:200-240).  Fields after `PPS` are additions of this engine. */
typedef struct pty_params {
  char jobID[128];
  char algorithm[8];      /* "ePIE", "DM" or "MLs" */
  char fp[256];           /* data file pattern, '#' marking the file index conversion (e.g. "scan/d_#06d.bin");
                             used by pty_init when no patterns were set: .bin (raw float32) or .csv files */
  int fs;
  char hdf5path[128];
  int dpf;
  double beamSize;        /* m */
  char probeGuess[256];   /* CSV probe guess file (reference format) or "" */
  char objectGuess[256];  /* CSV object guess file or "" */
  int size;               /* detector / probe size N */
  int qx, qy, nx, ny;     /* file ingest: crop centre (qx, qy) and raw pattern size nx x ny */
  int scanDimsx, scanDimsy;
  int spiralScan, flipScanAxis, mirror1stScanAxis, mirror2ndScanAxis;
  double stepx, stepy;    /* m */
  int probeModes;
  double lambd, dx_d, z;  /* m */
  int iter;
  int T;                  /* wall-time limit in s (0 = none) */
  int jitterRadius;
  double delta_p;
  int threshold, rotate90, sqrtData, fftShiftData, binaryOutput;
  int simulate;           /* 1: ePIE / DM patterns from the forward model of data/lena<size>.pgm (magnitude) and
                             data/baboon<size>.pgm (phase), read relative to the working directory, and a simulated
                             probe with a seeded random phase (src/IPhaser.cpp:93-117) */
  int phaseConstraint, updateProbe, updateModes, beamstopMask;
  char lf[256];           /* positions list file or "" */
  int PPS;
  /* --- additions --- */
  uint64_t seed;          /* seed of the ePIE visiting order, the MLs groups and the position jitter (reference:
                             time(NULL) / rand() / curand) */
  int calculateRMS;       /* compute the per-iteration error metric (the reference's Python path never does) */
  int device;             /* CUDA device ordinal */
  int wave;               /* DM patterns per wave of its three kernels (0 = automatic) */
  int precision;          /* FFT arithmetic: 0 FP32 (default); 1 tensor-core stages: at N = 256 split-BF16
                             (pty_fft2_tc) for MLs (its group transforms) and ePIE (then run as a per-position kernel
                             chain around the tensor-core transforms instead of the fused FP32 kernel); at N = 512
                             for DM, whose column pass computes its 32-point DFT stages as split-FP16 GEMMs.  Other
                             sizes refuse 1 (PTY_ERR_UNSUPPORTED). */
  int mlsCore;            /* MLs: 0 (default) the reference's path, which its Python API always runs
                             (src/Parameters.h:162-163: variable probe with one extra mode, variable intensity,
                             sub-pixel probe shift, position search from iteration PPS); 1 the fixed-probe core
                             without them */
  int save;               /* pty_run writes the results (pty_write_results to outputDir, r = iteration / save)
                             after every `save`-th iteration; 0 = never.  The reference's command line has this
                             checkpoint (src/IPhaser.cpp:384-385); its Python path leaves it at 999999 */
  char outputDir[256];    /* directory of those checkpoint files ("" = "data", the reference's) */
  double driftx, drifty;  /* linear drift of the generated scan positions, in m per row (x) and per column (y) of
                             the mesh array (Cartesian: raster row i and column j; list and spiral: index / 1024
                             and index % 1024), added before the pixel conversion like the reference's
                             command-line option `drift` (d_generateMesh, src/ScanMeshKernels.cu:86-87); 0 = none */
  int bitDepth;           /* detector bit depth, 1..32 (0 = not given: 32), the reference's command-line `bitDepth`.
                             ePIE lets pixels with amplitude >= the saturation level float (no modulus constraint,
                             src/utilitiesKernels.cu:619-682); the level is 2^bitDepth - 1 - threshold, square-rooted
                             with sqrtData, truncated to an integer at each step like the reference's
                             pixelSaturation (src/Parameters.cpp:54-62), and set only when bitDepth, threshold or
                             sqrtData is given (otherwise no pixel floats) */
} pty_params;

typedef struct pty_session pty_session;

/* Fill `p` with the reference's Python-call defaults.  Replaces the default block of
 * ptychopy_algorithmnp (src/ptychopy.c:282-323). */
int pty_params_init(pty_params* p);

/* Fill `p` from a command-line string in the format of the reference's `ptycho` program, e.g.
 * "./ptycho -jobID=sim -scanDims=30,30 -step=50e-9,50e-9 -i=100 -size=256 -lambda=2.48e-10 -dx_d=172e-6 -z=1
 * -simulate=1": white-space separated "-name=value" options after the program name, over the command line's own
 * defaults (beamSize 1e-7, lambda 2.48e-10, z 1, scanDims 12 x 12, size 256, PPS 5; the rest as pty_params_init),
 * each option with the reference's range check.  Names match exactly, ignoring case; the last occurrence wins.
 * `-drift=dx,dy` sets driftx / drifty, `-bitDepth=b` bitDepth.  PTY_ERR_INVALID for a text value longer than its
 * field or a bitDepth above 32; `p` is left unchanged on an error.  Replaces the tokeniser of the command-string entry points
 * (src/ptychopy.c:543-576) and Parameters::parseFromCommandLine (src/Parameters.cpp:66-375) with the defaults of
 * src/Parameters.h:67-170. */
int pty_params_from_cmdline(const char* cmdstr, pty_params* p);

/* Create a reconstruction session on p->device.  Replaces `new IPhaser` + CXParams::parseFromCPython
 * (src/ptychopy.c:474-482, src/Parameters.cpp:380-653); the parameter struct is per session, not a
 * process-wide singleton. */
int pty_session_create(const pty_params* p, pty_session** out);

/* Release all device and host resources.  Replaces `delete phaser` (src/ptychopy.c:489). */
int pty_session_destroy(pty_session* s);

/* Diffraction data, P patterns of N x N, as float32 (dtype PTY_F32) or float64 (PTY_F64), raster order
 * i*scanDimsy+j.  float32 data may also be passed as a device pointer (unified addressing).  ePIE/DM take amplitudes, MLs intensities (it square-roots them), as in the reference.
 * Replaces Diffractions::loadarr (src/Diffractions.cpp:159-186) fed from diffractionNP (src/ptychopy.c:357-362). */
int pty_set_patterns(pty_session* s, const void* host, int dtype, int P, int N);

/* Scan positions in metres, P x 2 (x, y) float64.  Replaces ListScanMesh::loadarr (src/ListScanMesh.cpp:91-103)
 * fed from positionNP (src/ptychopy.c:364-376).  Without it a Cartesian raster is generated
 * (CartesianScanMesh::generateMesh, src/CartesianScanMesh.cpp:57-92). */
int pty_set_positions(pty_session* s, const double* xy_m, int P);

/* Initial object, complex64 X x Y (must equal the size the scan geometry implies; see pty_get_dims).
 * Replaces Sample::loadarr (src/Sample.cpp:184-198) fed from objectNP (src/ptychopy.c:378-421). */
int pty_set_object(pty_session* s, const float* c64, int X, int Y);

/* Initial probe modes, complex64 K x N x N, K <= probeModes.  K = 1 replaces Probe::init's probearr branch
 * (src/Probe.cpp:354-358, fed from probeNP at src/ptychopy.c:423-471); K > 1 supplies all modes (extension). */
int pty_set_probe(pty_session* s, const float* c64, int K, int N);

/* Build geometry, probe guess and device state.  Replaces IPhaser::init + prePhase (src/IPhaser.cpp:224-365).
 * Fails (PTY_ERR_INVALID) when patterns are missing or a position is negative. */
int pty_init(pty_session* s);

/* One iteration of the session's algorithm (iteration counter i+1 drives the phaseConstraint / updateProbe /
 * updateModes schedule).  Replaces IPhaser::phasestepvis / phaseStep (src/IPhaser.cpp:391-398,479-494) and the
 * epiestep / mlsstep calls (src/ptychopy.c:955-962,1036-1043).  err (may be NULL) receives the error metric
 * (0 unless calculateRMS). */
int pty_step(pty_session* s, double* err);

/* `iters` iterations (errs may be NULL or hold `iters` values).  Replaces IPhaser::phaseLoop
 * (src/IPhaser.cpp:367-389). */
int pty_run(pty_session* s, int iters, double* errs);

/* Multi-GPU DM by position shards (one process per GPU).  The reference runs one GPU per reconstruction (its
 * MPIPhaser stitches separate reconstructions and is not a counterpart); DM's increments are sums over positions, so
 * a scan splits over GPUs with one reduction of the increments per iteration.
 *
 * pty_set_shard: this session holds positions [first, first + P) of a scan of `total` positions, P being the pattern
 * count given to pty_set_patterns; geometry and object size are the whole scan's.  Call before pty_init; DM only; the
 * probe must be given (probeNP or probeGuess).  Sharded sessions step with pty_dm_step_local (this shard's waves:
 * the object / probe increments accumulate on the device), a sum of the increments over all shards in place on the
 * session's stream (pty_dm_increments gives the complex64 buffers and their element counts; e.g. an NCCL
 * all-reduce), then pty_dm_step_finish (apply, intensity sums, factors), after which every shard holds the same
 * object and probe. */
int pty_set_shard(pty_session* s, int first, int total);
int pty_dm_step_local(pty_session* s);
int pty_dm_increments(pty_session* s, void** dO, size_t* n_obj, void** dP, size_t* n_probe);
int pty_dm_step_finish(pty_session* s);

/* Autotuner (no counterpart in the reference, which has one launch configuration per kernel).  Before pty_init,
 * with the patterns (and positions, probe, object) set: times the launch variants of the session's algorithm for
 * `iters` iterations each (two interleaved rounds, the faster kept) on temporary sessions with the same inputs
 * (DM: patterns per wave, one lane or two lanes of waves in flight; ePIE: shared-memory cluster, cluster or
 * whole-GPU kernel, or the per-position kernel chain with 2, 4 or 8 rows per CTA in its FFT passes), keeps the
 * fastest for this session, and writes a one-line summary with every candidate's ms per iteration into `report`
 * (may be NULL).  MLs has no variants. */
int pty_autotune(pty_session* s, int iters, char* report, int report_len);

/* Learned warm start (no counterpart in the reference, which starts from a constant object, src/Sample.cpp:216-220,
 * or objectNP).  Before pty_init: the parameters (n_params floats, the layout ptychopy_b200/warmstart.py's Net
 * trains: per layer the Cout x Cin x 3 x 3 weights then the Cout biases) of the width-`width` encoder-decoder for the
 * session's N x N patterns; n_params = 0 removes it.  pty_init then runs the network on the session's patterns
 * (BF16 tensor cores), stitches and integrates its predictions into the starting object (instead of the constant
 * start; exclusive with objectNP / objectGuess) and, for DM, starts the exit waves at P * O.  ePIE and DM only;
 * N a multiple of 16, the object at most 512 x 512. */
int pty_set_warm_start(pty_session* s, const float* params, size_t n_params, int width);

/* DM only, after pty_init: sets every exit wave to P * O at its position (probe mode 0, the object and probe as
 * they are now).  The reference starts DM from zero exit waves (m_psiOld, src/DM.cu:95-98), which equals this for its
 * zero object; for a given object (objectNP, a warm start) the zero start makes the first update
 * P_F(2 P O) - P O ~ 0 and discards the object, while this start keeps it. */
int pty_dm_psi_from_object(pty_session* s);

/* Warm-start network kernels (no counterpart in the reference, which has no learned component): float32 NCHW
 * device buffers, asynchronous on `stream`.  pty_nn_conv3x3: y = bias + 3x3 convolution of x (weights Cout x Cin x 3
 * x 3, stride 1, zero padding 1; bias may be NULL), then max(y, 0) if relu != 0.  pty_nn_conv3x3_bwd: gradients of
 * that convolution (without the ReLU) for dy: dx (may be NULL), dw and db (may be NULL), overwritten.
 * pty_nn_relu (in place) / _bwd (g *= y > 0); pty_nn_pool2: 2x2 average to H x W; pty_nn_up2: nearest upsampling of
 * H x W; their _bwd the gradients (H, W the small size, planes = batch x channels).  pty_nn_mse: weighted mean
 * squared error, weight w[i % plane] (w may be NULL: all 1): g = 2 w (p - t) / n and *loss = sum w (p - t)^2 / n.
 * pty_nn_adam: one Adam step (bias-corrected, step >= 1). */
int pty_nn_conv3x3(const float* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H, int W,
                   int relu, void* stream);
int pty_nn_conv3x3_bwd(const float* x, const float* w, const float* dy, float* dx, float* dw, float* db, int B,
                       int Cin, int Cout, int H, int W, void* stream);
int pty_nn_relu(float* a, size_t n, void* stream);
int pty_nn_relu_bwd(const float* y, float* g, size_t n, void* stream);
int pty_nn_pool2(const float* x, float* y, size_t planes, int H, int W, void* stream);
int pty_nn_pool2_bwd(const float* dy, float* dx, size_t planes, int H, int W, void* stream);
int pty_nn_up2(const float* x, float* y, size_t planes, int H, int W, void* stream);
int pty_nn_up2_bwd(const float* dy, float* dx, size_t planes, int H, int W, void* stream);
int pty_nn_mse(const float* p, const float* t, const float* w, size_t plane, float* g, size_t n, double* loss,
               void* stream);
int pty_nn_adam(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                int step, void* stream);

/* Warm start of the object from the network's per-position predictions (no counterpart in the reference, which
 * starts from a constant object, src/Sample.cpp:216-220, or a user-supplied objectNP).  Device pointers.
 * pty_warm_input: network input x[b][i][j] = scale * log1p(amp[b][(i + N/2) % N][(j + N/2) % N]) (B x N x N).
 * pty_warm_stitch: sums the network outputs out (P x 3 x S x S: amplitude, row and column phase differences
 * phi(i+1,j) - phi(i,j) and phi(i,j+1) - phi(i,j), decoded as amp_mean + o * amp_scale and o * grad_scale) of the
 * central S x S window of each position (pixel positions P x 2, rounded) into acc (4 x X x Y: weighted amplitude,
 * row and column differences, and the weight), weighting by weight (S x S); deterministic.
 * pty_warm_object: the object from acc: amplitude = weighted mean (amp_fill where the weight is <= wmin), phase = the
 * least-squares integral of the mean differences (FFT Poisson solve on the periodic M x M grid, M the power of two
 * >= max(X, Y), at most 512), then the whole object scaled so that sum_p sum |P O_p|^2 * N^2 equals the data's
 * sum amp^2 (amp: P x N x N, probe N x N complex64).  work: 6 M^2 + 4 floats.  Returns after the stream is done. */
int pty_warm_input(const float* amp, float* x, int B, int N, float scale, void* stream);

/* Tensor-core (tcgen05) BF16 inference path of the warm-start network (no counterpart in the reference).
 * Activations are NHWC BF16 device buffers.  pty_tc_weights_size: BF16 elements of a packed layer (Cout <= 256),
 * -1 if unsupported; pty_tc_pack_weights: packs FP32 weights (Cout x Cin x 3 x 3) into that layout.
 * pty_tc_conv3x3: y = bias + 3x3 convolution (output H x W) of the input, then max(y, 0) if relu; FP32 accumulation
 * in tensor memory.  Input in_mode 0: x NHWC BF16 B x H x W x Cin (Cin a multiple of 8 or at most 8); 1: x NHWC BF16
 * B x H/2 x W/2 x Cin, read 2x nearest-upsampled; 2: x FP32 amplitudes B x H x W (Cin = 1) read as
 * in_scale * log1p(amp) with the zero frequency moved to the centre.  Output out_mode 0: y NHWC BF16 (Cout a
 * multiple of 8); 1: y NCHW FP32; 2: y NHWC BF16 2x2-average-pooled to H/2 x W/2 (H even, W a multiple of 16; or
 * H a multiple of 16 and W of 8 for the thin layers below).  Thin layers (Cin 16, 32 or 64, packed weights plus
 * three input halos within one CTA's shared memory, H a multiple of 16, W of 8, in_mode 0 or 1) run as nine shifted
 * GEMMs over an input halo held in shared memory; the rest as an implicit GEMM with im2col staging.
 * *err (device int, zero on entry) receives a non-zero code if a pipeline wait timed out.
 * pty_tc_first_layer: the network's first layer on CUDA cores (K = 9 is too thin for tensor cores): y (NHWC BF16,
 * B x H/2 x W/2 x 16) = pool2(relu(bias + conv3x3(in_scale * log1p(centred amp)))) for FP32 amplitudes amp
 * (B x H x W) and FP32 weights (16 x 1 x 3 x 3), inputs and weights rounded to BF16 like the tensor-core layers.
 * pty_tc_last_layer: the output layer on CUDA cores: y (NCHW FP32) = bias + conv3x3(x), x NHWC BF16 with Cin = 32,
 * Cout <= 4, FP32 weights (rounded to BF16).
 * pty_tc_pool2 / pty_tc_up2: 2x2 average pooling to H x W / nearest upsampling of H x W, NHWC BF16, C channels.
 * pty_tc_to_bf16: n FP32 values to BF16.  All asynchronous on `stream`. */
int pty_tc_weights_size(int Cin, int Cout);
int pty_tc_pack_weights(const float* w, int Cin, int Cout, void* wpk, void* stream);
int pty_tc_conv3x3(const void* x, const void* wpk, const float* bias, void* y, int B, int Cin, int Cout, int H, int W,
                   int relu, int in_mode, int out_mode, float in_scale, int* err, void* stream);
int pty_tc_first_layer(const float* amp, const float* w, const float* bias, void* y, int B, int Cout, int H, int W,
                       float in_scale, void* stream);
int pty_tc_last_layer(const void* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H,
                      int W, void* stream);
int pty_tc_pool2(const void* x, void* y, int B, int H, int W, int C, void* stream);

/* Failure detection of the bounded device waits, without a GPU fault.  codes[0]: an mbarrier wait on a phase that
 * nothing completes gave up (1 expected); codes[1]: the same wait after one arrival did not (0 expected);
 * codes[2]: 64 grid barriers over 16 CTAs of a cooperative launch that reach their count timed out (0 expected);
 * codes[3]: a grid barrier expecting one arrival too many timed out and every CTA returned (1 expected).
 * Synchronous, on the current device, a few milliseconds. */
int pty_selftest_bounded_waits(int* codes);
int pty_tc_up2(const void* x, void* y, int B, int H, int W, int C, void* stream);
int pty_tc_to_bf16(const float* x, void* y, size_t n, void* stream);
int pty_warm_stitch(const float* out, const float* pos_px, int P, const float* weight, int S, int N, float amp_mean,
                    float amp_scale, float grad_scale, float* acc, int X, int Y, void* stream);
int pty_warm_object(const float* acc, int X, int Y, float wmin, float amp_fill, const float* probe_c64, int N,
                    const float* pos_px, int P, const float* amp, float* work, float* obj_c64, void* stream);

/* Forward model of simulation mode: amp_out[i] = |FFT2(O_bilinear(pos_px[i]) * P)| (P x N x N float32) for an
 * object (X x Y complex64), one probe mode (N x N complex64) and pixel positions (P x 2, x = row; the fractional part
 * is the bilinear texture offset).  Replaces Diffractions::simulate (src/Diffractions.cpp:80-117, d_simulatePSI
 * src/SampleKernels.cu:113-122); the reference builds its object from PGM images, here the caller passes it.
 * obj_c64, probe_c64 and amp_out may be host or device memory, pos_px is host memory; runs on the current device. */
int pty_simulate(const float* obj_c64, int X, int Y, const float* probe_c64, int N, const float* pos_px, int P,
                 float* amp_out);

/* `iters` iterations of each of n initialised sessions (any mix of ePIE, DM and MLs on one device), interleaved:
 * every round enqueues one iteration of every session on that session's own stream, without host
 * synchronisation between DM and MLs steps, so independent scans of uneven sizes share the GPU.  Returns after all
 * streams have finished.  No counterpart in the reference, which runs one reconstruction per process (its
 * IPhaser::phaseLoop, src/IPhaser.cpp:367-389, per session); error metrics are not collected. */
int pty_batch_run(pty_session* const* sessions, int n, int iters);

/* Sizes: object X, Y; probe modes K, size N; pattern count P; iterations done. */
int pty_get_dims(const pty_session* s, int* X, int* Y, int* K, int* N, int* P, int* iters_done);

/* Copy the object (X x Y complex64) to the host.  Replaces epieresobj / mlsresobj (src/ptychopy.c:964-976). */
int pty_get_object(pty_session* s, float* c64_out, int X, int Y);

/* Copy the session's diffraction data (P x N x N float32, natural layout) to the host: the patterns as the
 * iterations read them, after file ingest and its preprocessing or after simulation mode's forward model.  No single
 * reference counterpart (Diffractions::getPatterns, src/Diffractions.h, is its internal accessor). */
int pty_get_patterns(pty_session* s, float* out, int P, int N);

/* Copy the probe stack (K x N x N complex64).  Replaces epieresprobe / mlsresprobe (src/ptychopy.c:978-990). */
int pty_get_probe(pty_session* s, float* c64_out, int K, int N);

/* Device memory freed by destroyed sessions stays cached for the next session of this process (unmapping the
 * buffers of a large DM session took up to 160 ms).  This returns the cache of `device` (-1: every device) to the
 * driver.  No reference counterpart (the reference frees with cudaFree). */
int pty_release_cached_memory(int device);

/* Scan positions in pixels after the -min shift, P x 2 float32 (IPtychoScanMesh::getScanPositions).  MLs keeps
 * the ML mesh's centred positions; on its default path these are the current, refined positions (m_positions). */
int pty_get_positions(const pty_session* s, float* xy_px, int P);

/* MLs default path: the extra (variable) probe mode E (N x N complex64) and the probe evolution weights evo0
 * (intensity) and evo1 (extra mode), P doubles each (Probe::m_extramodes, m_probe_evolution).  Any pointer may be
 * NULL.  PTY_ERR_STATE for other algorithms and for mlsCore = 1. */
int pty_get_mls_state(const pty_session* s, float* E_c64, double* evo0, double* evo1, int N, int P);

/* Write `<dir>/<jobID>_probes_<r>.{csv|bin}` and `<dir>/<jobID>_object_<r>.{csv|bin}`.  Replaces
 * IPhaser::writeResultsToDisk (src/IPhaser.cpp:417-428) with the CSV format of Cuda2DArray::save
 * (src/Cuda2DArray.hpp:439-464, src/Cuda2DArray.cpp:46-52). */
int pty_write_results(pty_session* s, const char* dir, int r, int binary);

/* Run all subsequent device work of the session on this cudaStream_t (NULL = the session's own stream). */
int pty_set_stream(pty_session* s, void* cuda_stream);

/* Number of this library's kernel launches issued by the session so far (graph nodes counted per launch). */
int64_t pty_kernel_launches(const pty_session* s);

/* Message of the last failure on the calling thread ("" if none). */
const char* pty_last_error(void);

/* ---- device-pointer operators (building blocks, used by the parity tests) ---------------------------- */

/* The whole-mode ingest's preprocessing of `count` raw patterns (rows x cols float32, device) into size x size
 * patterns (device): crop / zero-pad around the centre (qx, qy) unless the raw pattern is already size x size
 * (h_symmetrizeDiffraction, src/DiffractionLoader.cpp:86-107), a quarter turn when rotate90 % 4 == 1 (d_rot90,
 * src/DiffractionLoader.cpp:116-121), then the quadrant swap when fftShift != 0 (h_shiftFFT,
 * src/DiffractionLoader.cpp:123-125).  Asynchronous on `stream`. */
int pty_preprocess_patterns(const float* raw_dev, int count, int rows, int cols, int size, int qx, int qy,
                            int rotate90, int fftShift, float* out_dev, void* stream);

/* In-place batched 2-D FFT of `batch` N x N complex64 arrays in device memory (unnormalised; forward uses
 * exp(-2*pi*i*k*n/N), the CUFFT_FORWARD convention).  Replaces the cuFFT plans of FFTPlanner
 * (src/CudaFFTPlan.cpp:72-101).  `work_dev` is a device buffer of batch*N*N complex64. */
int pty_fft2_dev(void* data_dev, void* work_dev, int batch, int N, int inverse, void* cuda_stream);

/* Mixed-precision batched 2-D FFT on the tensor cores (no counterpart in the reference, which calls cuFFT in FP32,
 * src/CudaFFTPlan.cpp:91-101): every 256-point line transform is two radix-16 DFT stages computed as tcgen05 GEMMs
 * with split-BF16 operands (x = x_hi + x_lo, the three products x_hi F_hi + x_lo F_hi + x_hi F_lo) and FP32
 * accumulation, with FP32 twiddles between the stages.  In place on data (batch x N x N complex64, N = 256), work the
 * same size; unnormalised like pty_fft2_dev.  *err (device int, zero on entry) receives a non-zero code if a
 * tensor-core wait timed out.  Asynchronous on `stream`. */
int pty_fft2_tc(void* data, void* work, int batch, int N, int inverse, int* err, void* stream);

/* Allocation-free variant of pty_fft2_dev.  No counterpart in the reference (it has no entry point that avoids
 * allocation).  For callers that cannot call cudaMalloc: hosts that hand the library only buffers they allocated
 * up front and forbid allocation afterwards, such as an acquisition service that owns all device memory of the
 * GPU for the length of a run.  The work buffer and twiddle tables live in a static device array inside this
 * library (8 MiB plus 8 KiB), so the call allocates nothing; the caller passes only the data, transformed in place
 * (batch x N x N complex64, N in {32, 64, 128, 256, 512}).  Requests with batch*N*N*8 > 8 MiB are rejected with
 * PTY_ERR_INVALID.
 * The static array occupies device memory from the moment the CUDA runtime loads this library's device code onto
 * a GPU until the process exits.  With the runtime's default lazy loading that happens on the first call on that
 * device (which also resolves the array's address and fills the twiddles with a synchronous copy), and each
 * transform size's kernels are loaded on the first call with that size, so those first calls need free device
 * memory (~8 MiB, then the code): make one call per size the host will use at start-up, before it claims the
 * GPU's memory and before any stream capture (or run with CUDA_MODULE_LOADING=EAGER, which loads everything when
 * the CUDA context is created).  Later calls allocate nothing.  The launch is asynchronous on `cuda_stream`.  All
 * calls on a device share the one scratch array, which keeps the last call's contents (it is fully overwritten
 * before it is read, so nothing needs clearing); calls that overlap on the GPU, e.g. on two streams at once, race
 * on it and must be serialised by the caller. */
int pty_fft2_dev_noalloc(void* data_dev, int batch, int N, int inverse, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* PTYCHOPY_B200_H_ */
