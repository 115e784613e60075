// Host-side session state of one reconstruction (the engine's counterpart of the reference's IPhaser with its
// Sample, Probe, Diffractions and scan-mesh members, src/IPhaser.h:58-115), owned through the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ptychopy_b200.h"

namespace pty {

enum Algo { ALGO_EPIE = 0, ALGO_DM = 1, ALGO_MLS = 2 };

// Thrown inside the library and turned into a status code + message at the C boundary.
struct Error {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);

// Scan geometry in pixels (IPtychoScanMesh): positions shifted by -min, object size ceil(max - min + N).
struct Geometry {
  std::vector<float> pos;  // 2*P (x = row, y = column)
  int X = 0, Y = 0;
};
double sample_pixel_size(double lambda, double z, double dx_d, int N);
// dfx, dfy: the scan drift in metres per mesh-array row / column (0 = none).
Geometry cartesian_geometry(int nx, int ny, double stepx, double stepy, double dx_s, int N, bool mirrorX,
                            bool mirrorY, bool flip, unsigned jitter, uint64_t seed, float dfx, float dfy);
Geometry list_geometry(const std::vector<double>& xy_m, double dx_s, int N, bool flip, unsigned jitter,
                       uint64_t seed, float dfx, float dfy);
Geometry spiral_geometry(int P, double stepx, double stepy, double dx_s, int N, bool flip, unsigned jitter,
                         uint64_t seed, float dfx, float dfy);
std::vector<double> read_position_file(const std::string& path, int P);

// SplitMix64 stream and the ePIE visiting order (pick `next % remaining`, erase; src/ePIE.cpp:93-97).
uint64_t splitmix64(uint64_t& state);
void visiting_order(uint64_t& state, int P, std::vector<int>& order);

// Device buffer.  Its memory comes from and returns to a per-device cache of freed blocks (session.cu).
struct DeviceBuf {
  void* p = nullptr;
  size_t bytes = 0;      // requested size
  size_t cap = 0;        // size of the underlying block
  int dev = -1;
  DeviceBuf() = default;
  DeviceBuf(const DeviceBuf&) = delete;  // one owner per block: a copy would return it to the cache twice
  DeviceBuf& operator=(const DeviceBuf&) = delete;
  void alloc(size_t n, const char* what);
  void free();
  // exchange the blocks of two buffers (every field: a block returns to the cache under its own size)
  void swap(DeviceBuf& o) {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
    std::swap(cap, o.cap);
    std::swap(dev, o.dev);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
  ~DeviceBuf() { free(); }
};

struct EpieState;  // device state of the persistent ePIE kernel (kernels_epie.cu)
struct MlsState;   // device state of the MLs core (kernels_mls.cu)

// ML-mesh geometry (src/CartesianScanMesh.cpp:94-177, src/IPtychoScanMesh.cpp:123-184): object ceil(extent * 1.2)
// per axis, window starts round(pos + ceil(X/2 - N/2)) - 1 from the raw centred positions, and the object ROI that
// calc_object_norm uses.
struct MlsGeometry {
  int X = 0, Y = 0;
  std::vector<int> r0, c0;
  int roi[4] = {0, 0, 0, 0};  // x0, y0, nx, ny (0-based)
};
MlsGeometry mls_geometry(const std::vector<float>& raw, int N);
// Learned warm start (warm_start.cu): parameter count of the width-w network for N x N patterns, and the
// inference + assembly that writes the session's starting object inside pty_init.
size_t warm_param_count(int N, int w);
void run_warm_start(pty_session* s);
// Whole-mode ingest (ingest.cu): the P patterns of the data files named by the session's fp, preprocessed on the
// device into the session's pattern buffer.
void ingest_patterns(pty_session* s, int P);
// Simulation mode (sim_mode.cu): the patterns from the forward model of the reference's PGM object and simulated
// probe at the session's scan positions (geometry set); the object and probe of the simulation, for the tests.
void simulate_session_patterns(pty_session* s);
std::vector<float> sim_object_from_files(int N, int X, int Y);
std::vector<float> sim_probe(int N, double beamSize, double dx_s, uint64_t seed);

std::vector<float> raw_cartesian_positions(int nx, int ny, double stepx, double stepy, double dx_s, bool mirrorX,
                                           bool mirrorY, float dfx, float dfy);

}  // namespace pty

struct pty_session {
  pty_params prm{};
  pty::Algo algo = pty::ALGO_EPIE;
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int N = 0, K = 1, P = 0, X = 0, Y = 0;
  int iter = 0;
  bool initialized = false;
  int64_t launches = 0;

  // inputs
  bool have_patterns = false;
  std::vector<double> pos_m;  // positions in metres (positionNP) or empty
  std::vector<float> obj_h;   // objectNP (X*Y complex) or empty
  std::vector<float> probe_h; // probeNP (Kg*N*N complex) or empty
  int probe_given_modes = 0;
  std::vector<float> warm_params;  // trained warm-start network (pty_set_warm_start) or empty
  int warm_width = 0;
  int fft_rows = 0;       // ePIE kernel chain: rows per CTA of its transform passes (0 automatic; set by the autotuner)
  int epie_variant = -1;  // ePIE kernel: -1 automatic, 0 shared-memory cluster, 1 cluster, 2 whole-GPU, 3 a chain
                          // of whole-GPU kernels per position (autotuner; precision = 1 always runs the chain)

  // geometry
  pty::Geometry geo;
  std::vector<int> offs;  // rounded offsets, 2*P

  // device state
  pty::DeviceBuf amp;    // P*N*N float (natural layout; sessions of the cluster ePIE kernel transpose each plane)
  bool amp_transposed = false;
  pty::DeviceBuf obj, probe, ocache, pcache;
  pty::DeviceBuf tw, dOffs, scal;
  // DM
  pty::DeviceBuf psi, dO, dP, W1, W2, slots;
  int dm_lanes = 1;                // waves in flight side by side (W1 / W2 hold one wave per lane)
  int dm_lanes_req = 0;            // 0: automatic (two when there are two waves or more); 1: one lane (autotuner)
  cudaStream_t dm_side = nullptr;  // the second lane's stream (forked from and joined to the session's stream)
  cudaEvent_t dm_fork = nullptr, dm_join = nullptr;
  pty::DeviceBuf dm_err;  // wait-timeout flag of the tensor-core column pass (precision = 1)
  int wave = 0, nwaves = 0;
  cudaGraphExec_t graphs[4] = {nullptr, nullptr, nullptr, nullptr};
  // position sharding (DM over several GPUs): this session holds positions [shard_first, shard_first + P) of a scan
  // of shard_total positions; local step (waves) and finish (apply the summed increments) are separate graphs
  int shard_first = 0, shard_total = 0;
  cudaGraphExec_t graphs_local[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t graphs_fin[2] = {nullptr, nullptr};
  int pending_iter = 0;
  // ePIE
  pty::EpieState* ep = nullptr;
  // MLs
  pty::MlsState* ml = nullptr;
  uint64_t rng = 0;
  double objMax0 = 0, probeMax0 = 1;
  bool useAll = false, modesInitialized = false;
  std::vector<double> sqsum;
};
