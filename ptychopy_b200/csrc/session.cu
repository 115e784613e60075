// Host orchestration and the C ABI (include/ptychopy_b200.h).  One pty_session is one reconstruction: the
// reference's IPhaser + CXParams pair (src/IPhaser.cpp:224-365, src/Parameters.cpp:380-653), with parameters
// held per session instead of in a process-wide singleton.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "kernels.h"
#include "kernels_epie.h"
#include "kernels_mls.h"
#include "session.h"

namespace pty {

static thread_local std::string g_last_error;

[[noreturn]] void fail(int code, const std::string& msg) { throw Error{code, msg}; }

// Sets the calling thread's pty_last_error() message (for entry points outside the guarded() wrapper).
void set_last_error(const std::string& msg) { g_last_error = msg; }

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  const int code = (e == cudaErrorMemoryAllocation) ? PTY_ERR_OOM : PTY_ERR_CUDA;
  fail(code, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

void need_device_index(int d) {
  if (d < 0 || d >= 64) fail(PTY_ERR_UNSUPPORTED, "device ordinal " + std::to_string(d) + " above the buffer cache's 64");
}

// Freed device blocks are kept per device and handed to the next request of at least their size and at most a
// quarter more: cudaFree of a DM session's buffers (about 3 GB at 512^2 x 900 patterns) unmaps the memory and took
// 10-160 ms, up to a third of a 100-iteration dmnp call, and the next session mapped it again.
// Ordering is per stream: inside a session's call the calling thread is bound to the session's stream (set_device;
// guarded() restores the previous binding on return), a freed block enters the cache with an event recorded on that stream after its last use, and the next taker waits
// for that event on its own stream; a new buffer is cleared on the bound stream and that stream alone is
// synchronised.  Without a bound stream (the stand-alone entry points) both fall back to a device synchronisation.
// pty_release_cached_memory returns the cache to the driver; so does an allocation that fails, before its one retry.
namespace {
constexpr int kMaxDevices = 64;
struct CachedBlock {
  void* p;
  cudaEvent_t ready;  // recorded after the block's last use, or null (already idle)
};
std::mutex g_cache_mu;
std::multimap<size_t, CachedBlock> g_cache[kMaxDevices];
thread_local cudaStream_t t_stream = nullptr;

void* cache_take(int dev, size_t n, size_t* cap, cudaEvent_t* ready) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto& c = g_cache[dev];
  auto it = c.lower_bound(n);
  if (it == c.end() || it->first > n + n / 4) return nullptr;
  void* q = it->second.p;
  *ready = it->second.ready;
  *cap = it->first;
  c.erase(it);
  return q;
}

void cache_release(int dev) {
  std::multimap<size_t, CachedBlock> blocks;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    blocks.swap(g_cache[dev]);
  }
  if (blocks.empty()) return;
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  for (auto& kv : blocks) {
    if (kv.second.ready) {
      cudaEventSynchronize(kv.second.ready);
      cudaEventDestroy(kv.second.ready);
    }
    cudaFree(kv.second.p);
  }
  if (cur != dev) cudaSetDevice(cur);
}
}  // namespace

void DeviceBuf::alloc(size_t n, const char* what) {
  free();
  if (n == 0) n = 16;
  // a failure names the buffer and the CUDA call (the message is built only then)
  auto checked = [what](cudaError_t e, const auto& step) {
    if (e != cudaSuccess) check_cuda(e, (std::string(what) + ": " + step()).c_str());
  };
  int d = 0;
  checked(cudaGetDevice(&d), [] { return std::string("cudaGetDevice"); });
  need_device_index(d);
  size_t got = 0;
  cudaEvent_t ready = nullptr;
  void* q = cache_take(d, n, &got, &ready);
  const bool recycled = q != nullptr;
  if (q && ready) {  // the block's last user may still be running
    const cudaError_t e = t_stream ? cudaStreamWaitEvent(t_stream, ready, 0) : cudaEventSynchronize(ready);
    cudaEventDestroy(ready);
    if (e != cudaSuccess) {
      cudaFree(q);
      checked(e, [] { return std::string("wait for the recycled block's last use"); });
    }
  }
  if (!q) {
    cudaError_t e = cudaMalloc(&q, n);
    if (e == cudaErrorMemoryAllocation) {  // give the cache back and try once more
      cudaGetLastError();
      cache_release(d);
      e = cudaMalloc(&q, n);
    }
    checked(e, [n] { return "cudaMalloc of " + std::to_string(n) + " bytes"; });
    got = n;
  }
  // every buffer starts at zero (accumulators, counters and padding rely on it), whether recycled or fresh (cudaMalloc
  // does not promise cleared memory: pages this process freed may come back as they were); complete before return,
  // since synchronous copies on the legacy stream are not ordered against the sessions' non-blocking streams
  auto clear = [&](const char* call) {
    return [=] {
      return "clearing " + std::to_string(n) + " bytes of a " + std::to_string(got) + "-byte " +
             (recycled ? "recycled" : "new") + " block (" + call + ")";
    };
  };
  if (t_stream) {
    checked(cudaMemsetAsync(q, 0, n, t_stream), clear("cudaMemsetAsync"));
    checked(cudaStreamSynchronize(t_stream), clear("stream synchronize"));
  } else {
    checked(cudaMemset(q, 0, n), clear("cudaMemset"));
    checked(cudaDeviceSynchronize(), clear("device synchronize"));
  }
  p = q;
  bytes = n;
  cap = got;
  dev = d;
}
void DeviceBuf::free() {
  if (p && dev < 0) {  // not from alloc: owned plainly
    cudaFree(p);
  } else if (p) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaEvent_t ready = nullptr;
    if (t_stream && cur == dev && cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) == cudaSuccess) {
      if (cudaEventRecord(ready, t_stream) != cudaSuccess) {
        cudaEventDestroy(ready);
        ready = nullptr;
        cudaDeviceSynchronize();
      }
    } else {
      ready = nullptr;
      cudaDeviceSynchronize();
    }
    {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      g_cache[dev].emplace(cap, CachedBlock{p, ready});
    }
    if (cur != dev) cudaSetDevice(cur);
  }
  p = nullptr;
  bytes = 0;
  cap = 0;
}

// ---- geometry (FP32 like the reference's device code) -------------------------------------------------
// dx_s = lambda*z/(N*dx_d) returned as real_t (float) by Parameters::samplePlanePixelSize (src/Parameters.h:175-179)
double sample_pixel_size(double lambda, double z, double dx_d, int N) {
  return double(float((lambda * z) / (double(N) * dx_d)));
}

// min/max over the M entries of the mesh array, object size ceil(max - min + N) and the -min shift of the first P
// (src/IPtychoScanMesh.cpp:86-109: calculateMeshDimensions reduces over the whole array).
static void finish_geometry(const std::vector<float>& raw, int P, int M, int N, bool flip, Geometry& g) {
  float mnx = std::numeric_limits<float>::max(), mny = mnx, mxx = -mnx, mxy = -mnx;
  for (int i = 0; i < M; ++i) {
    mnx = std::min(mnx, raw[2 * i]);
    mxx = std::max(mxx, raw[2 * i]);
    mny = std::min(mny, raw[2 * i + 1]);
    mxy = std::max(mxy, raw[2 * i + 1]);
  }
  volatile float ex = (mxx - mnx) + float(N);
  volatile float ey = (mxy - mny) + float(N);
  g.X = int(std::ceil(float(ex)));
  g.Y = int(std::ceil(float(ey)));
  g.pos.resize(2 * size_t(P));
  for (int i = 0; i < P; ++i) {
    const float tx = raw[2 * i], ty = raw[2 * i + 1];
    g.pos[2 * i] = flip ? ty - mny : tx - mnx;
    g.pos[2 * i + 1] = flip ? tx - mnx : ty - mny;
  }
}

// Position jitter, r - u*2r per axis in pixels (src/ScanMeshKernels.cu:53-60, where u comes from curand with a
// time seed).  Seeded here: SplitMix64 from seed ^ 0x6A09E667F3BCC909, u = ((next >> 40) + 1) * 2^-24 in (0, 1],
// x before y, positions in mesh-array order (padding included).  Added to raw (already in pixels).
static void add_jitter(std::vector<float>& raw, unsigned radius, uint64_t seed) {
  if (!radius) return;
  uint64_t st = seed ^ 0x6A09E667F3BCC909ull;
  const float r = float(radius);
  for (float& v : raw) {
    const float u = float((splitmix64(st) >> 40) + 1) * (1.0f / 16777216.0f);
    volatile float t = u * 2.0f;
    volatile float t2 = t * r;
    volatile float j = r - t2;
    volatile float w = v + j;
    v = w;
  }
}

// The reference's scan drift (d_generateMesh, src/ScanMeshKernels.cu:86-87): `v += index * drift` in metres and in
// float, index = the mesh array's row (x) or column (y).  Its compiler fuses the add with the multiply that formed
// v where there is one (Cartesian, spiral: fma(a, step, index * drift), measured against the reference's compiled
// kernel) and with index * drift where v is a loaded value (list: fma(index, drift, v)).
static inline float add_drift(float v, int index, float drift) {
  return drift != 0.f ? std::fma(float(index), drift, v) : v;
}
static inline float mul_add_drift(float a, float step, int index, float drift) {
  if (drift == 0.f) return a * step;
  volatile float d = float(index) * drift;
  return std::fma(a, step, float(d));
}

// Cartesian raster (d_generateMesh<1>, src/ScanMeshKernels.cu:46-93): index i*ny+j,
// ((i - (nx-1)/2) * stepx + i * driftx) * (1 / dx_s) in float.
Geometry cartesian_geometry(int nx, int ny, double stepx, double stepy, double dx_s, int N, bool mirrorX,
                            bool mirrorY, bool flip, unsigned jitter, uint64_t seed, float dfx, float dfy) {
  const float inv = float(1.0 / dx_s), sx = float(stepx), sy = float(stepy);
  std::vector<float> raw(2 * size_t(nx) * ny);
  const float mdx = float(nx - 1) * 0.5f, mdy = float(ny - 1) * 0.5f;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      volatile float dx = mirrorX ? (mdx - float(i)) : (float(i) - mdx);
      volatile float vx = mul_add_drift(float(dx), sx, i, dfx);
      volatile float dy = mirrorY ? (mdy - float(j)) : (float(j) - mdy);
      volatile float vy = mul_add_drift(float(dy), sy, j, dfy);
      volatile float px = float(vx) * inv, py = float(vy) * inv;
      raw[2 * (size_t(i) * ny + j)] = px;
      raw[2 * (size_t(i) * ny + j) + 1] = py;
    }
  add_jitter(raw, jitter, seed);
  Geometry g;
  finish_geometry(raw, nx * ny, nx * ny, N, flip, g);
  return g;
}

// Position list in metres (ListScanMesh::loadarr + d_generateMesh<2>, src/ListScanMesh.cpp:91-129).  The mesh
// array holds whole 1024-wide rows; entries past P stay (0, 0) (plus drift and jitter) and join the min/max.
Geometry list_geometry(const std::vector<double>& xy_m, double dx_s, int N, bool flip, unsigned jitter,
                       uint64_t seed, float dfx, float dfy) {
  const int P = int(xy_m.size() / 2);
  const int M = (P + 1023) / 1024 * 1024;
  const float inv = float(1.0 / dx_s);
  std::vector<float> raw(2 * size_t(M), 0.f);
  for (int i = 0; i < M; ++i) {
    const float x0 = i < P ? float(xy_m[2 * i]) : 0.f, y0 = i < P ? float(xy_m[2 * i + 1]) : 0.f;
    volatile float x = add_drift(x0, i / 1024, dfx), y = add_drift(y0, i % 1024, dfy);
    volatile float px = float(x) * inv, py = float(y) * inv;
    raw[2 * i] = px;
    raw[2 * i + 1] = py;
  }
  add_jitter(raw, jitter, seed);
  Geometry g;
  finish_geometry(raw, P, M, N, flip, g);
  return g;
}

// Spiral (d_generateMesh<3>, src/ScanMeshKernels.cu:77-82; SpiralScanMesh::generateMesh,
// src/SpiralScanMesh.cpp:57-84): point i at sqrt(i) * (cos, sin)(4 sqrt(i)) * step / dx_s.  Every entry of the
// 1024-wide mesh array is a spiral point, so the min/max cover ceil(P/1024)*1024 points.  cos/sin of the float
// argument are evaluated in double and rounded to float.
Geometry spiral_geometry(int P, double stepx, double stepy, double dx_s, int N, bool flip, unsigned jitter,
                         uint64_t seed, float dfx, float dfy) {
  const int M = (P + 1023) / 1024 * 1024;
  const float inv = float(1.0 / dx_s), sx = float(stepx), sy = float(stepy);
  std::vector<float> raw(2 * size_t(M));
  for (int i = 0; i < M; ++i) {
    const float r = std::sqrt(float(i));
    const float a = 4.0f * r;
    const float c = float(std::cos(double(a))), sn = float(std::sin(double(a)));
    volatile float vx = r * c, vy = r * sn;
    volatile float wx = mul_add_drift(vx, sx, i / 1024, dfx), wy = mul_add_drift(vy, sy, i % 1024, dfy);
    volatile float px = wx * inv, py = wy * inv;
    raw[2 * i] = px;
    raw[2 * i + 1] = py;
  }
  add_jitter(raw, jitter, seed);
  Geometry g;
  finish_geometry(raw, P, M, N, flip, g);
  return g;
}

// Position list file (ListScanMesh::loadList, src/ListScanMesh.cpp:65-89): P lines "x,y" in metres.
std::vector<double> read_position_file(const std::string& path, int P) {
  std::ifstream f(path);
  if (!f.is_open()) fail(PTY_ERR_IO, "cannot open the position list file " + path);
  std::vector<double> xy(2 * size_t(P));
  for (int i = 0; i < P; ++i) {
    char comma = 0;
    if (!(f >> xy[2 * i]) || !(f >> comma) || comma != ',' || !(f >> xy[2 * i + 1]))
      fail(PTY_ERR_INVALID, "position list file " + path + ": line " + std::to_string(i + 1) +
                                " is not 'x,y' (expected " + std::to_string(P) + " lines)");
  }
  return xy;
}

// Raw (centred, not shifted) Cartesian positions of the ML mesh: the same FP32 formula as cartesian_geometry.
std::vector<float> raw_cartesian_positions(int nx, int ny, double stepx, double stepy, double dx_s, bool mirrorX,
                                           bool mirrorY, float dfx, float dfy) {
  const float inv = float(1.0 / dx_s), sx = float(stepx), sy = float(stepy);
  std::vector<float> raw(2 * size_t(nx) * ny);
  const float mdx = float(nx - 1) * 0.5f, mdy = float(ny - 1) * 0.5f;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      volatile float dx = mirrorX ? (mdx - float(i)) : (float(i) - mdx);
      volatile float vx = mul_add_drift(float(dx), sx, i, dfx);
      volatile float dy = mirrorY ? (mdy - float(j)) : (float(j) - mdy);
      volatile float vy = mul_add_drift(float(dy), sy, j, dfy);
      volatile float px = float(vx) * inv, py = float(vy) * inv;
      raw[2 * (size_t(i) * ny + j)] = px;
      raw[2 * (size_t(i) * ny + j) + 1] = py;
    }
  return raw;
}

MlsGeometry mls_geometry(const std::vector<float>& raw, int N) {
  const int P = int(raw.size() / 2);
  float mnx = std::numeric_limits<float>::max(), mny = mnx, mxx = -mnx, mxy = -mnx;
  for (int i = 0; i < P; ++i) {
    mnx = std::min(mnx, raw[2 * i]);
    mxx = std::max(mxx, raw[2 * i]);
    mny = std::min(mny, raw[2 * i + 1]);
    mxy = std::max(mxy, raw[2 * i + 1]);
  }
  // the extent loop works in a 1e5-wide frame; note its x bounds come from the positions' y and vice versa
  const float frame = std::ceil(1e5f * 1.0f / 2 - float(N) * 1.0f / 2);
  const float cx = (mxx + mnx) / 2, cy = (mxy + mny) / 2;
  long long lox = 1LL << 40, hix = -1, loy = 1LL << 40, hiy = -1;
  for (int i = 0; i < P; ++i) {
    const long long tx = (long long)std::round(raw[2 * i + 1] - cy + frame);
    lox = std::min(lox, tx - 1);
    hix = std::max(hix, tx + N - 2);
    const long long ty = (long long)std::round(raw[2 * i] - cx + frame);
    loy = std::min(loy, ty - 1);
    hiy = std::max(hiy, ty + N - 2);
  }
  MlsGeometry g;
  g.X = int(std::ceil(double(float(hix - lox) * (1 + 0.2f))));
  g.Y = int(std::ceil(double(float(hiy - loy) * (1 + 0.2f))));
  const float ox = std::ceil(float(g.X) * 1.0f / 2 - float(N) * 1.0f / 2);
  const float oy = std::ceil(float(g.Y) * 1.0f / 2 - float(N) * 1.0f / 2);
  g.r0.resize(P);
  g.c0.resize(P);
  for (int i = 0; i < P; ++i) {
    g.r0[i] = int(std::round(raw[2 * i] + ox)) - 1;
    g.c0[i] = int(std::round(raw[2 * i + 1] + oy)) - 1;
  }
  const long long ax = (long long)std::round(g.X * 0.5 + mnx), bx = (long long)std::round(g.X * 0.5 + mxx) - 1;
  const long long ay = (long long)std::round(g.Y * 0.5 + mny), by = (long long)std::round(g.Y * 0.5 + mxy) - 1;
  g.roi[0] = int(ax - 1);
  g.roi[1] = int(ay - 1);
  g.roi[2] = int(bx - ax + 1);
  g.roi[3] = int(by - ay + 1);
  // kept inside the object (the reference indexes it unchecked); an empty range stays empty
  for (int a = 0; a < 2; ++a) {
    const int len = a == 0 ? g.X : g.Y;
    const int end = std::min(len, g.roi[a] + std::max(g.roi[a + 2], 0));
    g.roi[a] = std::max(0, std::min(g.roi[a], len));
    g.roi[a + 2] = std::max(0, end - g.roi[a]);
  }
  return g;
}

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void visiting_order(uint64_t& state, int P, std::vector<int>& order) {
  std::vector<int> rem(P);
  for (int i = 0; i < P; ++i) rem[i] = i;
  order.resize(P);
  for (int s = 0; s < P; ++s) {
    const int k = int(splitmix64(state) % uint64_t(rem.size()));
    order[s] = rem[k];
    rem.erase(rem.begin() + k);
  }
}

// Device state of the persistent ePIE kernel.
struct EpieState {
  DeviceBuf pos, order, W1, W2, TM, pm, sc, sq, modesCopy, ip, gsync;
  bool chain = false;     // the per-position kernel chain (variant 3, or precision = 1)
  bool chain_tc = false;  // its transforms on the tensor cores (precision = 1)
  DeviceBuf cpsi, cwork, pmax2, tcerr;
  // the chain's iteration as a CUDA graph per schedule regime (active modes, probe update, phase constraint,
  // error metric); the visiting order is read from device memory at each replay
  std::map<unsigned, cudaGraphExec_t> chain_graphs;
  int C = 1, TX = 0, TY = 0;
  bool tm_valid = false;
  bool sm = false;    // shared-memory-resident kernel (small windows, one mode)
  bool grid = false;  // whole-GPU variant of k_epie (N = 256, 512): C CTAs in a cooperative launch
  int* order_h = nullptr;  // pinned
  ~EpieState() {
    if (order_h) cudaFreeHost(order_h);
    for (auto& kv : chain_graphs) cudaGraphExecDestroy(kv.second);
  }
};

// Device state of the MLs core.
// Group tables of one iteration, packed: members (ng x Gmax, -1 padded) | sizes (ng) | boxes (4 ng).  Two sets
// (device copy, pinned host staging, copy-done event, graph reading it) alternate between iterations, so the host
// builds iteration i+1's tables while the GPU runs iteration i and a step needs no synchronisation.
struct MlsTables {
  DeviceBuf dev;
  int* host = nullptr;
  cudaEvent_t copied = nullptr;
  cudaGraphExec_t graph = nullptr;
};

struct MlsState {
  MlsGeometry geo;
  DeviceBuf pobj, S, pum, objp, psi, work, starts, sums, errk, betas, err, norms, maxill, tcerr;
  // the reference-default path: extra mode, evolution weights, positions, sub-pixel shifts, per-position probes and
  // directions, gradient images, scratch sums, max of p_object
  bool variable = false;
  DeviceBuf E, evo, pos, pos_o, sub, vp, pu, aux, vs, pmax, psik, mtmp, vupd, work2;
  cudaStream_t side = nullptr;  // the position search's stream
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int Gmax = 1, ng = 1;
  size_t table_ints = 0;
  MlsTables tab[2];
  // the default path's graphs differ by iteration regime (MlsVarFlags): one per (table set, flags)
  std::map<unsigned, cudaGraphExec_t> var_graphs;
  int64_t steps = 0;
  ~MlsState() {
    for (MlsTables& t : tab) {
      if (t.graph) cudaGraphExecDestroy(t.graph);
      if (t.copied) cudaEventDestroy(t.copied);
      if (t.host) cudaFreeHost(t.host);
    }
    for (auto& kv : var_graphs) cudaGraphExecDestroy(kv.second);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
  }
};

// Seeded stand-ins for the reference's time-seeded draws of the MLs default path: curand uniforms for the extra
// mode (initVarModes, src/Probe.cpp:497-505, d_initVarMOdes src/ProbeKernels.cu:99-110: r1 e^{2 pi i r2}, all r1
// drawn before all r2) and normalRandom for the extra-mode weights (1e-6 N(0,1), src/Probe.cpp:520-525).  SplitMix64
// from seed ^ 0x3C6EF372FE94F82B, u = (bits >> 11 + 0.5) 2^-53, Box-Muller's cos branch, one normal per pair.
// With K > 1 probe modes, 2 (K - 1) normals for the modes' phase tilts (initMLH, src/Probe.cpp:422-431) are drawn
// after the extra mode and before the weights.
void mls_variable_draws(uint64_t seed, int N, int P, int K, std::vector<float2>& E, std::vector<double>& tilts,
                        std::vector<double>& evo1) {
  uint64_t st = seed ^ 0x3C6EF372FE94F82Bull;
  auto u = [&] { return (double(splitmix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
  const size_t NN = size_t(N) * N;
  std::vector<double> r1(NN), r2(NN);
  for (auto& v : r1) v = u();
  for (auto& v : r2) v = u();
  E.resize(NN);
  for (size_t i = 0; i < NN; ++i)
    E[i] = make_float2(float(r1[i] * std::cos(2 * M_PI * r2[i])), float(r1[i] * std::sin(2 * M_PI * r2[i])));
  auto normal = [&] {
    const double a = u(), b = u();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(2 * M_PI * b);
  };
  tilts.resize(2 * size_t(K > 1 ? K - 1 : 0));
  for (auto& v : tilts) v = normal();
  evo1.resize(P);
  for (auto& v : evo1) v = 1e-6 * normal();
}

// Eigen-decomposition of a Hermitian K x K matrix (row-major, complex as double2) by cyclic complex Jacobi
// rotations.  Eigenvectors (columns of V, unit norm) in descending |eigenvalue|, each turned so that its first
// component of at least half the largest magnitude is real and positive (robust to the equal-magnitude components
// of equal-power modes): the reference's ComplexEigenSolver fixes no phase.
void hermitian_eigen(int K, const std::vector<double2>& Ain, std::vector<double2>& Vout) {
  using C = std::complex<double>;
  std::vector<C> A(size_t(K) * K), V(size_t(K) * K, C(0, 0));
  for (size_t i = 0; i < A.size(); ++i) A[i] = C(Ain[i].x, Ain[i].y);
  for (int i = 0; i < K; ++i) V[size_t(i) * K + i] = 1;
  double scale = 0;
  for (const C& v : A) scale += std::norm(v);
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0;
    for (int p = 0; p < K; ++p)
      for (int q = p + 1; q < K; ++q) off += std::norm(A[size_t(p) * K + q]);
    if (off <= 1e-30 * scale) break;
    for (int p = 0; p < K; ++p)
      for (int q = p + 1; q < K; ++q) {
        const C apq = A[size_t(p) * K + q];
        const double m = std::abs(apq);
        if (m == 0.0) continue;
        const double app = A[size_t(p) * K + p].real(), aqq = A[size_t(q) * K + q].real();
        const double th = 0.5 * std::atan2(2 * m, aqq - app);
        const double c = std::cos(th), s = std::sin(th);
        const C em = std::conj(apq) / m;
        for (int k = 0; k < K; ++k) {
          const C x = A[size_t(k) * K + p], y = A[size_t(k) * K + q];
          A[size_t(k) * K + p] = c * x - s * em * y;
          A[size_t(k) * K + q] = s * x + c * em * y;
          const C vx = V[size_t(k) * K + p], vy = V[size_t(k) * K + q];
          V[size_t(k) * K + p] = c * vx - s * em * vy;
          V[size_t(k) * K + q] = s * vx + c * em * vy;
        }
        for (int k = 0; k < K; ++k) {
          const C x = A[size_t(p) * K + k], y = A[size_t(q) * K + k];
          A[size_t(p) * K + k] = c * x - s * std::conj(em) * y;
          A[size_t(q) * K + k] = s * x + c * std::conj(em) * y;
        }
      }
  }
  std::vector<int> idx(K);
  for (int i = 0; i < K; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
    return std::abs(A[size_t(x) * K + x].real()) > std::abs(A[size_t(y) * K + y].real());
  });
  Vout.resize(size_t(K) * K);
  for (int j = 0; j < K; ++j) {
    const int c = idx[j];
    double mx = 0;
    for (int k = 0; k < K; ++k) mx = std::max(mx, std::abs(V[size_t(k) * K + c]));
    int best = 0;
    while (best < K - 1 && std::abs(V[size_t(best) * K + c]) < 0.5 * mx) ++best;
    const C v = V[size_t(best) * K + c];
    const C ph = std::abs(v) > 0 ? std::conj(v) / std::abs(v) : C(1, 0);
    for (int k = 0; k < K; ++k) {
      const C w = V[size_t(k) * K + c] * ph;
      Vout[size_t(k) * K + j] = make_double2(w.real(), w.imag());
    }
  }
}

}  // namespace pty

using namespace pty;

namespace {

template <typename F>
int guarded(F&& f) {
  struct Rebind {  // the caller's stream binding, back in place however f ends
    cudaStream_t saved = t_stream;
    ~Rebind() { t_stream = saved; }
  } rebind;
  try {
    f();
    g_last_error.clear();
    return PTY_OK;
  } catch (const Error& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return PTY_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return PTY_ERR_INVALID;
  }
}

void need(bool cond, const std::string& msg, int code = PTY_ERR_INVALID) {
  if (!cond) fail(code, msg);
}

// The session's device, and its stream as the order for the device buffers allocated and freed from here on.
void set_device(pty_session* s) {
  check_cuda(cudaSetDevice(s->dev), "cudaSetDevice");
  t_stream = s->stream;
}

// A session's own stream.  MLs and ePIE are chains of small dependent kernels whose time is their latency; DM runs
// few large kernels.  The chains get the device's highest stream priority, so that beside other sessions (a batch)
// their blocks are dispatched ahead of queued bulk work.  (The batched 8 DM + 8 MLs configuration measured the same
// with and without it, 195 K vs 194 K patterns/s: its long MLs chains were not waiting behind the DM kernels.)
void create_session_stream(pty_session* s, cudaStream_t* st) {
  int least = 0, greatest = 0;
  check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
  const int prio = (s->algo == ALGO_MLS || s->algo == ALGO_EPIE) ? greatest : least;
  check_cuda(cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, prio), "stream");
}

Algo parse_algo(const char* a) {
  std::string s(a);
  if (s == "ePIE") return ALGO_EPIE;
  if (s == "DM") return ALGO_DM;
  if (s == "MLs") return ALGO_MLS;
  fail(PTY_ERR_INVALID, "unknown algorithm '" + s + "' (expected ePIE, DM or MLs)");
}

// Float32 host->device copy of P*N*N values from float32 or float64 host data.
void upload_patterns(pty_session* s, const void* host, int dtype, size_t n) {
  s->amp.alloc(n * sizeof(float), "patterns");
  if (dtype == PTY_F32) {
    // cudaMemcpyDefault: the source may be host memory (pageable or pinned) or, through UVA, device memory
    check_cuda(cudaMemcpyAsync(s->amp.p, host, n * sizeof(float), cudaMemcpyDefault, s->stream), "H2D patterns");
  } else {
    const double* src = static_cast<const double*>(host);
    const size_t chunk = size_t(1) << 22;
    float* stage = nullptr;
    check_cuda(cudaMallocHost(&stage, chunk * sizeof(float)), "pinned staging");
    try {
      for (size_t off = 0; off < n; off += chunk) {
        const size_t m = std::min(chunk, n - off);
        check_cuda(cudaStreamSynchronize(s->stream), "staging sync");
        for (size_t i = 0; i < m; ++i) stage[i] = float(src[off + i]);
        check_cuda(cudaMemcpyAsync(s->amp.as<float>() + off, stage, m * sizeof(float), cudaMemcpyHostToDevice,
                                   s->stream),
                   "H2D patterns");
      }
      check_cuda(cudaStreamSynchronize(s->stream), "staging sync");
    } catch (...) {
      cudaFreeHost(stage);
      throw;
    }
    cudaFreeHost(stage);
  }
}

// Reference CSV cell: `re` then '+' when im >= 0, `im`, 'j' (src/Cuda2DArray.cpp:46-52); ", " between cells.
void write_complex_file(const std::string& path, const float* c64, size_t rows, size_t cols, bool binary) {
  std::ofstream f(path, binary ? std::ios::out | std::ios::binary : std::ios::out);
  if (!f.is_open()) fail(PTY_ERR_IO, "cannot open " + path + " for writing");
  if (binary) {
    f.write(reinterpret_cast<const char*>(c64), std::streamsize(rows * cols * 2 * sizeof(float)));
  } else {
    for (size_t x = 0; x < rows; ++x) {
      for (size_t y = 0; y < cols; ++y) {
        const float re = c64[2 * (x * cols + y)], im = c64[2 * (x * cols + y) + 1];
        f << re;
        if (im >= 0) f << "+";
        f << im << "j";
        if (y + 1 < cols) f << ", ";
      }
      f << std::endl;
    }
  }
  if (!f.good()) fail(PTY_ERR_IO, "write failed: " + path);
}

// IPhaser::writeResultsToDisk (src/IPhaser.cpp:417-428): <dir>/<jobID>_probes_<r>.<csv|bin> and _object_.
void write_results(pty_session* s, const std::string& dir, int r, bool binary) {
  set_device(s);
  std::vector<float> pr(2 * size_t(s->K) * s->N * s->N), ob(2 * size_t(s->X) * s->Y);
  check_cuda(cudaMemcpyAsync(pr.data(), s->probe.p, pr.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream),
             "D2H");
  check_cuda(cudaMemcpyAsync(ob.data(), s->obj.p, ob.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream),
             "D2H");
  check_cuda(cudaStreamSynchronize(s->stream), "D2H results");
  const std::string ext = binary ? "bin" : "csv";
  const std::string base = dir + "/" + s->prm.jobID;
  write_complex_file(base + "_probes_" + std::to_string(r) + "." + ext, pr.data(), size_t(s->K) * s->N, s->N, binary);
  write_complex_file(base + "_object_" + std::to_string(r) + "." + ext, ob.data(), s->X, s->Y, binary);
}

// Reads a complex CSV in the reference's format (probeGuess / objectGuess files).
std::vector<float> read_complex_csv(const std::string& path, size_t& rows, size_t& cols) {
  std::ifstream f(path);
  if (!f.is_open()) fail(PTY_ERR_IO, "cannot open " + path);
  std::vector<float> out;
  std::string line;
  rows = 0;
  cols = 0;
  while (std::getline(f, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    size_t n = 0;
    std::stringstream ls(line);
    std::string cell;
    while (std::getline(ls, cell, ',')) {
      std::string c;
      for (char ch : cell)
        if (ch != ' ' && ch != '(' && ch != ')' && ch != '\r') c += ch;
      if (!c.empty() && (c.back() == 'j' || c.back() == 'i')) c.pop_back();
      // split at the sign that starts the imaginary part (not an exponent sign, not the leading sign)
      size_t cut = std::string::npos;
      for (size_t k = c.size(); k-- > 1;)
        if ((c[k] == '+' || c[k] == '-') && c[k - 1] != 'e' && c[k - 1] != 'E') {
          cut = k;
          break;
        }
      float re = 0, im = 0;
      if (cut == std::string::npos) {
        re = std::stof(c);
      } else {
        re = std::stof(c.substr(0, cut));
        im = std::stof(c.substr(cut));
      }
      out.push_back(re);
      out.push_back(im);
      ++n;
    }
    if (cols == 0) cols = n;
    if (n != cols) fail(PTY_ERR_INVALID, "ragged CSV rows in " + path);
    ++rows;
  }
  return out;
}

// The ePIE modulus step's saturation level (Parameters::updatePixelSaturation, src/Parameters.cpp:54-62):
// 2^bitDepth - 1 - threshold, square-rooted with sqrtData, truncated to an integer at each step as the reference's
// unsigned pixelSaturation holds it (a threshold above the range gives 0: every pixel floats).  +inf, so that no
// pixel floats, unless bitDepth, threshold or sqrtData set it.
float saturation_level(const pty_params& p) {
  if (p.bitDepth <= 0 && p.threshold <= 0 && !p.sqrtData) return std::numeric_limits<float>::infinity();
  const int bits = p.bitDepth > 0 ? p.bitDepth : 32;
  double v = std::floor(std::ldexp(1.0, bits) - 1.0 - double(std::max(p.threshold, 0)));
  if (v < 0) v = 0;
  if (p.sqrtData) v = std::floor(std::sqrt(v));
  return float(v);
}

// ---------------------------------------------------------------------------- initialisation
void init_geometry(pty_session* s) {
  const pty_params& p = s->prm;
  const double dx_s = sample_pixel_size(p.lambd, p.z, p.dx_d, s->N);
  // mesh choice of IPhaser::initScanMesh (src/IPhaser.cpp:128-152): positionNP, else a list file, else a spiral,
  // else the Cartesian raster
  need(p.jitterRadius >= 0, "jitterRadius must be >= 0");
  const unsigned jit = unsigned(p.jitterRadius);
  const float dfx = float(p.driftx), dfy = float(p.drifty);  // the reference's float2 drift
  const int Ptot = s->shard_total > 0 ? s->shard_total : s->P;  // the whole scan's positions
  if (!s->pos_m.empty()) {
    s->geo = list_geometry(s->pos_m, dx_s, s->N, p.flipScanAxis != 0, jit, p.seed, dfx, dfy);
  } else if (p.lf[0]) {
    s->geo = list_geometry(read_position_file(p.lf, Ptot), dx_s, s->N, p.flipScanAxis != 0, jit, p.seed, dfx, dfy);
  } else if (p.spiralScan) {
    s->geo = spiral_geometry(Ptot, p.stepx, p.stepy, dx_s, s->N, p.flipScanAxis != 0, jit, p.seed, dfx, dfy);
  } else {
    s->geo = cartesian_geometry(p.scanDimsx, p.scanDimsy, p.stepx, p.stepy, dx_s, s->N, p.mirror1stScanAxis != 0,
                                p.mirror2ndScanAxis != 0, p.flipScanAxis != 0, jit, p.seed, dfx, dfy);
  }
  if (s->shard_total > 0)  // keep this shard's positions; the object size stays the whole scan's
    s->geo.pos = std::vector<float>(s->geo.pos.begin() + 2 * size_t(s->shard_first),
                                    s->geo.pos.begin() + 2 * size_t(s->shard_first + s->P));
  s->X = s->geo.X;
  s->Y = s->geo.Y;
  s->offs.resize(2 * size_t(s->P));
  for (int i = 0; i < s->P; ++i) {
    const float qx = s->geo.pos[2 * i], qy = s->geo.pos[2 * i + 1];
    // src/ePIE.cpp:100-105 stops the process on a negative position; here it is an error status.
    need(qx >= 0 && qy >= 0, "scan position " + std::to_string(i) + " is negative: object array too small");
    const int ox = int(std::round(qx)), oy = int(std::round(qy));
    need(ox + s->N <= s->X && oy + s->N <= s->Y,
         "scan position " + std::to_string(i) + " places the probe window outside the object");
    s->offs[2 * i] = ox;
    s->offs[2 * i + 1] = oy;
  }
}

void init_probe(pty_session* s, const float* avg_dev) {
  const size_t NN = size_t(s->N) * s->N;
  s->probe.alloc(sizeof(float2) * NN * s->K, "probe");
  s->pcache.alloc(sizeof(float) * NN * s->K, "probe cache");
  check_cuda(cudaMemsetAsync(s->probe.p, 0, s->probe.bytes, s->stream), "memset probe");
  check_cuda(cudaMemsetAsync(s->pcache.p, 0, s->pcache.bytes, s->stream), "memset probe cache");
  DeviceBuf d;
  d.alloc(4 * sizeof(double), "scalars");
  float pmax = 1.0f;
  if (s->prm.probeGuess[0]) {
    size_t r = 0, c = 0;
    std::vector<float> h = read_complex_csv(s->prm.probeGuess, r, c);
    need(r == size_t(s->N) && c == size_t(s->N), "probeGuess file is not N x N");
    check_cuda(cudaMemcpyAsync(s->probe.p, h.data(), sizeof(float2) * NN, cudaMemcpyHostToDevice, s->stream),
               "H2D probe");
    check_cuda(cudaStreamSynchronize(s->stream), "sync");
    // Probe::init file branch ends in updateIntensities() (src/Probe.cpp:344-353)
    check_cuda(abs2(s->probe.as<float2>(), s->pcache.as<float>(), NN * s->K, s->stream), "abs2");
    check_cuda(probe_modal_max(s->pcache.as<float>(), s->K, NN, 0, d.as<float>(), s->stream), "modal max");
    check_cuda(cudaMemcpyAsync(&pmax, d.p, sizeof(float), cudaMemcpyDeviceToHost, s->stream), "D2H");
  } else if (!s->probe_h.empty()) {
    check_cuda(cudaMemcpyAsync(s->probe.p, s->probe_h.data(), sizeof(float2) * NN * s->probe_given_modes,
                               cudaMemcpyHostToDevice, s->stream),
               "H2D probe");
    s->modesInitialized = s->probe_given_modes > 1;
    pmax = 1.0f;  // Probe::m_maxIntensity keeps its constructor value; the intensity cache stays zero
  } else {
    // Probe guess (src/Probe.cpp:360-372): sinc*Gaussian, projected onto the mean amplitude, max|P| = 1.
    const int N = s->N;
    check_cuda(probe_start(s->probe.as<float2>(), N, float(double(N) / (2 * 2.35)),
                           float(sample_pixel_size(s->prm.lambd, s->prm.z, s->prm.dx_d, N) / s->prm.beamSize),
                           s->stream),
               "probe start");
    DeviceBuf work;
    work.alloc(sizeof(float2) * NN, "fft work");
    check_cuda(fft2(s->probe.as<float2>(), work.as<float2>(), s->tw.as<float2>(), 1, N, false, s->stream), "fft2");
    check_cuda(modulus_project(s->probe.as<float2>(), avg_dev, int(NN), float(1.0 / double(NN)), s->stream),
               "modulus");
    check_cuda(fft2(s->probe.as<float2>(), work.as<float2>(), s->tw.as<float2>(), 1, N, true, s->stream), "ifft2");
    check_cuda(reduce_abs_max(s->probe.as<float2>(), NN * s->K, d.as<double>(), s->stream), "max");
    check_cuda(scale_by_inverse(s->probe.as<float2>(), NN * s->K, d.as<double>(), s->stream), "normalize");
    check_cuda(abs2(s->probe.as<float2>(), s->pcache.as<float>(), NN * s->K, s->stream), "abs2");
    check_cuda(probe_modal_max(s->pcache.as<float>(), s->K, NN, 0, d.as<float>() + 2, s->stream), "modal max");
    check_cuda(cudaMemcpyAsync(&pmax, d.as<float>() + 2, sizeof(float), cudaMemcpyDeviceToHost, s->stream), "D2H");
  }
  check_cuda(cudaStreamSynchronize(s->stream), "probe init");
  s->probeMax0 = pmax;
}

void init_object(pty_session* s) {
  const size_t XY = size_t(s->X) * s->Y;
  s->obj.alloc(sizeof(float2) * XY, "object");
  check_cuda(cudaMemsetAsync(s->obj.p, 0, s->obj.bytes, s->stream), "memset object");
  if (s->prm.objectGuess[0]) {
    // Sample::loadGuess centres the guess in the object (h_setObjectArray, src/SampleKernels.cu:620-636)
    size_t r = 0, c = 0;
    std::vector<float> h = read_complex_csv(s->prm.objectGuess, r, c);
    need(r <= size_t(s->X) && c <= size_t(s->Y), "objectGuess is larger than the object array");
    const size_t offx = s->X / 2 - r / 2, offy = s->Y / 2 - c / 2;
    check_cuda(cudaMemcpy2DAsync(s->obj.as<float2>() + offx * s->Y + offy, sizeof(float2) * s->Y, h.data(),
                                 sizeof(float2) * c, sizeof(float2) * c, r, cudaMemcpyHostToDevice, s->stream),
               "H2D object guess");
    check_cuda(cudaStreamSynchronize(s->stream), "sync");
  } else if (!s->obj_h.empty()) {
    check_cuda(cudaMemcpyAsync(s->obj.p, s->obj_h.data(), sizeof(float2) * XY, cudaMemcpyHostToDevice, s->stream),
               "H2D object");
  }
  s->objMax0 = 0;  // Sample::clearObjectArray (src/Sample.cpp:216-220); loadarr does not touch it
}

// The ePIE kernel of a session: the per-position chain (precision = 1, chosen, or automatic where it measured
// fastest: with several probe modes at 256^2 3.1x the fused cluster kernel, 76.8 vs 237 ms per iteration; at 512^2
// with one mode 1.15x the whole-GPU kernel, 39.8 vs 45.7 ms), else the shared-memory kernel where it applies and is
// not overridden, else the cluster or whole-GPU kernel.
bool epie_uses_chain(const pty_session* s) {
  const int var = s->epie_variant;
  return s->prm.precision != 0 || var == 3 || (var < 0 && ((s->K > 1 && s->N >= 256) || s->N >= 512));
}
bool epie_uses_sm_kernel(const pty_session* s) {
  return !epie_uses_chain(s) && epie_uses_smem(s->N, s->K) && (s->epie_variant < 0 || s->epie_variant == 0);
}

void init_epie(pty_session* s) {
  auto* ep = new EpieState;
  s->ep = ep;
  const size_t NN = size_t(s->N) * s->N, XY = size_t(s->X) * s->Y;
  const int var = s->epie_variant;
  ep->chain_tc = s->prm.precision != 0;
  ep->chain = epie_uses_chain(s);
  ep->sm = epie_uses_sm_kernel(s);
  if (ep->chain) {
    if (ep->chain_tc) {
      need(s->N == 256, "precision=1 (tensor-core FFT stages) needs 256 x 256 patterns", PTY_ERR_UNSUPPORTED);
      check_cuda(fft2_tc_prepare(), "tensor-core FFT set-up");
    }
    ep->cpsi.alloc(sizeof(float2) * NN * s->K, "exit waves");
    ep->cwork.alloc(sizeof(float2) * NN * s->K, "FFT work");
    ep->pmax2.alloc(2 * sizeof(float), "probe maxima");
    ep->tcerr.alloc(sizeof(int), "tensor-core flag");
  } else if (ep->sm) {
    check_cuda(epie_sm_prepare(s->N), "ePIE kernel set-up");
  } else {
    const int Cg = (var < 0 || var == 2) ? epie_grid_prepare(s->N, var == 2) : 0;
    if (Cg > 0) {
      ep->grid = true;
      ep->C = Cg;
    } else {
      check_cuda(epie_prepare(s->N, &ep->C), "ePIE kernel set-up (cluster size)");
    }
  }
  // grid-barrier count and generation, then the timeout flag
  ep->gsync.alloc(4 * sizeof(unsigned), "grid barrier");
  check_cuda(cudaMemsetAsync(ep->gsync.p, 0, ep->gsync.bytes, s->stream), "memset barrier");
  ep->pos.alloc(sizeof(float2) * s->P, "positions");
  check_cuda(cudaMemcpyAsync(ep->pos.p, s->geo.pos.data(), sizeof(float2) * s->P, cudaMemcpyHostToDevice, s->stream),
             "H2D positions");
  ep->order.alloc(sizeof(int) * s->P, "order");
  check_cuda(cudaMallocHost(&ep->order_h, sizeof(int) * s->P), "pinned order");
  ep->W1.alloc(sizeof(float2) * NN * s->K, "W1");
  ep->W2.alloc(sizeof(float2) * NN * s->K, "W2");
  ep->TX = (s->X + 15) / 16;
  ep->TY = (s->Y + 15) / 16;
  ep->TM.alloc(sizeof(float) * ep->TX * ep->TY, "tile maxima");
  ep->pm.alloc(sizeof(float) * 512, "partial maxima");  // one per CTA, two sets (position parity)
  ep->sc.alloc(sizeof(EpieScalars), "scalars");
  ep->ip.alloc(4 * sizeof(double), "inner products");
  s->ocache.alloc(sizeof(float) * XY, "object cache");
  check_cuda(cudaMemsetAsync(s->ocache.p, 0, s->ocache.bytes, s->stream), "memset cache");
  EpieScalars sc{float(s->objMax0), float(s->probeMax0), 0.0};
  check_cuda(cudaMemcpyAsync(ep->sc.p, &sc, sizeof(sc), cudaMemcpyHostToDevice, s->stream), "H2D scalars");
  ep->sq.alloc(sizeof(double) * s->P, "pattern sums");
  std::vector<double> ones(s->P, 1.0);
  if (s->prm.calculateRMS) {
    check_cuda(plane_sums(s->amp.as<float>(), s->P, NN, ep->sq.as<double>(), s->stream), "pattern sums");
  } else {
    check_cuda(cudaMemcpyAsync(ep->sq.p, ones.data(), sizeof(double) * s->P, cudaMemcpyHostToDevice, s->stream),
               "H2D sums");
  }
  check_cuda(cudaStreamSynchronize(s->stream), "ePIE init");
}

void init_dm(pty_session* s) {
  const size_t NN = size_t(s->N) * s->N, XY = size_t(s->X) * s->Y;
  s->psi.alloc(sizeof(float2) * NN * s->P, "DM exit waves");
  check_cuda(cudaMemsetAsync(s->psi.p, 0, s->psi.bytes, s->stream), "memset psi");
  s->dO.alloc(sizeof(float2) * XY, "dO");
  check_cuda(cudaMemsetAsync(s->dO.p, 0, s->dO.bytes, s->stream), "memset dO");
  s->dP.alloc(sizeof(float2) * NN, "dP");
  check_cuda(cudaMemsetAsync(s->dP.p, 0, s->dP.bytes, s->stream), "memset dP");
  // wave: patterns per pipeline pass (W1 + W2 = 2 * wave * 8N^2 bytes)
  check_cuda(dm_prepare(s->N), "DM kernel set-up");
  if (s->prm.precision) s->dm_err.alloc(sizeof(int), "DM wait flag");
  int wave = s->prm.wave;
  if (wave <= 0) wave = dm_wave_size(s->N, s->P);
  wave = std::min(wave, s->P);
  s->wave = wave;
  s->nwaves = (s->P + wave - 1) / wave;
  // two lanes: consecutive waves alternate between the session's stream and a second one, so that one wave's
  // kernels fill the other's tails and launch gaps (900 x 512^2: 2.78-2.88 ms per iteration with 2 lanes of 113-pattern
  // waves against 2.99-3.01 ms with one lane of 225-pattern waves; 3 or 4 lanes measured the same as 2)
  s->dm_lanes = (s->nwaves >= 2 && s->dm_lanes_req != 1) ? 2 : 1;
  if (s->dm_lanes == 2) {
    create_session_stream(s, &s->dm_side);
    check_cuda(cudaEventCreateWithFlags(&s->dm_fork, cudaEventDisableTiming), "event");
    check_cuda(cudaEventCreateWithFlags(&s->dm_join, cudaEventDisableTiming), "event");
  }
  s->W1.alloc(sizeof(float2) * NN * wave * s->dm_lanes, "W1");
  s->W2.alloc(sizeof(float2) * NN * wave * s->dm_lanes, "W2");
  std::vector<int> slots(s->P);
  for (int i = 0; i < s->P; ++i) slots[i] = i;
  s->slots.alloc(sizeof(int) * s->P, "slots");
  check_cuda(cudaMemcpyAsync(s->slots.p, slots.data(), sizeof(int) * s->P, cudaMemcpyHostToDevice, s->stream),
             "H2D slots");
  s->scal.alloc(8 * sizeof(double), "DM scalars");
  const double h[8] = {0, 0, 1.0 / s->objMax0, 1.0 / s->probeMax0, s->objMax0, s->probeMax0, 0, 0};
  check_cuda(cudaMemcpyAsync(s->scal.p, h, sizeof(h), cudaMemcpyHostToDevice, s->stream), "H2D DM scalars");
  check_cuda(cudaStreamSynchronize(s->stream), "DM init");
}

// MLs set-up: ML-mesh geometry, sqrt of the intensities, probe (given or the guess), flat or given object, and the
// initEvo normalisations (src/Probe.cpp:507-613): object scaled by sqrt(sum |O|^2 illum / sum illum), probe by
// 1/corr with corr = sqrt(median_i(mean|P|^2 / (sum I_i / N^2)) * N^2), p_object = illum / corr^2, MAX_ILLUM.
void init_mls(pty_session* s) {
  const pty_params& p = s->prm;
  need(s->K == 1 || p.mlsCore == 0, "the MLs core (mlsCore=1) supports one probe mode (probeModes=1)",
       PTY_ERR_UNSUPPORTED);
  need(s->K <= 64, "MLs supports up to 64 probe modes", PTY_ERR_UNSUPPORTED);
  need(p.precision == 0 || s->N == 256, "precision=1 (tensor-core FFT stages) needs 256 x 256 patterns",
       PTY_ERR_UNSUPPORTED);
  auto* ml = new MlsState;
  s->ml = ml;
  if (p.precision) {
    check_cuda(fft2_tc_prepare(), "tensor-core FFT set-up");
    ml->tcerr.alloc(sizeof(int), "tensor-core flag");
    check_cuda(cudaMemsetAsync(ml->tcerr.p, 0, sizeof(int), s->stream), "memset flag");
  }
  const int N = s->N, P = s->P;
  const size_t NN = size_t(N) * N;
  const double dx_s = sample_pixel_size(p.lambd, p.z, p.dx_d, N);
  std::vector<float> raw;
  if (!s->pos_m.empty() || p.lf[0]) {
    const std::vector<double> xy = s->pos_m.empty() ? read_position_file(p.lf, P) : s->pos_m;
    const float inv = float(1.0 / dx_s), dfx = float(p.driftx), dfy = float(p.drifty);
    raw.resize(2 * size_t(P));
    for (int i = 0; i < P; ++i) {
      raw[2 * i] = add_drift(float(xy[2 * i]), i / 1024, dfx) * inv;
      raw[2 * i + 1] = add_drift(float(xy[2 * i + 1]), i % 1024, dfy) * inv;
    }
  } else {
    // the reference's spiral mesh has no ML variant (SpiralScanMesh::generateMeshML is empty); jitter is not part
    // of this engine's ML mesh
    need(p.spiralScan == 0 && p.jitterRadius == 0, "MLs supports Cartesian or listed positions without jitter",
         PTY_ERR_UNSUPPORTED);
    raw = raw_cartesian_positions(p.scanDimsx, p.scanDimsy, p.stepx, p.stepy, dx_s, p.mirror1stScanAxis != 0,
                                  p.mirror2ndScanAxis != 0, float(p.driftx), float(p.drifty));
  }
  ml->geo = mls_geometry(raw, N);
  const int gX = s->X, gY = s->Y;
  s->X = ml->geo.X;
  s->Y = ml->geo.Y;
  if (!s->obj_h.empty()) need(gX == s->X && gY == s->Y, "objectNP shape differs from the MLs object size");
  std::vector<int2> st(P);
  for (int i = 0; i < P; ++i) {
    need(ml->geo.r0[i] >= 0 && ml->geo.c0[i] >= 0 && ml->geo.r0[i] + N <= s->X && ml->geo.c0[i] + N <= s->Y,
         "MLs window " + std::to_string(i) + " lies outside the object");
    st[i] = make_int2(ml->geo.r0[i], ml->geo.c0[i]);
  }
  s->geo.pos.assign(raw.begin(), raw.end());
  ml->variable = p.mlsCore == 0;
  // remove_extra_degree re-centres the extra-mode weights of the first min(2, P) positions; with one position that
  // zeroes its only weight and update_variable_probe then divides by zero
  need(!ml->variable || P >= 2, "the MLs default path needs at least 2 positions (mlsCore=1 runs one)",
       PTY_ERR_UNSUPPORTED);
  ml->starts.alloc(sizeof(int2) * P, "MLs starts");
  check_cuda(cudaMemcpyAsync(ml->starts.p, st.data(), sizeof(int2) * P, cudaMemcpyHostToDevice, s->stream), "H2D");
  // intensity sums (Diffractions::fillSquaredSums) then amplitudes = sqrt(I) (Diffractions::squaredRoot)
  DeviceBuf sq;
  sq.alloc(sizeof(double) * P, "sums");
  check_cuda(plane_sums(s->amp.as<float>(), P, NN, sq.as<double>(), s->stream), "intensity sums");
  std::vector<double> isum(P);
  check_cuda(cudaMemcpyAsync(isum.data(), sq.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s->stream), "D2H");
  check_cuda(sqrt_inplace(s->amp.as<float>(), size_t(P) * NN, s->stream), "sqrt");
  if (p.probeGuess[0] == 0 && s->probe_h.empty()) {
    // no probe given: the zone-plate guess of initMLH (src/IPhaser.cpp:283-291, src/Probe.cpp:376-420)
    s->probe.alloc(sizeof(float2) * NN * s->K, "probe");
    s->pcache.alloc(sizeof(float) * NN * s->K, "probe cache");
    check_cuda(cudaMemsetAsync(s->probe.p, 0, s->probe.bytes, s->stream), "memset probe");
    check_cuda(cudaMemsetAsync(s->pcache.p, 0, s->pcache.bytes, s->stream), "memset probe cache");
    DeviceBuf pf, work;
    pf.alloc(sizeof(float2) * NN, "zone-plate propagator");
    work.alloc(sizeof(float2) * NN, "fft work");
    check_cuda(mls_zone_plate_probe(s->probe.as<float2>(), pf.as<float2>(), work.as<float2>(), s->tw.as<float2>(), N,
                                    p.lambd, dx_s, p.beamSize, s->stream),
               "zone-plate probe");
    check_cuda(cudaStreamSynchronize(s->stream), "zone-plate probe");
  } else {
    init_probe(s, nullptr);
  }
  const size_t XY = size_t(s->X) * s->Y;
  s->obj.alloc(sizeof(float2) * XY, "object");
  if (!s->obj_h.empty())
    check_cuda(cudaMemcpyAsync(s->obj.p, s->obj_h.data(), sizeof(float2) * XY, cudaMemcpyHostToDevice, s->stream),
               "H2D object");
  else
    check_cuda(fill_complex(s->obj.as<float2>(), XY, make_float2(1.f, 0.f), s->stream), "flat object");
  std::vector<float2> Eh;
  if (ml->variable) {
    // initEvo (src/Probe.cpp:511-560): intensity weights 1; the extra mode to unit RMS, its weights carry the norm
    std::vector<double> evo(2 * size_t(P), 1.0), evo1, tilts;
    mls_variable_draws(p.seed, N, P, s->K, Eh, tilts, evo1);
    if (s->K > 1) {
      // modes 1..K-1 from mode 0 (initMLH, src/Probe.cpp:422-490): phase tilts, then recombination by the
      // eigenvectors of their Gram matrix
      const int K = s->K;
      DeviceBuf dt, dg, tmp;
      dt.alloc(sizeof(double) * tilts.size(), "mode tilts");
      dg.alloc(sizeof(double2) * K * K, "mode Gram matrix");
      tmp.alloc(sizeof(float2) * NN * K, "modes");
      check_cuda(cudaMemcpyAsync(dt.p, tilts.data(), dt.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
      check_cuda(mls_mode_tilts(s->probe.as<float2>(), K, N, dt.as<double>(), s->stream), "mode tilts");
      check_cuda(mls_mode_gram(s->probe.as<float2>(), K, N, dg.as<double2>(), s->stream), "mode Gram matrix");
      std::vector<double2> gram(size_t(K) * K), V;
      check_cuda(cudaMemcpyAsync(gram.data(), dg.p, dg.bytes, cudaMemcpyDeviceToHost, s->stream), "D2H");
      check_cuda(cudaStreamSynchronize(s->stream), "mode Gram matrix");
      hermitian_eigen(K, gram, V);
      check_cuda(cudaMemcpyAsync(dg.p, V.data(), dg.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
      check_cuda(mls_mode_combine(s->probe.as<float2>(), tmp.as<float2>(), K, N, dg.as<double2>(), s->stream),
                 "mode recombination");
      check_cuda(cudaStreamSynchronize(s->stream), "probe modes");
    }
    double se = 0;
    for (const float2& v : Eh) se += double(v.x) * v.x + double(v.y) * v.y;
    const double rE = std::sqrt(se / double(NN));
    for (float2& v : Eh) v = make_float2(float(v.x * (1.0 / rE)), float(v.y * (1.0 / rE)));
    for (int i = 0; i < P; ++i) evo[P + i] = evo1[i] * rE;
    ml->E.alloc(sizeof(float2) * NN, "extra probe mode");
    ml->evo.alloc(sizeof(double) * 2 * P, "probe evolution");
    ml->pos.alloc(sizeof(float) * 2 * P, "MLs positions");
    ml->pos_o.alloc(sizeof(float) * 2 * P, "MLs original positions");
    ml->sub.alloc(sizeof(float2) * P, "sub-pixel shifts");
    check_cuda(cudaMemcpyAsync(ml->E.p, Eh.data(), ml->E.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
    check_cuda(cudaMemcpyAsync(ml->evo.p, evo.data(), ml->evo.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
    check_cuda(cudaMemcpyAsync(ml->pos.p, raw.data(), ml->pos.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
    check_cuda(cudaMemcpyAsync(ml->pos_o.p, raw.data(), ml->pos_o.bytes, cudaMemcpyHostToDevice, s->stream), "H2D");
    check_cuda(cudaMemsetAsync(ml->sub.p, 0, ml->sub.bytes, s->stream), "memset");
    check_cuda(cudaStreamSynchronize(s->stream), "MLs set-up");  // Eh, evo and raw are host temporaries
  }
  ml->pobj.alloc(sizeof(float) * XY, "illumination");
  ml->norms.alloc(2 * sizeof(double), "norm sums");
  ml->maxill.alloc(sizeof(float), "max illumination");
  check_cuda(cudaMemsetAsync(ml->pobj.p, 0, ml->pobj.bytes, s->stream), "memset");
  check_cuda(mls_illum_add(ml->pobj.as<float>(), s->probe.as<float2>(), ml->starts.as<int2>(), P, N, s->Y, 1.f,
                           s->stream),
             "illumination");
  check_cuda(mls_norm_sums(ml->pobj.as<float>(), s->obj.as<float2>(), s->Y, 0, 0, s->X, s->Y, 0, ml->norms.as<double>(),
                           s->stream),
             "object norm");
  check_cuda(scale_by_norm(s->obj.as<float2>(), XY, ml->norms.as<double>(), 1, s->stream), "object norm");
  DeviceBuf d;
  d.alloc(sizeof(double), "sum");
  check_cuda(reduce_sum_sq(s->probe.as<float2>(), NN * s->K, d.as<double>(), s->stream), "probe power");
  double psum = 0;
  check_cuda(cudaMemcpyAsync(&psum, d.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "D2H");
  check_cuda(cudaStreamSynchronize(s->stream), "MLs set-up");
  const double meanillum = psum / double(NN);
  std::vector<double> corrv(P);
  for (int i = 0; i < P; ++i) corrv[i] = meanillum / (isum[i] / double(NN));
  std::sort(corrv.begin(), corrv.end());
  double corr = (P % 2) ? corrv[P / 2] : 0.5 * (corrv[P / 2 - 1] + corrv[P / 2]);
  corr = std::sqrt(corr * double(NN));
  check_cuda(scale_complex(s->probe.as<float2>(), NN * s->K, float(1.0 / corr), s->stream), "probe scale");
  if (ml->variable) check_cuda(scale_complex(ml->E.as<float2>(), NN, float(1.0 / corr), s->stream), "extra mode scale");
  check_cuda(scale_real(ml->pobj.as<float>(), XY, float(1.0 / (corr * corr)), s->stream), "illumination scale");
  check_cuda(max_real(ml->pobj.as<float>(), XY, ml->maxill.as<float>(), s->stream), "MAX_ILLUM");
  // group buffers
  ml->Gmax = std::max(1, P / 100);
  ml->ng = (P + ml->Gmax - 1) / ml->Gmax;
  const size_t GN = size_t(ml->Gmax) * NN;
  ml->S.alloc(sizeof(float2) * XY, "S");
  ml->pum.alloc(sizeof(float2) * NN, "probe direction");
  ml->objp.alloc(sizeof(float2) * GN, "windows");
  ml->psi.alloc(sizeof(float2) * GN, "exit waves");
  ml->work.alloc(sizeof(float2) * GN * (ml->variable ? std::max(2, s->K - 1) : 1), "FFT work");
  if (ml->variable) {
    ml->vp.alloc(sizeof(float2) * GN, "position probes");
    ml->pu.alloc(sizeof(float2) * GN, "probe directions");
    ml->aux.alloc(sizeof(float2) * 2 * GN, "gradient images");
    ml->vs.alloc(sizeof(double) * mls_var_scratch_doubles(ml->Gmax), "MLs sums");
    ml->pmax.alloc(sizeof(float), "illumination maximum");
    ml->vupd.alloc(sizeof(float2) * NN, "extra-mode update");
    ml->work2.alloc(sizeof(float2) * 2 * GN, "position-search FFT work");
    create_session_stream(s, &ml->side);  // the position search's stream
    check_cuda(cudaEventCreateWithFlags(&ml->ev_fork, cudaEventDisableTiming), "event");
    check_cuda(cudaEventCreateWithFlags(&ml->ev_join, cudaEventDisableTiming), "event");
    if (mls_var_fused(s->N, s->K, s->prm.precision != 0))
      check_cuda(mls_var_prepare(s->N), "MLs cluster launch set-up");
    if (s->K > 1) {
      ml->psik.alloc(sizeof(float2) * GN * (s->K - 1), "exit waves of the other modes");
      ml->mtmp.alloc(sizeof(float2) * NN * s->K, "mode scratch");
    }
    for (DeviceBuf* b : {&ml->vp, &ml->pu, &ml->aux, &ml->vs})
      check_cuda(cudaMemsetAsync(b->p, 0, b->bytes, s->stream), "memset");
  }
  ml->table_ints = size_t(ml->ng) * ml->Gmax + 5 * size_t(ml->ng);
  for (MlsTables& t : ml->tab) {
    t.dev.alloc(sizeof(int) * ml->table_ints, "group tables");
    check_cuda(cudaMallocHost(&t.host, sizeof(int) * ml->table_ints), "pinned group tables");
    check_cuda(cudaEventCreateWithFlags(&t.copied, cudaEventDisableTiming), "event");
  }
  ml->sums.alloc(sizeof(double) * (6 * ml->Gmax + 1), "LSQ sums");  // + the LSQ launch's block counter
  ml->errk.alloc(sizeof(double) * ml->Gmax, "errors");
  ml->betas.alloc(sizeof(double) * 4, "steps");
  ml->err.alloc(sizeof(double), "error");
  for (DeviceBuf* b : {&ml->S, &ml->pum, &ml->sums, &ml->errk})
    check_cuda(cudaMemsetAsync(b->p, 0, b->bytes, s->stream), "memset");
  check_cuda(cudaStreamSynchronize(s->stream), "MLs set-up");
}

MlsBuffers mls_buffers(pty_session* s, int parity) {
  MlsState* ml = s->ml;
  MlsBuffers b{};
  b.obj = s->obj.as<float2>();
  b.probe = s->probe.as<float2>();
  b.amp = s->amp.as<float>();
  b.pobj = ml->pobj.as<float>();
  b.S = ml->S.as<float2>();
  b.pum = ml->pum.as<float2>();
  b.objp = ml->objp.as<float2>();
  b.psi = ml->psi.as<float2>();
  b.work = ml->work.as<float2>();
  b.starts = ml->starts.as<int2>();
  b.members = ml->tab[parity].dev.as<int>();
  b.gsize = b.members + size_t(ml->ng) * ml->Gmax;
  b.bbox = b.gsize + ml->ng;
  b.sums = ml->sums.as<double>();
  b.lsq_done = reinterpret_cast<unsigned*>(b.sums + 6 * ml->Gmax);
  b.errk = ml->errk.as<double>();
  b.betas = ml->betas.as<double>();
  b.err = ml->err.as<double>();
  b.normsums = ml->norms.as<double>();
  b.maxIllum = ml->maxill.as<float>();
  b.tw = s->tw.as<float2>();
  for (int i = 0; i < 4; ++i) b.roi[i] = ml->geo.roi[i];
  b.N = s->N;
  b.P = s->P;
  b.X = s->X;
  b.Y = s->Y;
  b.Gmax = ml->Gmax;
  b.delta_p = float(s->prm.delta_p);
  b.beta_obj = 1.0 * 0.9;    // beta_object * beta_LSQ (src/Parameters.h:158-165 defaults)
  b.beta_probe = 1.0 * 0.9;  // beta_probe * beta_LSQ
  b.tc = s->prm.precision ? 1 : 0;
  b.tc_err = ml->tcerr.as<int>();
  if (ml->variable) {
    b.E = ml->E.as<float2>();
    b.evo = ml->evo.as<double>();
    b.pos = ml->pos.as<float>();
    b.pos_o = ml->pos_o.as<float>();
    b.sub = ml->sub.as<float2>();
    b.win = ml->starts.as<int2>();
    b.boxw = const_cast<int*>(b.bbox);
    b.vp = ml->vp.as<float2>();
    b.pu = ml->pu.as<float2>();
    b.aux = ml->aux.as<float2>();
    b.vs = ml->vs.as<double>();
    b.pmax = ml->pmax.as<float>();
    b.cvx = std::ceil(float(s->X) * 1.0f / 2 - float(s->N) * 1.0f / 2);
    b.cvy = std::ceil(float(s->Y) * 1.0f / 2 - float(s->N) * 1.0f / 2);
    b.vupd = ml->vupd.as<float2>();
    b.work2 = ml->work2.as<float2>();
    b.side = ml->side;
    b.ev_fork = ml->ev_fork;
    b.ev_join = ml->ev_join;
    b.K = s->K;
    b.psik = ml->psik.as<float2>();
    b.mtmp = ml->mtmp.as<float2>();
  }
  return b;
}

// One MLs iteration: the iteration's random groups (a SplitMix64 permutation cut into groups of max(1, P/100), in a
// second shuffled order) are written to the device tables, then the iteration graph replays.
// shared_gpu: the step runs beside other scans' kernels (pty_batch_run), where the MLs groups use their separate
// transform passes (MLS_SEPARATE) rather than one launch of 16-CTA clusters, which waits for whole SM groups to free up
double step_mls(pty_session* s, bool want_err, bool shared_gpu = false) {
  MlsState* ml = s->ml;
  const int P = s->P, G = ml->Gmax, N = s->N;
  const int parity = int(ml->steps & 1);
  MlsTables& tb = ml->tab[parity];
  // this set's staging buffer was last copied two iterations ago
  check_cuda(cudaEventSynchronize(tb.copied), "group table reuse");
  std::vector<int> perm(P);
  for (int i = 0; i < P; ++i) perm[i] = i;
  for (int i = P - 1; i > 0; --i) std::swap(perm[i], perm[splitmix64(s->rng) % uint64_t(i + 1)]);
  std::vector<int> order(ml->ng);
  for (int i = 0; i < ml->ng; ++i) order[i] = i;
  for (int i = ml->ng - 1; i > 0; --i) std::swap(order[i], order[splitmix64(s->rng) % uint64_t(i + 1)]);
  int* mem = tb.host;
  int* gs = mem + size_t(ml->ng) * G;
  int* box = gs + ml->ng;
  std::fill(mem, mem + size_t(ml->ng) * G, -1);
  for (int gi = 0; gi < ml->ng; ++gi) {
    const int g = order[gi];
    const int lo = g * G, hi = std::min(P, (g + 1) * G);
    gs[gi] = hi - lo;
    int x0 = s->X, y0 = s->Y, x1 = 0, y1 = 0;
    for (int m = lo; m < hi; ++m) {
      const int j = perm[m];
      mem[size_t(gi) * G + (m - lo)] = j;
      x0 = std::min(x0, ml->geo.r0[j]);
      y0 = std::min(y0, ml->geo.c0[j]);
      x1 = std::max(x1, ml->geo.r0[j] + N);
      y1 = std::max(y1, ml->geo.c0[j] + N);
    }
    box[4 * gi] = x0;
    box[4 * gi + 1] = y0;
    box[4 * gi + 2] = x1 - x0;
    box[4 * gi + 3] = y1 - y0;
  }
  check_cuda(cudaMemcpyAsync(tb.dev.p, tb.host, sizeof(int) * ml->table_ints, cudaMemcpyHostToDevice, s->stream),
             "H2D groups");
  check_cuda(cudaEventRecord(tb.copied, s->stream), "event");
  check_cuda(cudaMemsetAsync(ml->err.p, 0, sizeof(double), s->stream), "memset");
  if (ml->variable) {
    // iteration regime (src/MLS.cpp:86-89,99-102,470-475): windows at iteration 1 and from PPS, remove_extra_degree
    // from 2, update_variable_probe from 3, position search from PPS
    const int64_t it = ml->steps + 1;
    const int pps = s->prm.PPS;
    unsigned flags = 0;
    if (it == 1 || it >= pps) flags |= MLS_WINDOWS;
    if (it > 1) flags |= MLS_REMOVE;
    if (it > 2) flags |= MLS_VARUPD;
    if (it >= pps) flags |= MLS_POSSEARCH;
    if (shared_gpu) flags |= MLS_SEPARATE;
    const unsigned key = unsigned(parity) | (flags << 1);
    cudaGraphExec_t& ge = ml->var_graphs[key];
    if (!ge) {
      const MlsBuffers b = mls_buffers(s, parity);
      cudaGraph_t graph = nullptr;
      check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
      const cudaError_t e = mls_iteration_var(b, ml->ng, flags, s->stream);
      const cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
      check_cuda(e, "MLs capture");
      check_cuda(e2, "end capture");
      const cudaError_t e3 = cudaGraphInstantiate(&ge, graph, 0);
      cudaGraphDestroy(graph);
      if (e3 != cudaSuccess) ml->var_graphs.erase(key);
      check_cuda(e3, "graph instantiate");
    }
    check_cuda(cudaGraphLaunch(ge, s->stream), "MLs graph launch");
    s->launches += mls_var_launches_per_iteration(ml->ng, flags, s->K, s->prm.precision != 0, s->N);
  } else {
  if (!tb.graph) {
    const MlsBuffers b = mls_buffers(s, parity);
    cudaGraph_t graph = nullptr;
    check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    const cudaError_t e = mls_iteration(b, ml->ng, s->stream);
    const cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
    check_cuda(e, "MLs capture");
    check_cuda(e2, "end capture");
    const cudaError_t e3 = cudaGraphInstantiate(&tb.graph, graph, 0);
    cudaGraphDestroy(graph);
    check_cuda(e3, "graph instantiate");
  }
  check_cuda(cudaGraphLaunch(tb.graph, s->stream), "MLs graph launch");
  s->launches += mls_launches_per_iteration(ml->ng);
  }
  ++ml->steps;
  if (s->prm.precision) {  // the tensor-core FFT reports a wait timeout through its device flag
    int flag = 0;
    check_cuda(cudaMemcpyAsync(&flag, ml->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "D2H flag");
    check_cuda(cudaStreamSynchronize(s->stream), "MLs iteration");
    need(flag == 0, "MLs: a tensor-core FFT wait timed out", PTY_ERR_CUDA);
  }
  if (!(want_err && s->prm.calculateRMS)) return 0.0;
  double e = 0;
  check_cuda(cudaMemcpyAsync(&e, ml->err.p, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "D2H error");
  check_cuda(cudaStreamSynchronize(s->stream), "MLs iteration");
  return e / P;
}

DMBuffers dm_buffers(pty_session* s) {
  DMBuffers b;
  b.psi = s->psi.as<float2>();
  b.amp = s->amp.as<float>();
  b.obj = s->obj.as<float2>();
  b.probe = s->probe.as<float2>();
  b.dO = s->dO.as<float2>();
  b.dP = s->dP.as<float2>();
  b.W1 = s->W1.as<float2>();
  b.W2 = s->W2.as<float2>();
  b.offs = s->dOffs.as<int2>();
  b.tw = s->tw.as<float2>();
  b.sums = s->scal.as<double>();
  b.fac = s->scal.as<double>() + 2;
  b.tc = s->prm.precision ? 1 : 0;
  b.err = s->prm.precision ? s->dm_err.as<int>() : nullptr;
  b.N = s->N;
  b.K = s->K;
  b.X = s->X;
  b.Y = s->Y;
  return b;
}

// The passes of one DM iteration over all waves (without finalize): three launches per wave.
cudaError_t dm_enqueue_waves(pty_session* s, const DMBuffers& b, bool pc, bool up) {
  cudaError_t err = cudaSuccess;
  const bool two = s->dm_lanes == 2;
  if (two) {  // fork: the second lane follows the iteration's earlier work
    err = cudaEventRecord(s->dm_fork, s->stream);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s->dm_side, s->dm_fork, 0);
  }
  const size_t lane_elems = size_t(s->N) * s->N * s->wave;
  for (int w = 0; w < s->nwaves && err == cudaSuccess; ++w) {
    DMWave wv;
    wv.slot_pat = s->slots.as<int>() + size_t(w) * s->wave;
    wv.count = std::min(s->wave, s->P - w * s->wave);
    const bool second = two && (w & 1);
    DMBuffers bl = b;
    if (second) {
      bl.W1 = b.W1 + lane_elems;
      bl.W2 = b.W2 + lane_elems;
    }
    err = dm_wave(bl, wv, pc, up, second ? s->dm_side : s->stream, nullptr);
  }
  if (two && err == cudaSuccess) {  // join
    err = cudaEventRecord(s->dm_join, s->dm_side);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(s->stream, s->dm_join, 0);
  }
  return err;
}

int64_t dm_wave_launches(const pty_session* s) { return 3 * int64_t(s->nwaves); }

// The tensor-core column pass (precision = 1) reports an expired wait through the session's device flag, read where
// the host synchronises anyway (end of pty_run, results, finish of a shard step).
void dm_check_flag(pty_session* s) {
  if (s->algo != ALGO_DM || !s->prm.precision || !s->dm_err.p) return;
  int flag = 0;
  check_cuda(cudaMemcpyAsync(&flag, s->dm_err.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "D2H flag");
  check_cuda(cudaStreamSynchronize(s->stream), "DM iteration");
  need(flag == 0, "DM: a tensor-core wait timed out (the iteration did not complete)", PTY_ERR_CUDA);
}

// One DM iteration: waves of (fwd_rows, cols, inv_rows) then finalize, replayed from a CUDA graph per flag state.
void step_dm(pty_session* s, int it) {
  const bool pc = it <= s->prm.phaseConstraint, up = it >= s->prm.updateProbe;
  const int gi = (pc ? 1 : 0) | (up ? 2 : 0);
  if (!s->graphs[gi]) {
    const DMBuffers b = dm_buffers(s);
    cudaGraph_t graph = nullptr;
    check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = dm_enqueue_waves(s, b, pc, up);
    if (err == cudaSuccess) err = dm_finalize(b, up, s->stream, nullptr);
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
    check_cuda(err, "DM capture");
    check_cuda(e2, "end capture");
    cudaGraphExec_t exec = nullptr;
    cudaError_t e3 = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    check_cuda(e3, "graph instantiate");
    s->graphs[gi] = exec;
  }
  check_cuda(cudaGraphLaunch(s->graphs[gi], s->stream), "DM graph launch");
  s->launches += dm_wave_launches(s) + 2;
}

// Sharded DM: the waves of iteration `it` (increments accumulate in dO / dP) and, separately, their application.
static cudaGraphExec_t capture_graph(pty_session* s, const std::function<cudaError_t()>& body) {
  cudaGraph_t graph = nullptr;
  check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
  const cudaError_t err = body();
  const cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
  check_cuda(err, "capture");
  check_cuda(e2, "end capture");
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e3 = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  check_cuda(e3, "graph instantiate");
  return exec;
}

void step_dm_local(pty_session* s, int it) {
  const bool pc = it <= s->prm.phaseConstraint, up = it >= s->prm.updateProbe;
  const int gi = (pc ? 1 : 0) | (up ? 2 : 0);
  if (!s->graphs_local[gi]) {
    const DMBuffers b = dm_buffers(s);
    s->graphs_local[gi] = capture_graph(s, [&]() { return dm_enqueue_waves(s, b, pc, up); });
  }
  check_cuda(cudaGraphLaunch(s->graphs_local[gi], s->stream), "DM graph launch");
  s->launches += dm_wave_launches(s);
}

void step_dm_finish(pty_session* s, int it) {
  const bool up = it >= s->prm.updateProbe;
  if (!s->graphs_fin[up ? 1 : 0]) {
    const DMBuffers b = dm_buffers(s);
    s->graphs_fin[up ? 1 : 0] = capture_graph(s, [&]() { return dm_finalize(b, up, s->stream, nullptr); });
  }
  check_cuda(cudaGraphLaunch(s->graphs_fin[up ? 1 : 0], s->stream), "DM graph launch");
  s->launches += 2;
}

// One ePIE iteration: the modal switch on the host side (beginModalReconstruction), then the persistent kernel.
double step_epie(pty_session* s, int it, bool want_err) {
  EpieState* ep = s->ep;
  const bool pc = it <= s->prm.phaseConstraint, up = it >= s->prm.updateProbe, um = it >= s->prm.updateModes;
  const size_t NN = size_t(s->N) * s->N;
  DeviceBuf tmp;
  if (um) {
    s->useAll = true;
    if (!s->modesInitialized) {  // initProbeModes (src/Probe.cpp:320-330)
      if (s->K > 1) {
        if (!ep->modesCopy.p) ep->modesCopy.alloc(sizeof(float2) * NN * s->K, "modes copy");
        check_cuda(epie_init_modes(s->probe.as<float2>(), s->pcache.as<float>(), s->K, s->N,
                                   ep->modesCopy.as<float2>(), ep->ip.as<double>(), s->stream),
                   "mode init");
        s->modesInitialized = true;
        s->launches += 1 + 2 * (s->K * (s->K - 1) / 2);
      }
      // updateMaxIntensity(): probeMax = modal max of the cache
      check_cuda(probe_modal_max(s->pcache.as<float>(), s->K, NN, 1, &reinterpret_cast<EpieScalars*>(ep->sc.p)->probeMax,
                                 s->stream),
                 "modal max");
      s->launches += 1;
    }
  }
  const int Ka = s->useAll ? s->K : 1;
  std::vector<int> order;
  visiting_order(s->rng, s->P, order);
  check_cuda(cudaStreamSynchronize(s->stream), "order buffer reuse");
  std::memcpy(ep->order_h, order.data(), sizeof(int) * s->P);
  check_cuda(cudaMemcpyAsync(ep->order.p, ep->order_h, sizeof(int) * s->P, cudaMemcpyHostToDevice, s->stream),
             "H2D order");
  if (up && !ep->tm_valid) {
    check_cuda(tile_max_all(s->ocache.as<float>(), s->X, s->Y, ep->TM.as<float>(), ep->TX, ep->TY, s->stream),
               "tile maxima");
    s->launches += 1;
  }
  ep->tm_valid = up;
  check_cuda(cudaMemsetAsync(&reinterpret_cast<EpieScalars*>(ep->sc.p)->err, 0, sizeof(double), s->stream), "memset");
  EpieArgs g;
  g.ampT = s->amp.as<float>();
  g.amp = s->amp.as<float>();
  g.obj = s->obj.as<float2>();
  g.ocache = s->ocache.as<float>();
  g.probe = s->probe.as<float2>();
  g.pcache = s->pcache.as<float>();
  g.pos = ep->pos.as<float2>();
  g.order = ep->order.as<int>();
  g.W1 = ep->W1.as<float2>();
  g.W2 = ep->W2.as<float2>();
  g.TM = ep->TM.as<float>();
  g.pm = ep->pm.as<float>();
  g.sc = ep->sc.as<EpieScalars>();
  g.tw = s->tw.as<float2>();
  g.sqsum = ep->sq.as<double>();
  g.saturation = saturation_level(s->prm);
  g.N = s->N;
  g.K = s->K;
  g.Ka = Ka;
  g.P = s->P;
  g.X = s->X;
  g.Y = s->Y;
  g.TX = ep->TX;
  g.TY = ep->TY;
  g.C = ep->C;
  g.pc = pc;
  g.up = up;
  g.rms = s->prm.calculateRMS ? 1 : 0;
  g.useAll = s->useAll ? 1 : 0;
  g.grid = ep->grid ? 1 : 0;
  g.gbar = ep->gsync.as<unsigned>();
  g.gerr = reinterpret_cast<int*>(ep->gsync.as<unsigned>() + 2);
  if (ep->chain) {
    EpieChainArgs cg;
    cg.amp = g.ampT;  // natural layout: the session transposes the planes only for the cluster / whole-GPU kernels
    cg.obj = g.obj;
    cg.ocache = g.ocache;
    cg.probe = g.probe;
    cg.pcache = g.pcache;
    cg.pos = g.pos;
    cg.order = g.order;
    cg.psi = ep->cpsi.as<float2>();
    cg.work = ep->cwork.as<float2>();
    cg.TM = g.TM;
    cg.sc = g.sc;
    cg.sqsum = g.sqsum;
    cg.pmax2 = ep->pmax2.as<float>();
    cg.tcerr = ep->tcerr.as<int>();
    cg.tw = g.tw;
    cg.saturation = g.saturation;
    cg.N = g.N;
    cg.K = g.K;
    cg.Ka = g.Ka;
    cg.P = g.P;
    cg.X = g.X;
    cg.Y = g.Y;
    cg.TX = g.TX;
    cg.TY = g.TY;
    cg.pc = g.pc;
    cg.up = g.up;
    cg.rms = g.rms;
    cg.useAll = g.useAll;
    cg.tc = ep->chain_tc ? 1 : 0;
    cg.frows = s->fft_rows;
    const unsigned key = unsigned(Ka) | (unsigned(up) << 8) | (unsigned(pc) << 9) | (unsigned(cg.rms) << 10);
    cudaGraphExec_t& ge = ep->chain_graphs[key];
    if (!ge) {
      cudaGraph_t graph = nullptr;
      check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
      const cudaError_t e1 = epie_chain_iteration(cg, s->stream);
      const cudaError_t e2 = cudaStreamEndCapture(s->stream, &graph);
      check_cuda(e1, "ePIE chain capture");
      check_cuda(e2, "end capture");
      const cudaError_t e3 = cudaGraphInstantiate(&ge, graph, 0);
      cudaGraphDestroy(graph);
      if (e3 != cudaSuccess) ep->chain_graphs.erase(key);
      check_cuda(e3, "graph instantiate");
    }
    check_cuda(cudaGraphLaunch(ge, s->stream), "ePIE chain");
    s->launches += epie_chain_launches(cg);
    if (ep->chain_tc) {  // the tensor-core transforms report a wait timeout through their device flag
      int flag = 0;
      check_cuda(cudaMemcpyAsync(&flag, cg.tcerr, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "D2H flag");
      check_cuda(cudaStreamSynchronize(s->stream), "ePIE iteration");
      need(flag == 0, "ePIE: a tensor-core FFT wait timed out", PTY_ERR_CUDA);
    }
  } else {
    check_cuda(ep->sm ? epie_sm_launch(g, s->stream) : epie_launch(g, s->stream), "ePIE kernel launch");
    s->launches += 1;
  }
  if (ep->grid) {  // the whole-GPU variant reports a grid-barrier timeout through a device flag
    int flag = 0;
    check_cuda(cudaMemcpyAsync(&flag, g.gerr, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "D2H flag");
    check_cuda(cudaStreamSynchronize(s->stream), "ePIE iteration");
    need(flag == 0, "ePIE: a grid barrier timed out (the iteration did not complete)", PTY_ERR_CUDA);
  }
  if (!want_err || !s->prm.calculateRMS) return 0.0;
  double e = 0;
  check_cuda(cudaMemcpyAsync(&e, &reinterpret_cast<EpieScalars*>(ep->sc.p)->err, sizeof(double),
                             cudaMemcpyDeviceToHost, s->stream),
             "D2H error");
  check_cuda(cudaStreamSynchronize(s->stream), "ePIE iteration");
  return e / s->P;
}

void destroy_session(pty_session* s) {
  if (!s) return;
  cudaSetDevice(s->dev);
  t_stream = s->stream;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& g : s->graphs)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : s->graphs_local)
    if (g) cudaGraphExecDestroy(g);
  for (auto& g : s->graphs_fin)
    if (g) cudaGraphExecDestroy(g);
  delete s->ep;
  s->ep = nullptr;
  delete s->ml;
  s->ml = nullptr;
  s->amp.free();
  s->obj.free();
  s->probe.free();
  s->ocache.free();
  s->pcache.free();
  s->tw.free();
  s->dOffs.free();
  s->scal.free();
  s->psi.free();
  s->dO.free();
  s->dP.free();
  s->W1.free();
  s->W2.free();
  s->slots.free();
  if (s->dm_side) cudaStreamDestroy(s->dm_side);
  if (s->dm_fork) cudaEventDestroy(s->dm_fork);
  if (s->dm_join) cudaEventDestroy(s->dm_join);
  t_stream = nullptr;
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

}  // namespace

// ============================================================================== C ABI
extern "C" {

int pty_params_init(pty_params* p) {
  if (!p) return PTY_ERR_INVALID;
  std::memset(p, 0, sizeof(*p));
  std::strcpy(p->algorithm, "ePIE");
  p->fs = 0;
  p->dpf = 1;
  p->beamSize = 400e-9;
  p->size = 512;
  p->qx = 128;
  p->qy = 128;
  p->nx = 256;
  p->ny = 256;
  p->scanDimsx = 26;
  p->scanDimsy = 26;
  p->stepx = 40e-9;
  p->stepy = 40e-9;
  p->probeModes = 1;
  p->lambd = 2.3843e-10;
  p->dx_d = 172e-6;
  p->z = 2.2;
  p->iter = 100;
  p->T = 0;
  p->jitterRadius = 0;
  p->delta_p = 0.1;
  p->phaseConstraint = 1;
  p->updateProbe = 10;
  p->updateModes = 20;
  p->PPS = 20;
  p->seed = 0x5EED5EEDull;
  p->calculateRMS = 0;
  p->device = 0;
  p->wave = 0;
  return PTY_OK;
}

int pty_session_create(const pty_params* p, pty_session** out) {
  if (!out) return PTY_ERR_INVALID;
  *out = nullptr;
  pty_session* s = nullptr;
  int rc = guarded([&] {
    need(p != nullptr, "null parameters");
    s = new pty_session;
    s->prm = *p;
    s->algo = parse_algo(p->algorithm);
    need(p->size > 16, "size must be larger than 16");  // src/Parameters.cpp:512-519
    need(p->probeModes >= 1, "probeModes must be >= 1");
    need(p->bitDepth >= 0 && p->bitDepth <= 32, "bitDepth must be 1..32 (0: not given)");
    need(p->scanDimsx > 0 && p->scanDimsy > 0, "scanDimsx and scanDimsy must be positive");
    need(p->lambd > 0 && p->z > 0 && p->dx_d > 0 && p->beamSize > 0, "lambd, z, dx_d, beamSize must be positive");
    if (p->fp[0]) {  // whole-mode ingest reads .bin and .csv; .h5 needs the HDF5 library, not linked here
      std::string ext(p->fp);
      const size_t dot = ext.find_last_of('.');
      ext = dot == std::string::npos ? "" : ext.substr(dot + 1);
      for (char& ch : ext) ch = char(std::tolower(static_cast<unsigned char>(ch)));
      need(ext != "h5", "HDF5 pattern files need the HDF5 library, which this build does not link; convert them to "
                        ".bin (raw float32) or .csv", PTY_ERR_UNSUPPORTED);
    }
    need(p->simulate == 0 || s->algo != ALGO_MLS,
         "simulate=1 is available for ePIE and DM (the reference's MLs simulation builds an ML mesh of its own)",
         PTY_ERR_UNSUPPORTED);
    need(p->beamstopMask == 0, "beamstop masks from files are not part of this engine", PTY_ERR_UNSUPPORTED);
    s->N = p->size;
    s->K = p->probeModes;
    s->rng = p->seed;
    int ndev = 0;
    check_cuda(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    need(p->device >= 0 && p->device < ndev, "device ordinal out of range");
    s->dev = p->device;
    set_device(s);
    create_session_stream(s, &s->stream);
    s->own_stream = true;
  });
  if (rc != PTY_OK) {
    destroy_session(s);
    return rc;
  }
  *out = s;
  return PTY_OK;
}

int pty_session_destroy(pty_session* s) {
  return guarded([&] { destroy_session(s); });
}

int pty_release_cached_memory(int device) {
  return guarded([&] {
    need(device >= -1 && device < 64, "device must be -1 (all) or an ordinal below 64");
    for (int d = 0; d < 64; ++d)
      if (device == -1 || device == d) cache_release(d);
  });
}

int pty_set_patterns(pty_session* s, const void* host, int dtype, int P, int N) {
  return guarded([&] {
    need(s && host, "null argument");
    need(!s->initialized, "patterns must be set before pty_init", PTY_ERR_STATE);
    need(dtype == PTY_F32 || dtype == PTY_F64, "dtype must be PTY_F32 or PTY_F64");
    need(N == s->N, "pattern size " + std::to_string(N) + " differs from size=" + std::to_string(s->N));
    need(fft_size_supported(N), "pattern size must be 32, 64, 128, 256 or 512");
    need(P >= 1, "need at least one pattern");
    set_device(s);
    s->P = P;
    upload_patterns(s, host, dtype, size_t(P) * N * N);
    check_cuda(cudaStreamSynchronize(s->stream), "patterns");
    s->have_patterns = true;
  });
}

int pty_set_positions(pty_session* s, const double* xy_m, int P) {
  return guarded([&] {
    need(s && xy_m, "null argument");
    need(!s->initialized, "positions must be set before pty_init", PTY_ERR_STATE);
    need(P >= 1, "need at least one position");
    s->pos_m.assign(xy_m, xy_m + 2 * size_t(P));
  });
}

int pty_set_object(pty_session* s, const float* c64, int X, int Y) {
  return guarded([&] {
    need(s && c64, "null argument");
    need(!s->initialized, "object must be set before pty_init", PTY_ERR_STATE);
    need(X > 0 && Y > 0, "bad object shape");
    s->obj_h.assign(c64, c64 + 2 * size_t(X) * Y);
    s->X = X;
    s->Y = Y;
  });
}

int pty_set_probe(pty_session* s, const float* c64, int K, int N) {
  return guarded([&] {
    need(s && c64, "null argument");
    need(!s->initialized, "probe must be set before pty_init", PTY_ERR_STATE);
    need(N == s->N, "probe size differs from size");
    need(K >= 1 && K <= s->K, "probe has more modes than probeModes");
    s->probe_h.assign(c64, c64 + 2 * size_t(K) * N * N);
    s->probe_given_modes = K;
  });
}

int pty_init(pty_session* s) {
  return guarded([&] {
    need(s != nullptr, "null session");
    need(!s->initialized, "session already initialised", PTY_ERR_STATE);
    set_device(s);
    const pty_params& p = s->prm;
    if (!s->have_patterns && p.simulate) {  // simulation mode: patterns from the forward model (sim_mode.cu)
      need(s->shard_total == 0, "position shards take their patterns from pty_set_patterns", PTY_ERR_UNSUPPORTED);
      s->P = s->pos_m.empty() ? p.scanDimsx * p.scanDimsy : int(s->pos_m.size() / 2);
      init_geometry(s);
      simulate_session_patterns(s);
    }
    if (!s->have_patterns && p.fp[0]) {  // whole-mode run: patterns from the data files (ingest.cu)
      need(s->shard_total == 0, "position shards take their patterns from pty_set_patterns", PTY_ERR_UNSUPPORTED);
      ingest_patterns(s, s->pos_m.empty() ? p.scanDimsx * p.scanDimsy : int(s->pos_m.size() / 2));
    }
    need(s->have_patterns, "no diffraction patterns (diffractionNP or fp) were given", PTY_ERR_STATE);
    const int Ptot = s->pos_m.empty() ? p.scanDimsx * p.scanDimsy : int(s->pos_m.size() / 2);
    if (s->shard_total > 0) {
      need(s->algo == ALGO_DM, "position shards are supported for DM only", PTY_ERR_UNSUPPORTED);
      need(s->shard_total == Ptot, "the shard's scan has " + std::to_string(s->shard_total) +
                                       " positions but the parameters describe " + std::to_string(Ptot));
      need(s->shard_first + s->P <= Ptot, "shard [" + std::to_string(s->shard_first) + ", " +
                                              std::to_string(s->shard_first + s->P) + ") exceeds the scan");
      need(!s->probe_h.empty() || p.probeGuess[0],
           "a DM shard needs the probe (probeNP or probeGuess): the guess uses every pattern of the scan");
    } else if (s->pos_m.empty()) {
      need(s->P == p.scanDimsx * p.scanDimsy,
           "pattern count " + std::to_string(s->P) + " differs from scanDimsx*scanDimsy = " +
               std::to_string(p.scanDimsx * p.scanDimsy));
    } else {
      need(int(s->pos_m.size() / 2) == s->P, "positionNP and diffractionNP have different lengths");
    }
    float2* twp = nullptr;
    check_cuda(make_twiddles(s->N, &twp, s->stream), "twiddles");
    s->tw.p = twp;  // allocated by make_twiddles; the cache takes it back like any block
    s->tw.bytes = s->tw.cap = sizeof(float2) * s->N;
    s->tw.dev = s->dev;
    need(s->algo != ALGO_DM || p.precision == 0 || s->N == 512,
         "precision=1 for DM (tensor-core column pass) needs 512 x 512 patterns", PTY_ERR_UNSUPPORTED);
    if (s->algo == ALGO_MLS) {
      need(s->warm_params.empty(), "the learned warm start is for ePIE and DM sessions", PTY_ERR_UNSUPPORTED);
      init_mls(s);
      s->initialized = true;
      return;
    }
    const int gX = s->X, gY = s->Y;
    init_geometry(s);
    if (!s->obj_h.empty())
      need(gX == s->X && gY == s->Y, "objectNP shape (" + std::to_string(gX) + ", " + std::to_string(gY) +
                                         ") differs from the scan's object size (" + std::to_string(s->X) + ", " +
                                         std::to_string(s->Y) + ")");
    s->dOffs.alloc(sizeof(int) * 2 * s->P, "offsets");
    check_cuda(cudaMemcpyAsync(s->dOffs.p, s->offs.data(), sizeof(int) * 2 * s->P, cudaMemcpyHostToDevice, s->stream),
               "H2D offsets");
    const size_t NN = size_t(s->N) * s->N;
    {
      DeviceBuf avg;
      if (p.probeGuess[0] == 0 && s->probe_h.empty()) {
        avg.alloc(sizeof(float) * NN, "mean amplitude");
        check_cuda(mean_amplitude(s->amp.as<float>(), s->P, s->N, avg.as<float>(), s->stream), "mean amplitude");
      }
      init_probe(s, avg.as<float>());
    }
    init_object(s);
    if (!s->warm_params.empty()) {
      need(s->shard_total == 0, "the warm start needs the whole scan's patterns (not a position shard)",
           PTY_ERR_UNSUPPORTED);
      need(s->obj_h.empty() && !p.objectGuess[0], "warmStart and objectNP / objectGuess are exclusive");
      need(s->N % 16 == 0, "the warm-start network needs N to be a multiple of 16");
      const size_t want = warm_param_count(s->N, s->warm_width);
      need(s->warm_params.size() == want, "warmStart has " + std::to_string(s->warm_params.size()) +
                                              " parameters; the width-" + std::to_string(s->warm_width) +
                                              " network for " + std::to_string(s->N) + "^2 patterns has " +
                                              std::to_string(want));
      run_warm_start(s);
    }
    // the cluster / whole-GPU ePIE kernels consume the amplitudes column-wise: transpose each plane once (DM, the
    // shared-memory ePIE kernel and the chain, whose modulus step walks the plane as its transforms leave it, read
    // them in their natural layout; which ePIE kernel runs also depends on the variant the autotuner chose)
    if (s->algo == ALGO_EPIE && !epie_uses_sm_kernel(s) && !epie_uses_chain(s)) {
      DeviceBuf t;
      t.alloc(s->amp.bytes, "transposed patterns");
      check_cuda(transpose_planes(s->amp.as<float>(), t.as<float>(), s->P, s->N, s->stream), "transpose");
      check_cuda(cudaStreamSynchronize(s->stream), "transpose");
      s->amp.swap(t);
      s->amp_transposed = true;
    }
    if (s->algo == ALGO_EPIE) {
      init_epie(s);
    } else {
      init_dm(s);
      if (!s->warm_params.empty()) {  // start DM from the warm object's exit waves, not from zero
        check_cuda(dm_psi_from_object(dm_buffers(s), s->P, s->stream), "exit waves from the warm object");
        check_cuda(cudaStreamSynchronize(s->stream), "exit waves from the warm object");
      }
    }
    s->initialized = true;
  });
}

int pty_step(pty_session* s, double* err) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->shard_total == 0, "a position shard steps with pty_dm_step_local, a reduction, pty_dm_step_finish",
         PTY_ERR_STATE);
    set_device(s);
    const int it = s->iter + 1;
    double e = 0;
    if (s->algo == ALGO_EPIE)
      e = step_epie(s, it, err != nullptr);
    else if (s->algo == ALGO_MLS)
      e = step_mls(s, err != nullptr);
    else
      step_dm(s, it);
    s->iter = it;
    if (err) *err = e;
  });
}

int pty_run(pty_session* s, int iters, double* errs) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->shard_total == 0, "a position shard steps with pty_dm_step_local, a reduction, pty_dm_step_finish",
         PTY_ERR_STATE);
    need(iters >= 0, "negative iteration count");
    set_device(s);
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < iters; ++i) {
      const int it = s->iter + 1;
      double e = 0;
      if (s->algo == ALGO_EPIE)
        e = step_epie(s, it, errs != nullptr);
      else if (s->algo == ALGO_MLS)
        e = step_mls(s, errs != nullptr);
      else
        step_dm(s, it);
      s->iter = it;
      if (errs) errs[i] = e;
      if (s->prm.save > 0 && it % s->prm.save == 0)  // checkpoint (IPhaser::phaseLoop, src/IPhaser.cpp:384-385)
        write_results(s, s->prm.outputDir[0] ? s->prm.outputDir : "data", it / s->prm.save, s->prm.binaryOutput != 0);
      if (s->prm.T > 0) {  // wall-time limit (src/IPhaser.cpp:386-387)
        check_cuda(cudaStreamSynchronize(s->stream), "iteration");
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= s->prm.T) break;
      }
    }
    check_cuda(cudaStreamSynchronize(s->stream), "pty_run");
    dm_check_flag(s);
  });
}

int pty_set_shard(pty_session* s, int first, int total) {
  return guarded([&] {
    need(s != nullptr, "null session");
    need(!s->initialized, "the shard must be set before pty_init", PTY_ERR_STATE);
    need(first >= 0 && total >= 1, "shard start must be >= 0 and the scan size >= 1");
    s->shard_first = first;
    s->shard_total = total;
  });
}

int pty_dm_step_local(pty_session* s) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->algo == ALGO_DM, "pty_dm_step_local is for DM sessions", PTY_ERR_STATE);
    need(s->pending_iter == 0, "pty_dm_step_finish has not run for the previous local step", PTY_ERR_STATE);
    set_device(s);
    const int it = s->iter + 1;
    step_dm_local(s, it);
    s->pending_iter = it;
  });
}

int pty_dm_increments(pty_session* s, void** dO, size_t* n_obj, void** dP, size_t* n_probe) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->algo == ALGO_DM, "increments exist for DM sessions only", PTY_ERR_STATE);
    if (dO) *dO = s->dO.p;
    if (n_obj) *n_obj = size_t(s->X) * s->Y;
    if (dP) *dP = s->dP.p;
    if (n_probe) *n_probe = size_t(s->N) * s->N;
  });
}

int pty_dm_step_finish(pty_session* s) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->pending_iter > 0, "pty_dm_step_local has not run", PTY_ERR_STATE);
    set_device(s);
    step_dm_finish(s, s->pending_iter);
    dm_check_flag(s);
    s->iter = s->pending_iter;
    s->pending_iter = 0;
  });
}

int pty_set_warm_start(pty_session* s, const float* params, size_t n_params, int width) {
  return guarded([&] {
    need(s != nullptr, "null session");
    need(!s->initialized, "the warm start must be set before pty_init", PTY_ERR_STATE);
    if (n_params == 0 || !params) {
      s->warm_params.clear();
      s->warm_width = 0;
      return;
    }
    need(width >= 1, "warm-start width must be positive");
    s->warm_params.assign(params, params + n_params);
    s->warm_width = width;
  });
}

int pty_dm_psi_from_object(pty_session* s) {
  return guarded([&] {
    need(s && s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->algo == ALGO_DM, "exit waves exist for DM only", PTY_ERR_UNSUPPORTED);
    need(s->pending_iter == 0, "a sharded step is in progress", PTY_ERR_STATE);
    set_device(s);
    check_cuda(dm_psi_from_object(dm_buffers(s), s->P, s->stream), "exit waves from the object");
    check_cuda(cudaStreamSynchronize(s->stream), "exit waves from the object");
  });
}

int pty_simulate(const float* obj_c64, int X, int Y, const float* probe_c64, int N, const float* pos_px, int P,
                 float* amp_out) {
  return guarded([&] {
    need(obj_c64 && probe_c64 && pos_px && amp_out, "null argument");
    need(X >= N && Y >= N && P >= 0, "object smaller than the probe window or negative pattern count");
    need(fft_size_supported(N), "N must be 32, 64, 128, 256 or 512");
    for (int i = 0; i < P; ++i)
      need(pos_px[2 * i] >= 0 && pos_px[2 * i + 1] >= 0, "position " + std::to_string(i) + " is negative");
    const size_t NN = size_t(N) * N, XY = size_t(X) * Y;
    const int chunk = int(std::max<size_t>(1, std::min<size_t>(size_t(P), (size_t(256) << 20) / (16 * NN))));
    cudaStream_t st = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    DeviceBuf obj, probe, pos, psi, work, amp;
    float2* tw = nullptr;
    try {
      obj.alloc(sizeof(float2) * XY, "object");
      probe.alloc(sizeof(float2) * NN, "probe");
      pos.alloc(sizeof(float2) * std::max(P, 1), "positions");
      psi.alloc(sizeof(float2) * NN * chunk, "exit waves");
      work.alloc(sizeof(float2) * NN * chunk, "FFT work");
      amp.alloc(sizeof(float) * NN * chunk, "amplitudes");
      check_cuda(cudaMemcpyAsync(obj.p, obj_c64, obj.bytes, cudaMemcpyDefault, st), "copy object");
      check_cuda(cudaMemcpyAsync(probe.p, probe_c64, probe.bytes, cudaMemcpyDefault, st), "copy probe");
      if (P) check_cuda(cudaMemcpyAsync(pos.p, pos_px, sizeof(float2) * P, cudaMemcpyDefault, st), "copy positions");
      check_cuda(make_twiddles(N, &tw, st), "twiddles");
      for (int i0 = 0; i0 < P; i0 += chunk) {
        const int cnt = std::min(chunk, P - i0);
        check_cuda(simulate_patterns(obj.as<float2>(), X, Y, probe.as<float2>(), N, pos.as<float2>() + i0, cnt,
                                     psi.as<float2>(), work.as<float2>(), tw, amp.as<float>(), st),
                   "simulate");
        check_cuda(cudaMemcpyAsync(amp_out + size_t(i0) * NN, amp.p, sizeof(float) * NN * cnt, cudaMemcpyDefault, st),
                   "copy amplitudes");
        check_cuda(cudaStreamSynchronize(st), "simulate");
      }
    } catch (...) {
      cudaStreamSynchronize(st);
      if (tw) cudaFree(tw);
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamSynchronize(st);
    cudaFree(tw);
    cudaStreamDestroy(st);
  });
}

int pty_batch_run(pty_session* const* sessions, int n, int iters) {
  return guarded([&] {
    need(sessions && n > 0, "no sessions");
    need(iters >= 0, "negative iteration count");
    for (int i = 0; i < n; ++i) {
      need(sessions[i] != nullptr, "null session in the batch");
      need(sessions[i]->initialized, "pty_init has not run for session " + std::to_string(i), PTY_ERR_STATE);
      need(sessions[i]->dev == sessions[0]->dev, "batched sessions must share one device");
      need(sessions[i]->shard_total == 0, "position shards do not run in a batch", PTY_ERR_STATE);
    }
    set_device(sessions[0]);
    // round-robin: one iteration of every scan per round, each on its own stream, no host synchronisation for DM
    // and MLs steps, so the scans' kernels run side by side
    for (int it = 0; it < iters; ++it)
      for (int i = 0; i < n; ++i) {
        pty_session* s = sessions[i];
        t_stream = s->stream;
        const int k = s->iter + 1;
        if (s->algo == ALGO_EPIE)
          step_epie(s, k, false);
        else if (s->algo == ALGO_MLS)
          step_mls(s, false, true);
        else
          step_dm(s, k);
        s->iter = k;
      }
    for (int i = 0; i < n; ++i) check_cuda(cudaStreamSynchronize(sessions[i]->stream), "pty_batch_run");
    for (int i = 0; i < n; ++i) dm_check_flag(sessions[i]);
  });
}

int pty_get_dims(const pty_session* s, int* X, int* Y, int* K, int* N, int* P, int* iters_done) {
  if (!s) return PTY_ERR_INVALID;
  if (X) *X = s->X;
  if (Y) *Y = s->Y;
  if (K) *K = s->K;
  if (N) *N = s->N;
  if (P) *P = s->P;
  if (iters_done) *iters_done = s->iter;
  return PTY_OK;
}

int pty_get_object(pty_session* s, float* out, int X, int Y) {
  return guarded([&] {
    need(s && out, "null argument");
    need(s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(X == s->X && Y == s->Y, "object buffer shape mismatch");
    set_device(s);
    check_cuda(cudaMemcpyAsync(out, s->obj.p, sizeof(float2) * size_t(X) * Y, cudaMemcpyDeviceToHost, s->stream),
               "D2H object");
    check_cuda(cudaStreamSynchronize(s->stream), "D2H object");
    dm_check_flag(s);
  });
}

int pty_get_patterns(pty_session* s, float* out, int P, int N) {
  return guarded([&] {
    need(s && out, "null argument");
    need(s->have_patterns, "the session has no patterns", PTY_ERR_STATE);
    need(P == s->P && N == s->N, "pattern shape differs from the session's");
    set_device(s);
    const size_t NN = size_t(N) * N;
    check_cuda(cudaMemcpyAsync(out, s->amp.p, sizeof(float) * NN * P, cudaMemcpyDeviceToHost, s->stream), "D2H");
    check_cuda(cudaStreamSynchronize(s->stream), "D2H patterns");
    if (s->amp_transposed) {  // back to the natural [x][y] layout
      std::vector<float> t(NN);
      for (int i = 0; i < P; ++i) {
        float* pl = out + NN * i;
        for (int x = 0; x < N; ++x)
          for (int y = 0; y < N; ++y) t[size_t(x) * N + y] = pl[size_t(y) * N + x];
        std::copy(t.begin(), t.end(), pl);
      }
    }
  });
}

int pty_get_probe(pty_session* s, float* out, int K, int N) {
  return guarded([&] {
    need(s && out, "null argument");
    need(s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(K == s->K && N == s->N, "probe buffer shape mismatch");
    set_device(s);
    check_cuda(cudaMemcpyAsync(out, s->probe.p, sizeof(float2) * size_t(K) * N * N, cudaMemcpyDeviceToHost,
                               s->stream),
               "D2H probe");
    check_cuda(cudaStreamSynchronize(s->stream), "D2H probe");
    dm_check_flag(s);
  });
}

int pty_get_positions(const pty_session* s, float* xy_px, int P) {
  return guarded([&] {
    need(s && xy_px, "null argument");
    need(s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(P == s->P, "position buffer length mismatch");
    if (s->ml && s->ml->variable) {  // the refined positions
      check_cuda(cudaSetDevice(s->dev), "cudaSetDevice");
      check_cuda(cudaMemcpyAsync(xy_px, s->ml->pos.p, sizeof(float) * 2 * size_t(P), cudaMemcpyDeviceToHost,
                                 s->stream),
                 "D2H positions");
      check_cuda(cudaStreamSynchronize(s->stream), "D2H positions");
      return;
    }
    std::memcpy(xy_px, s->geo.pos.data(), sizeof(float) * 2 * size_t(P));
  });
}

int pty_get_mls_state(const pty_session* s, float* E_c64, double* evo0, double* evo1, int N, int P) {
  return guarded([&] {
    need(s != nullptr, "null argument");
    need(s->initialized, "pty_init has not run", PTY_ERR_STATE);
    need(s->ml && s->ml->variable, "no MLs default-path state (another algorithm, or mlsCore = 1)", PTY_ERR_STATE);
    need(N == s->N && P == s->P, "buffer size mismatch");
    check_cuda(cudaSetDevice(s->dev), "cudaSetDevice");
    const size_t NN = size_t(N) * N;
    if (E_c64)
      check_cuda(cudaMemcpyAsync(E_c64, s->ml->E.p, sizeof(float2) * NN, cudaMemcpyDeviceToHost, s->stream), "D2H");
    if (evo0)
      check_cuda(cudaMemcpyAsync(evo0, s->ml->evo.p, sizeof(double) * P, cudaMemcpyDeviceToHost, s->stream), "D2H");
    if (evo1)
      check_cuda(cudaMemcpyAsync(evo1, s->ml->evo.as<double>() + P, sizeof(double) * P, cudaMemcpyDeviceToHost,
                                 s->stream),
                 "D2H");
    check_cuda(cudaStreamSynchronize(s->stream), "D2H MLs state");
  });
}

int pty_write_results(pty_session* s, const char* dir, int r, int binary) {
  return guarded([&] {
    need(s && dir, "null argument");
    need(s->initialized, "pty_init has not run", PTY_ERR_STATE);
    write_results(s, dir, r, binary != 0);
  });
}

int pty_set_stream(pty_session* s, void* st) {
  return guarded([&] {
    need(s != nullptr, "null session");
    set_device(s);
    check_cuda(cudaStreamSynchronize(s->stream), "stream switch");
    for (auto& g : s->graphs) {
      if (g) cudaGraphExecDestroy(g);
      g = nullptr;
    }
    if (st) {
      if (s->own_stream) cudaStreamDestroy(s->stream);
      s->stream = static_cast<cudaStream_t>(st);
      s->own_stream = false;
    } else if (!s->own_stream) {
      create_session_stream(s, &s->stream);
      s->own_stream = true;
    }
  });
}

int64_t pty_kernel_launches(const pty_session* s) { return s ? s->launches : -1; }

const char* pty_last_error(void) { return g_last_error.c_str(); }

int pty_fft2_dev(void* data_dev, void* work_dev, int batch, int N, int inverse, void* st) {
  return guarded([&] {
    need(data_dev && work_dev && batch >= 1, "bad argument");
    need(fft_size_supported(N), "unsupported FFT size");
    cudaStream_t stream = static_cast<cudaStream_t>(st);
    float2* tw = nullptr;
    check_cuda(make_twiddles(N, &tw, stream), "twiddles");
    cudaError_t e = fft2(static_cast<float2*>(data_dev), static_cast<float2*>(work_dev), tw, batch, N, inverse != 0,
                         stream);
    cudaError_t e2 = cudaStreamSynchronize(stream);
    cudaFree(tw);
    check_cuda(e, "fft2");
    check_cuda(e2, "fft2 sync");
  });
}

}  // extern "C"
