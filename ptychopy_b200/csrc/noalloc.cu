// Allocation-free batched 2-D FFT (pty_fft2_dev_noalloc).
//
// pty_fft2_dev needs a caller-provided work buffer and allocates its twiddle table with cudaMalloc.  This variant
// allocates nothing: the work buffer and the twiddle tables of every supported size live in file-scope device
// arrays below.  A GPU holds them from the moment the runtime loads this file's device code onto it (under the
// default lazy module loading: the first call on that device) until the process exits.
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ptychopy_b200.h"
#include "fft_core.cuh"
#include "kernels.h"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

// Largest batch*N*N*8 bytes one call may transform.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kTwiddleSizes[5] = {32, 64, 128, 256, 512};
constexpr int kTwiddleTotal = 32 + 64 + 128 + 256 + 512;

static __device__ __align__(256) float2 g_noalloc_work[kNoAllocScratchBytes / sizeof(float2)];
static __device__ __align__(256) float2 g_noalloc_twiddles[kTwiddleTotal];

namespace {

struct DeviceScratch {
  bool ready = false;
  float2* work = nullptr;      // device address of g_noalloc_work on this device
  float2* twiddles = nullptr;  // device address of g_noalloc_twiddles on this device
};

constexpr int kMaxDevices = 64;
DeviceScratch g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

// Stage-1 twiddles of a length-N transform in the [k1][t] layout the FFT kernels read (computed in double).
void host_twiddles(int N, std::vector<float2>& out) {
  const int T = fft_lanes(N);
  const int E = N / T;
  out.resize(N);
  for (int k1 = 0; k1 < E; ++k1)
    for (int t = 0; t < T; ++t) {
      const double a = -2.0 * M_PI * double((long long)t * k1 % N) / double(N);
      out[k1 * T + t] = make_float2(float(std::cos(a)), float(std::sin(a)));
    }
}

int twiddle_offset(int N) {
  int off = 0;
  for (int n : kTwiddleSizes) {
    if (n == N) return off;
    off += n;
  }
  return -1;
}

// Once per device, with that device current: resolve the arrays' device addresses and fill the twiddles.
cudaError_t setup_device(int dev, DeviceScratch** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  DeviceScratch& d = g_scratch[dev];
  if (!d.ready) {
    void* w = nullptr;
    void* tw = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&w, g_noalloc_work);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(&tw, g_noalloc_twiddles);
    if (e != cudaSuccess) return e;
    std::vector<float2> all(kTwiddleTotal), one;
    for (int n : kTwiddleSizes) {
      host_twiddles(n, one);
      std::copy(one.begin(), one.end(), all.begin() + twiddle_offset(n));
    }
    e = cudaMemcpy(tw, all.data(), sizeof(float2) * kTwiddleTotal, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    d.work = static_cast<float2*>(w);
    d.twiddles = static_cast<float2*>(tw);
    d.ready = true;
  }
  *out = &d;
  return cudaSuccess;
}

int fail_with(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

}  // namespace
}  // namespace pty

extern "C" int pty_fft2_dev_noalloc(void* data_dev, int batch, int N, int inverse, void* cuda_stream) {
  using namespace pty;
  if (!data_dev || batch < 1) return fail_with(PTY_ERR_INVALID, "pty_fft2_dev_noalloc: null data or batch < 1");
  if (!fft_size_supported(N))
    return fail_with(PTY_ERR_INVALID, "pty_fft2_dev_noalloc: N must be 32, 64, 128, 256 or 512");
  const size_t need = size_t(batch) * size_t(N) * size_t(N) * sizeof(float2);
  if (need > kNoAllocScratchBytes)
    return fail_with(PTY_ERR_INVALID, "pty_fft2_dev_noalloc: batch*N*N*8 = " + std::to_string(need) +
                                          " bytes exceeds the 8 MiB static scratch (at most " +
                                          std::to_string(kNoAllocScratchBytes / (size_t(N) * N * sizeof(float2))) +
                                          " arrays of " + std::to_string(N) + "x" + std::to_string(N) + ")");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail_with(PTY_ERR_CUDA, std::string("pty_fft2_dev_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail_with(PTY_ERR_INVALID, "pty_fft2_dev_noalloc: device ordinal " + std::to_string(dev) +
                                          " is above the " + std::to_string(kMaxDevices - 1) + " this entry supports");
  DeviceScratch* sc = nullptr;
  e = setup_device(dev, &sc);
  if (e != cudaSuccess)
    return fail_with(PTY_ERR_CUDA, std::string("pty_fft2_dev_noalloc: scratch set-up: ") + cudaGetErrorString(e));
  e = fft2(static_cast<float2*>(data_dev), sc->work, sc->twiddles + twiddle_offset(N), batch, N, inverse != 0,
           static_cast<cudaStream_t>(cuda_stream));
  if (e != cudaSuccess)
    return fail_with(PTY_ERR_CUDA, std::string("pty_fft2_dev_noalloc: launch: ") + cudaGetErrorString(e));
  set_last_error("");
  return PTY_OK;
}
