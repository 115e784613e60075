// Generic building-block kernels: batched 2-D FFT (row transform + transposed store, applied twice),
// plane transposes, the probe-guess stages and small reductions.
#include <cmath>
#include <vector>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels.h"

namespace pty {

bool fft_size_supported(int N) { return N == 32 || N == 64 || N == 128 || N == 256 || N == 512; }

cudaError_t make_twiddles(int N, float2** d_tw, cudaStream_t st) {
  const int T = fft_lanes(N);
  if (!T || N > 512) return cudaErrorInvalidValue;
  const int E = N / T;
  std::vector<float2> h(N);
  for (int k1 = 0; k1 < E; ++k1)
    for (int t = 0; t < T; ++t) {
      double a = -2.0 * M_PI * double((long long)t * k1 % N) / double(N);
      h[k1 * T + t] = make_float2(float(std::cos(a)), float(std::sin(a)));
    }
  cudaError_t e = cudaMalloc(d_tw, sizeof(float2) * N);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(*d_tw, h.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);  // h goes out of scope
}

// ---- row transform + transposed store ------------------------------------------------------------------
template <int L, bool INV>
__global__ void __launch_bounds__(FftShape<L>::THREADS) k_fft_rows_t(const float2* __restrict__ in,
                                                                      float2* __restrict__ out,
                                                                      const float2* __restrict__ g_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  float2* s_tw = smem;
  float2* s_x = smem + L;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  const size_t plane = size_t(blockIdx.y) * L * L;
  const int x0 = blockIdx.x * R;
  load_twiddles<L>(s_tw, g_tw);
  __syncthreads();
  const float2* row = in + plane + size_t(x0 + v) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
  fft_vec<L, INV>(a, t, s_x + v * S::XCH, s_tw);
  store_rows_transposed<L, R>(a, out + plane, x0, v, t, s_x);
}

template <int L>
static cudaError_t launch_fft_pass(const float2* in, float2* out, const float2* tw, int batch, bool inverse,
                                   cudaStream_t st) {
  constexpr int R = FftShape<L>::RC, NT = FftShape<L>::THREADS;
  const size_t smem = rows_smem_bytes<L>();
  dim3 grid(L / R, batch);
  if (inverse) {
    cudaFuncSetAttribute(k_fft_rows_t<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    k_fft_rows_t<L, true><<<grid, NT, smem, st>>>(in, out, tw);
  } else {
    cudaFuncSetAttribute(k_fft_rows_t<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    k_fft_rows_t<L, false><<<grid, NT, smem, st>>>(in, out, tw);
  }
  return cudaGetLastError();
}

cudaError_t fft2(float2* data, float2* work, const float2* tw, int batch, int N, bool inverse, cudaStream_t st) {
  cudaError_t e;
#define PTY_FFT2(L)                                                        \
  case L:                                                                  \
    e = launch_fft_pass<L>(data, work, tw, batch, inverse, st);            \
    if (e != cudaSuccess) return e;                                        \
    return launch_fft_pass<L>(work, data, tw, batch, inverse, st);
  switch (N) {
    PTY_FFT2(32)
    PTY_FFT2(64)
    PTY_FFT2(128)
    PTY_FFT2(256)
    PTY_FFT2(512)
    default:
      return cudaErrorInvalidValue;
  }
#undef PTY_FFT2
}

// ---- plane transpose (32 x 32 tiles through shared memory) ----------------------------------------------
__global__ void k_transpose_planes(const float* __restrict__ in, float* __restrict__ out, int N) {
  __shared__ float tile[32][33];
  const size_t plane = size_t(blockIdx.z) * N * N;
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {
    int x = by + j, y = bx + threadIdx.x;
    if (x < N && y < N) tile[j][threadIdx.x] = in[plane + size_t(x) * N + y];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += 8) {
    int y = bx + j, x = by + threadIdx.x;
    if (x < N && y < N) out[plane + size_t(y) * N + x] = tile[threadIdx.x][j];
  }
}

cudaError_t transpose_planes(const float* in, float* out, int batch, int N, cudaStream_t st) {
  dim3 grid((N + 31) / 32, (N + 31) / 32, batch), block(32, 8);
  k_transpose_planes<<<grid, block, 0, st>>>(in, out, N);
  return cudaGetLastError();
}

// ---- probe guess stages ----------------------------------------------------------------------------------
__global__ void k_mean_amplitude(const float* __restrict__ amp, int P, size_t NN, float* __restrict__ avg) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < NN; i += size_t(gridDim.x) * blockDim.x) {
    double s = 0;
    for (int p = 0; p < P; ++p) s += amp[size_t(p) * NN + i];
    avg[i] = float(s / double(P));
  }
}

cudaError_t mean_amplitude(const float* amp, int P, int N, float* avg, cudaStream_t st) {
  size_t NN = size_t(N) * N;
  k_mean_amplitude<<<int((NN + 255) / 256), 256, 0, st>>>(amp, P, NN, avg);
  return cudaGetLastError();
}

// d_initProbe (src/ProbeKernels.cu:207-218): |sinc(r*dx_s/beam) * exp(-(r/window)^2)| measured from N/2.
__global__ void k_probe_start(float2* __restrict__ probe0, int N, float window, float factor) {
  const int x = blockIdx.x;
  for (int y = threadIdx.x; y < N; y += blockDim.x) {
    float a = float(double(x) - N * 0.5), b = float(double(y) - N * 0.5);
    float r = sqrtf(a * a + b * b);
    float p = r * factor;
    p = (p != 0.f) ? sinpif(p) / (float(M_PI) * p) : 1.f;
    float g = expf(-(r * r) / (window * window));
    probe0[size_t(x) * N + y] = make_float2(fabsf(p * g), 0.f);
  }
}

cudaError_t probe_start(float2* probe0, int N, float window, float factor, cudaStream_t st) {
  k_probe_start<<<N, 256, 0, st>>>(probe0, N, window, factor);
  return cudaGetLastError();
}

__global__ void k_modulus_project(float2* __restrict__ spec, const float* __restrict__ avg, int n, float scale) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    spec[i] = modulus_replace(spec[i], avg[i] * scale);
}

cudaError_t modulus_project(float2* spec, const float* avg, int n, float scale, cudaStream_t st) {
  k_modulus_project<<<(n + 255) / 256, 256, 0, st>>>(spec, avg, n, scale);
  return cudaGetLastError();
}

// ---- reductions -----------------------------------------------------------------------------------------
__global__ void k_abs_max(const float2* __restrict__ a, size_t n, double* out) {
  double m = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    float2 v = a[i];
    m = fmax(m, double(sqrtf(v.x * v.x + v.y * v.y)));
  }
  m = block_reduce_max(m);
  if (threadIdx.x == 0) atomic_max_nonneg(out, m);
}

__global__ void k_sum_sq(const float2* __restrict__ a, size_t n, double* out) {
  double s = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    float2 v = a[i];
    s += double(v.x * v.x + v.y * v.y);
  }
  s = block_reduce_sum(s);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

static int reduce_grid(size_t n) {
  size_t g = (n + 255) / 256;
  return int(g > 1184 ? 1184 : (g < 1 ? 1 : g));
}

cudaError_t reduce_abs_max(const float2* a, size_t n, double* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
  if (e != cudaSuccess) return e;
  k_abs_max<<<reduce_grid(n), 256, 0, st>>>(a, n, out);
  return cudaGetLastError();
}

cudaError_t reduce_sum_sq(const float2* a, size_t n, double* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
  if (e != cudaSuccess) return e;
  k_sum_sq<<<reduce_grid(n), 256, 0, st>>>(a, n, out);
  return cudaGetLastError();
}

__global__ void k_scale_by_inverse(float2* __restrict__ a, size_t n, const double* __restrict__ denom) {
  const float s = float(1.0 / denom[0]);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = cscale(a[i], s);
}

cudaError_t scale_by_inverse(float2* a, size_t n, const double* denom, cudaStream_t st) {
  k_scale_by_inverse<<<reduce_grid(n), 256, 0, st>>>(a, n, denom);
  return cudaGetLastError();
}

__global__ void k_abs2(const float2* __restrict__ a, float* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    float2 v = a[i];
    float m = sqrtf(v.x * v.x + v.y * v.y);
    out[i] = m * m;
  }
}

cudaError_t abs2(const float2* a, float* out, size_t n, cudaStream_t st) {
  k_abs2<<<reduce_grid(n), 256, 0, st>>>(a, out, n);
  return cudaGetLastError();
}

__global__ void k_probe_modal_max(const float* __restrict__ cache, int K, size_t NN, int useAll, float* out) {
  float m = 0.f;
  if (useAll && K > 1) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < NN; i += size_t(gridDim.x) * blockDim.x) {
      float s = 0.f;
      for (int k = 0; k < K; ++k) s += cache[size_t(k) * NN + i];
      m = fmaxf(m, s);
    }
  } else {
    const size_t n = size_t(K) * NN;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
      m = fmaxf(m, cache[i]);
  }
  m = block_reduce_maxf(m);
  if (threadIdx.x == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(m));
}

cudaError_t probe_modal_max(const float* cache, int K, size_t NN, int useAll, float* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), st);
  if (e != cudaSuccess) return e;
  k_probe_modal_max<<<reduce_grid(NN), 256, 0, st>>>(cache, K, NN, useAll, out);
  return cudaGetLastError();
}

__global__ void k_scale_complex(float2* __restrict__ a, size_t n, float s) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = cscale(a[i], s);
}

cudaError_t scale_complex(float2* a, size_t n, float s, cudaStream_t st) {
  k_scale_complex<<<reduce_grid(n), 256, 0, st>>>(a, n, s);
  return cudaGetLastError();
}

__global__ void k_fill_complex(float2* __restrict__ a, size_t n, float2 v) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) a[i] = v;
}

cudaError_t fill_complex(float2* a, size_t n, float2 v, cudaStream_t st) {
  k_fill_complex<<<reduce_grid(n), 256, 0, st>>>(a, n, v);
  return cudaGetLastError();
}

__global__ void k_plane_sums(const float* __restrict__ a, size_t NN, double* __restrict__ out) {
  const float* pl = a + size_t(blockIdx.x) * NN;
  double s = 0;
  for (size_t i = threadIdx.x; i < NN; i += blockDim.x) s += pl[i];
  s = block_reduce_sum(s);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

cudaError_t plane_sums(const float* a, int P, size_t NN, double* out, cudaStream_t st) {
  k_plane_sums<<<P, 256, 0, st>>>(a, NN, out);
  return cudaGetLastError();
}

// Forward model of simulation mode (Diffractions::simulate, src/Diffractions.cpp:80-117, with d_simulatePSI,
// src/SampleKernels.cu:113-122): psi = bilinear O at (x + qx, y + qy) (texture fetch, 1/256 weights, clamp) times the
// probe, then FFT2 and modulus.  This kernel writes psi for `count` positions starting at pos.
__global__ void k_simulate_psi(const float2* __restrict__ obj, int X, int Y, const float2* __restrict__ probe, int N,
                               const float2* __restrict__ pos, int count, float2* __restrict__ psi) {
  const int i = blockIdx.y;
  if (i >= count) return;
  const float2 q = pos[i];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N * N; k += gridDim.x * blockDim.x) {
    const int x = k / N, y = k % N;
    int r0, r1, c0, c1;
    float wb, wa;
    tex_axis(q.x, x, X, r0, r1, wb);
    tex_axis(q.y, y, Y, c0, c1, wa);
    const float2 v00 = obj[size_t(r0) * Y + c0], v01 = obj[size_t(r0) * Y + c1];
    const float2 v10 = obj[size_t(r1) * Y + c0], v11 = obj[size_t(r1) * Y + c1];
    const float w00 = (1.f - wa) * (1.f - wb), w01 = wa * (1.f - wb), w10 = (1.f - wa) * wb, w11 = wa * wb;
    const float2 pt = make_float2(v00.x * w00 + v01.x * w01 + v10.x * w10 + v11.x * w11,
                                  v00.y * w00 + v01.y * w01 + v10.y * w10 + v11.y * w11);
    psi[size_t(i) * N * N + k] = cmul(pt, probe[k]);
  }
}

__global__ void k_abs(const float2* __restrict__ in, size_t n, float* __restrict__ out) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float2 v = in[i];
    out[i] = sqrtf(v.x * v.x + v.y * v.y);
  }
}

cudaError_t simulate_patterns(const float2* obj, int X, int Y, const float2* probe, int N, const float2* pos,
                              int count, float2* psi, float2* work, const float2* tw, float* amp, cudaStream_t st) {
  const int gx = (N * N + 255) / 256 < 64 ? (N * N + 255) / 256 : 64;
  k_simulate_psi<<<dim3(gx, count), 256, 0, st>>>(obj, X, Y, probe, N, pos, count, psi);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = fft2(psi, work, tw, count, N, false, st)) != cudaSuccess) return e;
  const size_t n = size_t(count) * N * N;
  k_abs<<<reduce_grid(n), 256, 0, st>>>(psi, n, amp);
  return cudaGetLastError();
}

}  // namespace pty
