// Device helpers shared by the engine's kernels: staging stores, the modulus replacement, phase clamp,
// block reductions.
#pragma once
#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace pty {

// Programmatic dependent launch: a kernel launched with launch_pdl (pdl.cuh) may start while its predecessor in the
// stream still runs; it waits here until that grid has completed and its memory is visible, then lets its own
// dependent launch begin.  Outside such a launch both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace pty

namespace pty {

// Shared memory of a row-transform CTA (FftShape<L>::RC rows): twiddles + max(exchange, transposed staging).
template <int L, int R>
__host__ __device__ constexpr size_t rows_smem_bytes_r() {
  constexpr int xch = R * FftShape<L>::XCH, stage = L * (R + 1);
  return sizeof(float2) * (L + (xch > stage ? xch : stage));
}
template <int L>
__host__ __device__ constexpr size_t rows_smem_bytes() {
  return rows_smem_bytes_r<L, FftShape<L>::RC>();
}

// The CTA holds rows x0..x0+R-1 (vector v = row x0+v) of a plane after fft_vec; element n = t + T*e of the row
// sits in a[out_slot(e)].  Writes the plane transposed, out[n*L + x0 + v], through a staging tile with pitch
// R+1 so both the register->shared write and the coalesced shared->global read are conflict-free.
template <int L, int R>
__device__ __forceinline__ void store_rows_transposed(const float2 (&a)[FftShape<L>::E], float2* __restrict__ out,
                                                      int x0, int v, int t, float2* stage) {
  constexpr int T = FftShape<L>::T, E = FftShape<L>::E;
  __syncthreads();  // stage aliases the exchange buffers of other warps
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    stage[(t + T * e) * (R + 1) + v] = a[out_slot<L>(e)];
  });
  __syncthreads();
  for (int i = threadIdx.x; i < L * R; i += blockDim.x) {
    const int vv = i % R, n = i / R;
    out[size_t(n) * L + x0 + vv] = stage[n * (R + 1) + vv];
  }
}

// Texture-coordinate emulation for one axis: integer index idx plus fractional base; clamp addressing.
__device__ __forceinline__ void tex_axis(float base, int idx, int extent, int& i0, int& i1, float& w) {
  const float c = float(idx) + base;
  const float tt = c + 0.5f;
  const float xb = tt - 0.5f;
  const float fl = floorf(xb);
  const float fr = xb - fl;
  w = floorf(fr * 256.f + 0.5f) * (1.f / 256.f);
  int i = int(fl);
  i0 = min(max(i, 0), extent - 1);
  i1 = min(max(i + 1, 0), extent - 1);
}

// Modulus replacement amp * exp(i*arg(psi)) (src/SampleKernels.cu:436-450, src/utilitiesKernels.cu:626-631).
// The reference takes arg through atan2; psi/|psi| is the same direction.  psi == 0 maps to phase 0.
__device__ __forceinline__ float2 modulus_replace(float2 psi, float amp) {
  const float m2 = psi.x * psi.x + psi.y * psi.y;
  if (m2 == 0.f) return make_float2(amp, 0.f);
  const float s = amp * rsqrtf(m2);
  return make_float2(psi.x * s, psi.y * s);
}

// constrainPhase (src/SampleKernels.cu:209-215): arg(v) > 0 is clamped to 0 (value becomes |v|, real);
// arg <= 0 is kept.  atan2(+0, x<0) = +pi counts as positive.
__device__ __forceinline__ float2 constrain_phase(float2 v) {
  const bool pos = (v.y > 0.f) || (v.y == 0.f && !signbit(v.y) && v.x < 0.f);
  const float m = sqrtf(v.x * v.x + v.y * v.y);  // branch-free: both results, then a select
  return make_float2(pos ? m : v.x, pos ? 0.f : v.y);
}

__device__ __forceinline__ double warp_reduce_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_reduce_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_reduce_maxf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reductions (blockDim.x a multiple of 32, <= 1024); the result is valid in thread 0.
__device__ __forceinline__ double block_reduce_sum(double v) {
  __shared__ double s[32];
  v = warp_reduce_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? s[l] : 0.0;
  if (w == 0) v = warp_reduce_sum(v);
  return v;
}
// M block-wide sums at once, with the same additions in the same order as M calls of block_reduce_sum but two CTA
// barriers in all; the results are valid in thread 0.
template <int M>
__device__ __forceinline__ void block_reduce_sum_n(double (&v)[M]) {
  __shared__ double s[M][32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int m = 0; m < M; ++m) v[m] = warp_reduce_sum(v[m]);
  __syncthreads();
  if (l == 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) s[m][w] = v[m];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = warp_reduce_sum(threadIdx.x < (blockDim.x >> 5) ? s[m][l] : 0.0);
  }
}
__device__ __forceinline__ double block_reduce_max(double v) {
  __shared__ double s[32];
  v = warp_reduce_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? s[l] : 0.0;
  if (w == 0) v = warp_reduce_max(v);
  return v;
}
__device__ __forceinline__ float block_reduce_maxf(float v) {
  __shared__ float s[32];
  v = warp_reduce_maxf(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? s[l] : 0.f;
  if (w == 0) v = warp_reduce_maxf(v);
  return v;
}

// Max of non-negative doubles: their bit patterns order like unsigned integers.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}

// Streaming accesses (touched once per iteration): cache-streaming policy, evicted first from L1/L2.
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float2* p, float2 v) { __stcs(p, v); }

}  // namespace pty
