// Row-transform passes of the batched 2-D FFT with fused loads and stores, launched with programmatic dependent
// launch.  Header-only templates, shared by the MLs default path (kernels_mls_var.cu) and the ePIE kernel chain
// (kernels_epie_chain.cu).
#pragma once
#include <cuda_runtime.h>

#include <utility>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "pdl.cuh"

namespace pty {

// ---- FFT passes with fused loads and stores -------------------------------------------------------------------
// One row-transform pass of the batched 2-D FFT (the k_fft_rows_t scheme: R rows per CTA, transposed store) with a
// prologue that produces each loaded element (plane b, row x, column y) and an epilogue that maps each stored element
// (plane b, row x, column y of the natural layout after the second pass) and may accumulate per-plane sums, finished
// once per CTA.  The first pass of a 2-D transform takes a prologue and stores plainly into the transposed work
// plane; the second loads plainly and takes an epilogue.
struct ProLoad {
  const float2* in;
  __device__ float2 operator()(int b, int x, int y, int L) const { return in[(size_t(b) * L + x) * L + y]; }
};
struct EpiStore {
  __device__ float2 operator()(int, int, int, int, float2 v) { return v; }
  __device__ void finish(int) {}
};

// Rows x0 .. x0 + RC - 1 of plane b: load through pro, transform, store transposed through epi.  s_tw holds the
// twiddles, s_x the exchange / staging buffers (rows_smem_bytes<L> with s_tw); starts with a CTA barrier so that
// calls may follow each other.
template <int L, bool INV, class Pro, class Epi, int R = FftShape<L>::RC>
__device__ __forceinline__ void fftx_rows(float2* out, const float2* s_tw, float2* s_x, int b, int x0, const Pro& pro,
                                          Epi& epi) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  __syncthreads();
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = pro(b, x0 + v, t + T * e, L);
  fft_vec<L, INV>(a, t, s_x + v * S::XCH, s_tw);
  __syncthreads();  // the staging tile aliases the exchange buffers of other warps
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    s_x[(t + T * e) * (R + 1) + v] = a[out_slot<L>(e)];
  });
  __syncthreads();
  float2* o = out + size_t(b) * L * L;
  for (int i = threadIdx.x; i < L * R; i += blockDim.x) {
    const int vv = i % R, n = i / R;
    o[size_t(n) * L + x0 + vv] = epi(b, n, x0 + vv, L, s_x[n * (R + 1) + vv]);
  }
}

// R rows per CTA (R x T threads): the default FftShape<L>::RC fills 256 threads; fewer rows spread a plane's rows over
// more CTAs (and SMs)
template <int L, bool INV, class Pro, class Epi, int R = FftShape<L>::RC>
__global__ void __launch_bounds__(R * FftShape<L>::T) k_fftx_pass(float2* __restrict__ out,
                                                                  const float2* __restrict__ g_tw, Pro pro, Epi epi) {
  static_assert(R * FftShape<L>::T % 32 == 0, "whole warps per CTA");
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  load_twiddles<L>(smem, g_tw);  // a table written before any transform runs: loaded before the wait
  pdl_enter();
  fftx_rows<L, INV, Pro, Epi, R>(out, smem, smem + L, blockIdx.y, blockIdx.x * R, pro, epi);
  epi.finish(blockIdx.y);
}

template <int L, bool INV, int R = FftShape<L>::RC, class Pro, class Epi>
inline cudaError_t launch_fftx(float2* out, const float2* tw, int batch, Pro pro, Epi epi, cudaStream_t st) {
  constexpr int NT = R * FftShape<L>::T;
  const size_t smem = rows_smem_bytes_r<L, R>();
  cudaError_t e = cudaFuncSetAttribute(k_fftx_pass<L, INV, Pro, Epi, R>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  return launch_pdl(k_fftx_pass<L, INV, Pro, Epi, R>, dim3(L / R, batch), NT, smem, st, out, tw, pro, epi);
}

// 2-D transform data-in (through pro) -> work (transposed) -> out (through epi); RMAX caps the rows per CTA, which
// stay at least a whole warp's worth (32 / T rows: the row transforms use warp-wide shuffles and syncs)
template <bool INV, class Pro, class Epi, int RMAX = 1024>
inline cudaError_t fftx2(int N, float2* work, float2* out, const float2* tw, int batch, Pro pro, Epi epi, cudaStream_t st) {
  cudaError_t e;
#define PTY_FFTX(L)                                                                                          \
  case L: {                                                                                                  \
    constexpr int RC = FftShape<L>::RC < RMAX ? FftShape<L>::RC : RMAX, RW = 32 / FftShape<L>::T;           \
    constexpr int R = RC > RW ? RC : RW;                                                                     \
    if ((e = launch_fftx<L, INV, R>(work, tw, batch, pro, EpiStore{}, st)) != cudaSuccess) return e;         \
    return launch_fftx<L, INV, R>(out, tw, batch, ProLoad{work}, epi, st);                                   \
  }
  switch (N) {
    PTY_FFTX(32)
    PTY_FFTX(64)
    PTY_FFTX(128)
    PTY_FFTX(256)
    PTY_FFTX(512)
    default:
      return cudaErrorInvalidValue;
  }
#undef PTY_FFTX
}

// ---- whole 2-D transforms inside one thread-block cluster ------------------------------------------------------
// A cluster of C CTAs owns one plane: CTA `rank` transforms row blocks rank, rank + C, ... of each pass, and the
// passes hand the plane to each other through global memory (L2) across cluster barriers, so that a chain of 2-D
// transforms with pointwise steps between them runs as one launch.
// barrier.cluster.arrive (release) + wait (acquire): cluster-scope ordering of the global-memory hand-offs.
__device__ __forceinline__ void cluster_sync_acqrel() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// in (through pro) -> work (transposed) -> out (through epi); ends with a cluster barrier, so out is complete for
// every CTA of the cluster on return
template <int L, bool INV, class Pro, class Epi>
__device__ __forceinline__ void fftx2_cluster(float2* work, float2* out, int b, int rank, int C, const float2* s_tw,
                                              float2* s_x, const Pro& pro, Epi epi) {
  constexpr int R = FftShape<L>::RC;
  EpiStore plain;
  for (int x0 = rank * R; x0 < L; x0 += C * R) fftx_rows<L, INV>(work, s_tw, s_x, b, x0, pro, plain);
  cluster_sync_acqrel();
  const ProLoad lw{work};
  for (int x0 = rank * R; x0 < L; x0 += C * R) fftx_rows<L, INV>(out, s_tw, s_x, b, x0, lw, epi);
  epi.finish(b);
  cluster_sync_acqrel();
}

// The shared-memory size and the opt-in to 16-CTA clusters of a cluster kernel, on the current device (function
// attributes are per device: set them on every device that launches the kernel)
template <class Kern>
inline cudaError_t set_cluster_attributes(Kern* kernel, size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

// Largest cluster of `kernel` (at most one CTA per row block of a plane and at most 16, the largest size, opted
// into) of which one fits on the device; 0 if none.  Sets the kernel's attributes on the current device.
template <class Kern>
inline int fit_cluster(Kern* kernel, int row_blocks, int threads, size_t smem) {
  if (set_cluster_attributes(kernel, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  for (int C = row_blocks < 16 ? row_blocks : 16; C >= 1; C /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) == cudaSuccess && n >= 1) return C;
    cudaGetLastError();
  }
  return 0;
}

// Launch of a grid of (C, planes) CTAs in clusters of C along x, with programmatic stream serialisation
template <typename... KArgs, typename... Args>
inline cudaError_t launch_cluster_pdl(void (*kernel)(KArgs...), int C, int planes, int threads, size_t smem,
                                      cudaStream_t st, Args&&... args) {
  if (C < 1) return cudaErrorInvalidConfiguration;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, planes);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

}  // namespace pty
