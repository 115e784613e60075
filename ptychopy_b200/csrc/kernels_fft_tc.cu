// Mixed-precision 2-D FFT on the tensor cores: every 256-point line transform is two radix-16 DFT stages computed as
// tcgen05 GEMMs with split-BF16 operands and FP32 accumulation in TMEM (the engine's FP32 FFT in fft_core.cuh is
// the reference path; this one exists to measure what the tensor cores give at which error).
//
// Line transform (n = 16 n1 + n2, k = k1 + 16 k2):
//   stage 1   Y[k1][n2] = sum_n1 W16^(n1 k1) x[16 n1 + n2]                    GEMM, M = (line, n2), K = n1
//   twiddle   Y[k1][n2] *= W256^(n2 k1)                                      FP32
//   stage 2   X[k1 + 16 k2] = sum_n2 W16^(n2 k2) Y[k1][n2]                    GEMM, M = (line, k1), K = n2
// Complex products in real arithmetic: [Re y, Im y] = [Re x, Im x] [[Re F, Im F], [-Im F, Re F]] (K = 32, N = 32).
// Split BF16: x = x_hi + x_lo, F = F_hi + F_lo (x_lo = bf16(x - x_hi)), and the three products x_hi F_hi + x_lo F_hi
// + x_hi F_lo are one GEMM over the concatenated K = 96: A = [x_hi | x_lo | x_hi], B = [F_hi; F_hi; F_lo]; the
// dropped x_lo F_lo term is ~2^-16 of the result.
//
// A CTA (128 threads, one TMEM accumulator of 32 columns) takes 8 lines at a time: it loads them coalesced into
// shared memory, thread m builds A row m, one thread issues the six K = 16 MMAs of a stage and commits to an
// mbarrier (bounded wait), thread m reads accumulator row m back with tcgen05.ld.  The pass writes its output
// transposed (line j of plane b becomes column j) through shared memory in 64-byte segments, so two passes give the
// 2-D transform in natural order.  No counterpart in the reference (cuFFT, src/CudaFFTPlan.cpp:91-101).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "../../include/ptychopy_b200.h"
#include "umma.cuh"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

namespace {

constexpr int FT_N = 256, FT_LINES = 8, FT_THREADS = 128, FT_K = 96, FT_NN = 32;
// shared memory: line buffer (8 x 256 complex FP32, also the output staging), A (128 x 96 BF16), B (32 x 96 BF16),
// twiddles W256^e (256 complex), the mbarrier
constexpr int FT_OFF_A = FT_LINES * FT_N * 8;            // 16 KB
constexpr int FT_OFF_B = FT_OFF_A + 128 * FT_K * 2;      // + 24 KB
constexpr int FT_OFF_TW = FT_OFF_B + FT_NN * FT_K * 2;   // + 6 KB
constexpr int FT_OFF_BAR = FT_OFF_TW + FT_N * 8;         // + 2 KB
constexpr int FT_SMEM = FT_OFF_BAR + 64;

// K-major no-swizzle core-matrix offset (bytes) of element (row r, k) in an operand of `rows` rows
__device__ __forceinline__ uint32_t op_off(int r, int k, int rows) {
  return uint32_t(((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// One pass: for each group of 8 lines (plane b, lines j0..j0+7 of `in`), the 256-point DFT of every line, written
// transposed into `out` (out[b][k][j] = X_j[k]).  sign = -1 forward, +1 inverse (unnormalised).
__global__ void __launch_bounds__(FT_THREADS, 1)
    k_fft_tc_pass(const float2* __restrict__ in, float2* __restrict__ out, int groups, float sign, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_skip;
  const int tid = threadIdx.x, warp = tid >> 5;
  float2* lines = reinterpret_cast<float2*>(smem);
  const float2* tw = reinterpret_cast<const float2*>(smem + FT_OFF_TW);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t a_s = sbase + FT_OFF_A, b_s = sbase + FT_OFF_B, bar = sbase + FT_OFF_BAR;
  const uint32_t idesc = umma_idesc_bf16(128, FT_NN);
  if (tid == 0) s_skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (s_skip || int(blockIdx.x) >= groups) return;

  // B = [F_hi; F_hi; F_lo] of the real-expanded 16-point DFT (rows: Re k1 then Im k1; K: Re n1 then Im n1)
  for (int q = tid; q < FT_NN * 32; q += FT_THREADS) {
    const int nn = q / 32, t = q % 32;
    const int k1 = nn & 15, n1 = t & 15;
    float s, c;
    sincospif(sign * 2.f * float((n1 * k1) & 15) / 16.f, &s, &c);  // F = e^{sign 2 pi i n1 k1 / 16}
    float v;
    if (nn < 16)
      v = t < 16 ? c : -s;  // Re y: Re F Re x - Im F Im x
    else
      v = t < 16 ? s : c;   // Im y: Im F Re x + Re F Im x
    __nv_bfloat16 hi, lo;
    split_bf16(v, hi, lo);
    __nv_bfloat16* B = reinterpret_cast<__nv_bfloat16*>(smem + FT_OFF_B);
    B[op_off(nn, t, FT_NN) / 2] = hi;
    B[op_off(nn, 32 + t, FT_NN) / 2] = hi;
    B[op_off(nn, 64 + t, FT_NN) / 2] = lo;
  }
  for (int e = tid; e < FT_N; e += FT_THREADS) {
    float s, c;
    sincospif(sign * 2.f * float(e) / float(FT_N), &s, &c);
    reinterpret_cast<float2*>(smem + FT_OFF_TW)[e] = make_float2(c, s);
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem, trow = tmem + (uint32_t(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  __nv_bfloat16* A = reinterpret_cast<__nv_bfloat16*>(smem + FT_OFF_A);

  // one GEMM stage: fence the generic A writes to the async proxy, six MMAs by one thread, bounded wait
  auto gemm = [&]() -> bool {
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < FT_K / 16; ++s)
        umma_bf16(tmem, umma_desc(a_s + uint32_t(s * 2 * 16 * 128), 16 * 128, 128),
                  umma_desc(b_s + uint32_t(s * 2 * 4 * 128), 4 * 128, 128), idesc, s > 0);
      umma_commit(bar);
    }
    const bool done = mbar_wait(bar, phase);
    phase ^= 1u;
    if (!done && tid == 0) atomicCAS(err, 0, 1);
    const bool all = !__syncthreads_or(!done);
    tc_fence_after();
    return all;
  };
  auto read_row = [&](float2 (&y)[16]) {
#pragma unroll
    for (int c8 = 0; c8 < 4; ++c8) {
      float v[8];
      tmem_ld8(trow + uint32_t(c8 * 8), v);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int col = c8 * 8 + e;
        if (col < 16)
          y[col].x = v[e];
        else
          y[col - 16].y = v[e];
      }
    }
  };

  const int li = tid >> 4, sub = tid & 15;  // A row m = tid: line li, sub-index n2 (stage 1) or k1 (stage 2)
  for (int g = blockIdx.x; g < groups && ok; g += gridDim.x) {
    const int b = g / (FT_N / FT_LINES), j0 = (g % (FT_N / FT_LINES)) * FT_LINES;
    const float2* src = in + (size_t(b) * FT_N + j0) * FT_N;
    // the 8 input lines (contiguous rows of the plane)
    for (int q = tid; q < FT_LINES * FT_N / 2; q += FT_THREADS)
      reinterpret_cast<float4*>(lines)[q] = reinterpret_cast<const float4*>(src)[q];
    __syncthreads();
    // stage 1: A row (li, n2) = [hi | lo | hi] of x[16 n1 + n2], Re then Im
    {
      __align__(16) __nv_bfloat16 hi[32], lo[32];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float2 x = lines[li * FT_N + 16 * n1 + sub];
        split_bf16(x.x, hi[n1], lo[n1]);
        split_bf16(x.y, hi[16 + n1], lo[16 + n1]);
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const uint4 h = reinterpret_cast<const uint4*>(hi)[c], l = reinterpret_cast<const uint4*>(lo)[c];
        *reinterpret_cast<uint4*>(smem + FT_OFF_A + op_off(tid, 8 * c, 128)) = h;
        *reinterpret_cast<uint4*>(smem + FT_OFF_A + op_off(tid, 32 + 8 * c, 128)) = l;
        *reinterpret_cast<uint4*>(smem + FT_OFF_A + op_off(tid, 64 + 8 * c, 128)) = h;
      }
    }
    if (!gemm()) {
      ok = false;
      break;
    }
    // twiddle, and A row (li, k1) of stage 2 receives Y[k1][n2] at K = n2 (this thread's n2 = sub)
    {
      float2 y[16];
      read_row(y);
      __syncthreads();  // every thread has read stage 1 before A is rewritten
#pragma unroll
      for (int k1 = 0; k1 < 16; ++k1) {
        const float2 w = tw[(sub * k1) & (FT_N - 1)];
        const float2 v = make_float2(y[k1].x * w.x - y[k1].y * w.y, y[k1].x * w.y + y[k1].y * w.x);
        __nv_bfloat16 rh, rl, ih, il;
        split_bf16(v.x, rh, rl);
        split_bf16(v.y, ih, il);
        const int r = li * 16 + k1;
        A[op_off(r, sub, 128) / 2] = rh;
        A[op_off(r, 16 + sub, 128) / 2] = ih;
        A[op_off(r, 32 + sub, 128) / 2] = rl;
        A[op_off(r, 48 + sub, 128) / 2] = il;
        A[op_off(r, 64 + sub, 128) / 2] = rh;
        A[op_off(r, 80 + sub, 128) / 2] = ih;
      }
    }
    tc_fence_before();
    if (!gemm()) {
      ok = false;
      break;
    }
    // X[k1 + 16 k2] of line li (this thread's k1 = sub) into the line buffer, then transposed coalesced stores
    {
      float2 z[16];
      read_row(z);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) lines[li * FT_N + sub + 16 * k2] = z[k2];
    }
    tc_fence_before();
    __syncthreads();
    float2* dst = out + size_t(b) * FT_N * FT_N + j0;
    for (int q = tid; q < FT_N * FT_LINES; q += FT_THREADS) {
      const int k = q / FT_LINES, l = q % FT_LINES;
      dst[size_t(k) * FT_N + l] = lines[l * FT_N + k];
    }
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(32) : "memory");
}

int fail(const std::string& msg, int code) {
  set_last_error(msg);
  return code;
}

constexpr int FT_MAX_DEV = 64;
std::atomic<int> g_fft_tc_sms[FT_MAX_DEV];  // SM count per device the kernel was prepared on (0: not yet)

int current_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= FT_MAX_DEV) return 0;
  return g_fft_tc_sms[dev].load();
}

}  // namespace

cudaError_t fft2_tc_prepare() {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess && (dev < 0 || dev >= FT_MAX_DEV)) e = cudaErrorInvalidDevice;
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_fft_tc_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, FT_SMEM);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) g_fft_tc_sms[dev].store(sms);
  return e;
}

cudaError_t fft2_tc(float2* data, float2* work, int batch, int N, bool inverse, int* err, cudaStream_t st) {
  const int sms = current_sms();
  if (N != FT_N || batch < 1 || sms == 0) return cudaErrorInvalidValue;
  const int groups = batch * (FT_N / FT_LINES);
  const int grid = groups < 4 * sms ? groups : 4 * sms;  // 4 CTAs per SM (48 KB, 32 TMEM columns)
  const float sign = inverse ? 1.f : -1.f;
  k_fft_tc_pass<<<grid, FT_THREADS, FT_SMEM, st>>>(data, work, groups, sign, err);
  k_fft_tc_pass<<<grid, FT_THREADS, FT_SMEM, st>>>(work, data, groups, sign, err);
  return cudaGetLastError();
}

}  // namespace pty

using namespace pty;

extern "C" int pty_fft2_tc(void* data, void* work, int batch, int N, int inverse, int* err, void* stream) {
  if (!data || !work || !err || batch < 1 || N != FT_N)
    return fail("pty_fft2_tc: bad argument (N must be 256)", PTY_ERR_INVALID);
  cudaError_t e = current_sms() ? cudaSuccess : fft2_tc_prepare();
  if (e == cudaSuccess)
    e = fft2_tc(static_cast<float2*>(data), static_cast<float2*>(work), batch, N, inverse != 0, err,
                static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return fail(std::string("pty_fft2_tc: ") + cudaGetErrorString(e), PTY_ERR_CUDA);
  return PTY_OK;
}
