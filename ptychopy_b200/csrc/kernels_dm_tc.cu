// DM column pass at 512^2 on the tensor cores (precision=1): the same work item as k_dm_cols (8 adjacent columns of
// one pattern: forward transform along x, modulus step, inverse transform along x; W1 in, W2 out, both row-major), with
// the 32-point stage of each 512-point column transform computed by tcgen05 MMAs.
//
// Column transform (n = s + 32 e, k = k1 + 16 k2, W_L = exp(-2 pi i / L)):
//   X[k1 + 16 k2] = sum_s W32^(s k2) * ( W512^(s k1) * sum_e W16^(e k1) x[s + 32 e] )
// Thread (s, c) of the CTA holds column c at rows s + 32 e in registers (coalesced loads), does the 16-point DFT over
// e and the twiddle in FP32 (fft_core.cuh); the 32-point DFT over s is a GEMM over the CTA's 128 rows m = 8 k1 + c:
// D[m][2 k2 + b] = sum_K A[m][K] B[K][2 k2 + b], K = 2 s + a (re, im interleaved), B the real form of W32^(s k2).
// The inverse transform of the modulus-constrained spectrum runs the other way: its 32-point stage over k2 is the same
// GEMM on the conjugated input (IDFT(D) = conj(DFT(conj(D))), and W32 is symmetric), straight from the accumulator rows
// m = 8 k1 + c; the twiddle conj(W512^(s k1)) follows, rows go through shared memory to the threads (s, c), and the
// 16-point inverse DFT over k1 in registers gives x[s + 32 e], stored to W2.
//
// Operands are FP16 pairs: every GEMM input v, scaled by a power of two per column so that |v| < 2^15, is
// v_hi + v_lo with v_hi = fp16(v) and v_lo = fp16(v - v_hi) (22 significant bits), the DFT matrix likewise, and
// D = A_hi B_hi + A_lo B_hi + A_hi B_lo accumulates in FP32 in tensor memory (the dropped A_lo B_lo is ~2^-22 of the
// result): FP32-level accuracy.  Shared-memory operands use the canonical K-major no-swizzle layout (8-row x 16-byte
// core matrices); the rows of one store instruction fall in distinct banks.  One thread issues the MMAs and commits
// to an mbarrier; every wait is bounded (on expiry a device flag is set, the CTA stops and frees its tensor memory).
// No counterpart in the reference (cuFFT with callbacks, src/SampleKernels.cu:416-490).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels.h"
#include "umma.cuh"

namespace pty {
namespace {

constexpr int TL = 512, TCB = 8, TTHREADS = 256, TE = 16, TS = 32;
constexpr int T_PITCH = 136;                               // float2 per s-row of the transpose buffer (conflict-free)
constexpr int A_SPLIT = 16384;                             // bytes of one FP16 operand tile (128 x 64)
constexpr int REGION = T_PITCH * TS * 8;                   // A (hi, lo) aliased with the transpose buffer
constexpr int OFF_B = REGION;                              // B hi, lo (64 x 64 FP16 each)
constexpr int B_SPLIT = 8192;
constexpr int OFF_TW = OFF_B + 2 * B_SPLIT;                // stage-1 twiddles [k1][s]
constexpr int OFF_SC = OFF_TW + TL * 8;                    // per-column maxima (2 x 8 ints)
constexpr int OFF_BAR = OFF_SC + 64;
constexpr int TC_SMEM = OFF_BAR + 16;
constexpr uint32_t A_LBO = 2048, B_LBO = 1024, TMEM_COLS = 64;
static_assert(2 * A_SPLIT <= REGION, "operand tile fits the shared region");

__device__ __forceinline__ uint32_t a_off(int m, int k) {
  return uint32_t((k >> 3) * A_LBO + (m >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint32_t b_off(int n, int k) {
  return uint32_t((k >> 3) * B_LBO + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

// This thread's 32 accumulator columns (16 complex values, re / im interleaved).
__device__ __forceinline__ void tmem_row32(uint32_t taddr, float2 (&v)[16]) {
  float lo[16], hi[16];
  tmem_ld16(taddr, lo);
  tmem_ld16(taddr + 16, hi);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = make_float2(lo[2 * j], lo[2 * j + 1]);
    v[8 + j] = make_float2(hi[2 * j], hi[2 * j + 1]);
  }
}

// Power-of-two scale that brings a maximum magnitude m below 2^15 (|fp16| < 65504), and its inverse.
__device__ __forceinline__ void pow2_scale(float m, float& sc, float& inv) {
  int k = 0;
  if (m > 0.f) {
    const int e = int((__float_as_uint(m) >> 23) & 0xffu) - 127;  // m in [2^e, 2^(e+1)) (subnormals: e = -127)
    k = 14 - e;
    k = k > 126 ? 126 : (k < -126 ? -126 : k);
  }
  sc = __uint_as_float(uint32_t(k + 127) << 23);
  inv = __uint_as_float(uint32_t(127 - k) << 23);
}

__device__ __forceinline__ void split_f16(float2 v, __half2& hi, __half2& lo) {
  hi = __floats2half2_rn(v.x, v.y);
  const float2 h = __half22float2(hi);
  lo = __floats2half2_rn(v.x - h.x, v.y - h.y);
}

// Maximum of |re|, |im| over the 8 columns' threads: a warp holds 4 threads per column (lanes c, c+8, c+16, c+24).
__device__ __forceinline__ void column_max(float m, int c, int* s_max) {
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 8));
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
  if ((threadIdx.x & 31) < 8) atomicMax(s_max + c, __float_as_int(m));
}

}  // namespace

__global__ void __launch_bounds__(TTHREADS, 3) k_dm_cols_tc(const DMBuffers b, const DMWave w) {
  constexpr int NB = TL / TCB;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_skip;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t a_hi = sbase, a_lo = sbase + A_SPLIT, bh = sbase + OFF_B, bl = sbase + OFF_B + B_SPLIT;
  const uint32_t bar = sbase + OFF_BAR, idesc = umma_idesc_f16(128, 64);
  float2* tw = reinterpret_cast<float2*>(smem + OFF_TW);
  float2* T = reinterpret_cast<float2*>(smem);
  int* s_max = reinterpret_cast<int*>(smem + OFF_SC);  // [0..7] forward, [8..15] inverse
  if (tid == 0) s_skip = *reinterpret_cast<volatile int*>(b.err);
  __syncthreads();
  if (s_skip) return;

  // B = the real form of W32^(s k2), split into FP16 hi / lo: B[2s + a][2 k2 + bb]
  for (int q = tid; q < 64 * 64; q += TTHREADS) {
    const int n = q >> 6, k = q & 63;  // n = 2 k2 + bb, k = 2 s + a
    const int k2 = n >> 1, bb = n & 1, s = k >> 1, a = k & 1;
    float sn, cs;
    sincospif(-2.f * float((s * k2) & 31) / 32.f, &sn, &cs);  // W32^(s k2) = cs + i sn
    const float v = bb == 0 ? (a == 0 ? cs : -sn) : (a == 0 ? sn : cs);
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    *reinterpret_cast<__half*>(smem + OFF_B + b_off(n, k)) = h;
    *reinterpret_cast<__half*>(smem + OFF_B + B_SPLIT + b_off(n, k)) = l;
  }
  for (int i = tid; i < TL; i += TTHREADS) tw[i] = b.tw[i];
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  // accumulator lanes of this warp (32 rows) and its half of the 64 columns
  const uint32_t trow = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t((warp >> 2) * 32);
  uint32_t phase = 0;

  // the 12 MMAs of one GEMM (K = 64 in four steps, three products each), then a bounded wait for all of them
  auto gemm = [&]() -> bool {
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint64_t dah = umma_desc(a_hi + uint32_t(j * 2 * A_LBO), A_LBO, 128);
        const uint64_t dal = umma_desc(a_lo + uint32_t(j * 2 * A_LBO), A_LBO, 128);
        const uint64_t dbh = umma_desc(bh + uint32_t(j * 2 * B_LBO), B_LBO, 128);
        const uint64_t dbl = umma_desc(bl + uint32_t(j * 2 * B_LBO), B_LBO, 128);
        umma_bf16(tmem, dah, dbh, idesc, j > 0);
        umma_bf16(tmem, dal, dbh, idesc, true);
        umma_bf16(tmem, dah, dbl, idesc, true);
      }
      umma_commit(bar);
    }
    const bool done = mbar_wait(bar, phase);
    if (!done && tid == 0) {
      atomicCAS(b.err, 0, 1);
      mbar_wait(bar, phase);  // a second bounded wait for the MMAs in flight before the CTA frees tensor memory
    }
    phase ^= 1u;
    const bool all = !__syncthreads_or(!done);
    tc_fence_after();
    return all;
  };

  const int c = tid & 7, s = tid >> 3;         // load / store thread: column c, rows s + 32 e
  const int em = (warp & 3) * 32 + lane;       // accumulator row m = 8 k1 + c of this thread
  const int ek1 = em >> 3, ec = em & 7, eh = warp >> 2;
  constexpr float nrm = 1.0f / float(TL * TL);
  for (int item = blockIdx.x; item < NB * w.count; item += gridDim.x) {
    const int p = w.slot_pat[item / NB], slot = item / NB, col0 = (item % NB) * TCB;
    if (tid < 16) s_max[tid] = 0;
    // ---- forward: 16-point DFT over e in registers, twiddle, split into A rows (k1, c), K = 2 s
    float2 a[TE];
    const float2* w1 = b.W1 + size_t(slot) * TL * TL + col0 + c;
#pragma unroll
    for (int e = 0; e < TE; ++e) a[e] = w1[size_t(s + TS * e) * TL];
    dft_reg<false>(a);
    float mx = 0.f;
    static_for<0, TE>([&](auto kc) {
      constexpr int k1 = decltype(kc)::value, q = bitrev(k1, TE);
      if constexpr (k1 > 0) a[q] = cmul(a[q], tw[k1 * TS + s]);
      mx = fmaxf(mx, fmaxf(fabsf(a[q].x), fabsf(a[q].y)));
    });
    __syncthreads();  // s_max cleared; the previous item's readers of T are done
    column_max(mx, c, s_max);
    __syncthreads();
    float sc, inv;
    pow2_scale(__int_as_float(s_max[c]), sc, inv);
    static_for<0, TE>([&](auto kc) {
      constexpr int k1 = decltype(kc)::value;
      __half2 hi, lo;
      split_f16(cscale(a[bitrev(k1, TE)], sc), hi, lo);
      const uint32_t off = a_off(8 * k1 + c, 2 * s);
      *reinterpret_cast<__half2*>(smem + off) = hi;
      *reinterpret_cast<__half2*>(smem + A_SPLIT + off) = lo;
    });
    // the amplitudes of this thread's spectrum rows, loaded while the GEMM runs: row kx = k1 + 16 k2, column c
    float am[16];
    {
      const float* A = b.amp + size_t(p) * TL * TL + col0 + ec;
#pragma unroll
      for (int j = 0; j < 16; ++j) am[j] = ld_stream(A + size_t(ek1 + 16 * (16 * eh + j)) * TL);
    }
    if (!gemm()) break;
    // ---- spectrum rows (k1, c), k2 = 16 eh .. 16 eh + 15: unscale, modulus step, D = Psi' - Psi / N^2
    float2 d[16];
    {
      float2 v[16];
      tmem_row32(trow, v);
      float sci, invi;
      pow2_scale(__int_as_float(s_max[ec]), sci, invi);
      float m2 = 0.f;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float2 ps = cscale(v[j], invi);
        const float2 rep = modulus_replace(ps, am[j] * nrm);
        d[j] = make_float2(rep.x - ps.x * nrm, rep.y - ps.y * nrm);
        m2 = fmaxf(m2, fmaxf(fabsf(d[j].x), fabsf(d[j].y)));
      }
      tc_fence_before();
      column_max(m2, ec, s_max + 8);
    }
    __syncthreads();
    {
      float sc2, inv2;
      pow2_scale(__int_as_float(s_max[8 + ec]), sc2, inv2);
#pragma unroll
      for (int q = 0; q < 4; ++q) {  // K chunk 4 eh + q: k2 = 16 eh + 4 q .. + 3, conjugated
        __half2 hi[4], lo[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float2 v = d[4 * q + u];
          split_f16(make_float2(v.x * sc2, -v.y * sc2), hi[u], lo[u]);
        }
        const uint32_t off = a_off(em, 8 * (4 * eh + q));
        *reinterpret_cast<uint4*>(smem + off) = *reinterpret_cast<uint4*>(hi);
        *reinterpret_cast<uint4*>(smem + A_SPLIT + off) = *reinterpret_cast<uint4*>(lo);
      }
    }
    if (!gemm()) break;
    // ---- inverse: rows (k1, c) hold G[s] for s = 16 eh .. + 15; conj, unscale, twiddle, to T[s][k1][c]
    {
      float2 v[16];
      tmem_row32(trow, v);
      float sc2, inv2;
      pow2_scale(__int_as_float(s_max[8 + ec]), sc2, inv2);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int ss = 16 * eh + j;
        float2 g = make_float2(v[j].x * inv2, -v[j].y * inv2);
        if (ek1) g = cmulc(g, tw[ek1 * TS + ss]);  // * conj(W512^(s k1))
        T[ss * T_PITCH + ek1 * 8 + ec] = g;
      }
      tc_fence_before();
    }
    __syncthreads();
    // ---- 16-point inverse DFT over k1 in registers: x[s + 32 e] of column c, to W2
#pragma unroll
    for (int k1 = 0; k1 < TE; ++k1) a[k1] = T[s * T_PITCH + k1 * 8 + c];
    dft_reg<true>(a);
    float2* w2 = b.W2 + size_t(slot) * TL * TL + col0 + c;
    static_for<0, TE>([&](auto ec) {
      constexpr int e = decltype(ec)::value;
      w2[size_t(s + TS * e) * TL] = a[bitrev(e, TE)];
    });
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

cudaError_t dm_cols_tc_prepare() {
  return cudaFuncSetAttribute(k_dm_cols_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
}

// Resident CTA slots of the tensor-core column kernel: 3 per SM (80 registers x 256 threads, 55 KB of shared memory
// and 64 tensor-memory columns each).
constexpr int TC_CTAS_PER_SM = 3;
static int dm_cols_tc_slots() {
  static const int s = [] {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return TC_CTAS_PER_SM * (sms > 0 ? sms : 1);
  }();
  return s;
}

cudaError_t dm_cols_tc(const DMBuffers& b, const DMWave& w, cudaStream_t st) {
  if (b.N != TL || !b.err) return cudaErrorInvalidValue;
  const int items = (TL / TCB) * w.count;
  k_dm_cols_tc<<<std::min(dm_cols_tc_slots(), items), TTHREADS, TC_SMEM, st>>>(b, w);
  return cudaGetLastError();
}

}  // namespace pty
