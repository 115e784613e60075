// Tensor-core (tcgen05) inference path of the warm-start network: 3x3 convolutions as implicit GEMMs with BF16
// activations and weights and FP32 accumulation in tensor memory, plus the NHWC pooling / upsampling between them.
//
// GEMM view of one layer: D[m][n] = sum_k A[m][k] B[n][k], m = output pixel (image-major, NHWC order), n = output
// channel, k = tap * Cin + ci (tap = 3 * (dy + 1) + (dx + 1)), A[m][k] = x[pixel m shifted by the tap][ci] (zero
// outside the image), B[n][k] = w[n][ci][tap].  A CTA owns 128 consecutive pixels and all N (<= 256) channels: the
// accumulator is 128 lanes x N columns of FP32 in TMEM.  K runs in stages of 64: the 128 threads stage the im2col
// rows of A with 16-byte cp.async (zero-fill outside the image) and one thread bulk-copies the pre-packed B slice
// (cp.async.bulk completing on an mbarrier), both in the canonical
// K-major no-swizzle layout (8-row x 16-byte core matrices; SBO = 128 B between 8-row groups, LBO = one K-chunk
// block between the two 8-element halves of a K=16 slice); one thread issues the stage's tcgen05.mma (M=128, K=16)
// and a tcgen05.commit to the stage buffer's mbarrier, so the next stage's loads overlap the tensor core.  Every
// mbarrier wait is bounded; on a timeout the kernel records an error code and leaves.  The epilogue reads TMEM with
// tcgen05.ld (warp w: lanes 32w..32w+31), adds the bias, applies ReLU and stores NHWC BF16 (or NCHW FP32 for the
// output layer).  No counterpart in the reference; the C ABI is in include/ptychopy_b200.h.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "../../include/ptychopy_b200.h"
#include "kernels_epie.h"
#include "umma.cuh"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

namespace {

constexpr int TC_M = 128;       // pixels per CTA (MMA M)
constexpr int TC_KC = 64;       // K per stage
constexpr int TC_THREADS = 128;
constexpr int TC_MAX_N = 256;

// 16-byte copy global -> shared for the im2col rows, allocating in L1 (ca): the nine taps (and the four readers of an
// upsampled pixel) re-read the same input lines.  src-size 0 writes 16 zero bytes.
__device__ __forceinline__ void cp_async16_cg(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16_l1(uint32_t dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared memory of one CTA: two stage buffers (A 128 x 64 BF16, then B Npad x 64 BF16) and two mbarriers.  The
// stage size follows the layer's Npad, so thin layers fit more CTAs per SM (TMEM: ncols x CTAs <= 512 columns).
struct TcSmem {
  static constexpr int A_BYTES = TC_M * TC_KC * 2;  // 16 KB
  __host__ __device__ static constexpr int stage(int Npad) { return A_BYTES + Npad * TC_KC * 2; }
  __host__ __device__ static constexpr int total(int Npad) { return 2 * stage(Npad) + 64; }
};

// err: set to a non-zero code on a wait timeout.  Persistent and software-pipelined: CTA b walks the work items i = 0, 1, ... (tile b + (i / nstages) * gridDim.x,
// K stage i % nstages).  Item i's operands are loaded into buffer i & 1 during iteration i - 1; in iteration i one
// thread issues its MMAs and commits them to mbarrier i & 1, then all threads prefetch item i + 1 into the other
// buffer once item i - 1's MMAs (its last reader) have completed, and after a tile's last stage the epilogue waits for
// the commit, reads the accumulator from TMEM and stores the tile.  Each barrier has at most one commit outstanding.
// Pixel of GEMM row r of a tile.  Natural order (consecutive pixels) unless the output is pooled: then each warp
// owns a 2-row x 16-column block (lane l: row 2 rp + l / 16, column 16 cb + l % 16), so the four pixels of a 2x2
// pooling window are lanes l, l ^ 1, l ^ 16, l ^ 17 of one warp.
__device__ __forceinline__ bool tc_pixel(long long tile, int r, int H, int W, long long Mtot, bool pooled, int& b,
                                         int& i, int& j) {
  if (!pooled) {
    const long long m = tile * TC_M + r;
    if (m >= Mtot) return false;
    const long long HW = (long long)H * W;
    b = int(m / HW);
    const int p = int(m - (long long)b * HW);
    i = p / W;
    j = p - i * W;
    return true;
  }
  const int cbs = W / 16, units_img = (H / 2) * cbs;
  const long long u = tile * (TC_M / 32) + (r >> 5);
  if (u >= Mtot / 32) return false;
  const int l = r & 31;
  b = int(u / units_img);
  const int rem = int(u - (long long)b * units_img), rp = rem / cbs, cb = rem - rp * cbs;
  i = 2 * rp + (l >> 4);
  j = 16 * cb + (l & 15);
  return true;
}

// in_mode 0: x NHWC BF16 (H x W x Cin); 1: x NHWC BF16 of H/2 x W/2, read 2x nearest-upsampled; 2: x FP32 amplitudes
// (B x H x W, Cin = 1) read as in_scale * log1p(amp) with the zero frequency moved to the centre.
// out_mode 0: y NHWC BF16 (Cout channels); 1: y NCHW FP32; 2: y NHWC BF16 2x2-average-pooled (H/2 x W/2).
__global__ void __launch_bounds__(TC_THREADS, 5)  // 5 CTAs per SM for the narrow layers (<= 96 registers)
    k_conv_tc(const void* __restrict__ x, const __nv_bfloat16* __restrict__ wpk, const float* __restrict__ bias,
              void* __restrict__ y, int B, int H, int W, int Cin, int Cout, int Npad, int Kp, int relu, int in_mode,
              int out_mode, float in_scale, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_skip;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  const int STAGE = TcSmem::stage(Npad);
  // bar0/bar1: MMAs of the buffer's item done (tcgen05.commit); full0/full1: the buffer's weight slice has landed
  const uint32_t bar0 = sbase + 2 * STAGE, bar1 = bar0 + 8, full0 = bar0 + 16, full1 = bar0 + 24;
  __shared__ int s_abort;
  const int HW = H * W;
  const long long Mtot = (long long)B * HW;
  const long long ntiles = (Mtot + TC_M - 1) / TC_M;
  const int K = 9 * Cin;
  const int nstages = (Kp + TC_KC - 1) / TC_KC;
  const uint32_t ncols = Npad <= 32 ? 32u : (Npad <= 64 ? 64u : (Npad <= 128 ? 128u : 256u));
  const uint32_t idesc = umma_idesc_bf16(TC_M, Npad);
  const bool b_bulk = Npad >= 128;  // weight slices of >= 16 KB per stage go through the bulk-copy unit
  if (tid == 0) s_skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (s_skip || (long long)blockIdx.x >= ntiles) return;  // uniform across the CTA
  const long long my_tiles = (ntiles - 1 - blockIdx.x) / gridDim.x + 1;
  const long long nitems = my_tiles * nstages;

  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    mbar_init(full0, 1);
    mbar_init(full1, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  // cp.async loads of work item i into buffer i & 1 (this thread's A row and its share of the B slice)
  auto load_item = [&](long long i) {
    const long long tile = blockIdx.x + (i / nstages) * gridDim.x;
    const int s = int(i % nstages);
    const uint32_t a_s = sbase + uint32_t((i & 1) * STAGE), b_s = a_s + TcSmem::A_BYTES;
    const int kc = min(TC_KC, Kp - s * TC_KC);  // multiple of 16
    int pb = 0, pi = 0, pj = 0;
    const bool row_ok = tc_pixel(tile, tid, H, W, Mtot, out_mode == 2, pb, pi, pj);
    const __nv_bfloat16* xb = static_cast<const __nv_bfloat16*>(x);
    const int Hs = in_mode == 1 ? H / 2 : H, Ws = in_mode == 1 ? W / 2 : W;  // stored input size
    const uint32_t dst0 = a_s + uint32_t(((tid >> 3) * 8 + (tid & 7)) * 16);
    if (Cin % TC_KC == 0) {  // the stage's 64 k lie in one tap: one address, eight consecutive 16-byte chunks
      const int tap = (s * TC_KC) / Cin, ci0 = s * TC_KC - tap * Cin;
      int si = pi + tap / 3 - 1, sj = pj + tap % 3 - 1;
      const bool v = row_ok && si >= 0 && si < H && sj >= 0 && sj < W;
      if (in_mode == 1) {
        si >>= 1;
        sj >>= 1;
      }
      const __nv_bfloat16* src = v ? xb + (((long long)pb * Hs + si) * Ws + sj) * Cin + ci0 : xb;
#pragma unroll
      for (int c = 0; c < TC_KC / 8; ++c) cp_async16_l1(dst0 + uint32_t(c * (TC_M / 8) * 128), v ? src + 8 * c : xb, v);
    } else if ((Cin & 7) == 0) {  // Cin in {8, 16, 32, ...}: a stage spans several taps; one address per tap
      for (int c = 0; c < kc / 8;) {
        const int k0 = s * TC_KC + c * 8;
        const int tap = k0 / Cin, ci0 = k0 - tap * Cin;
        const int run = min((Cin - ci0) >> 3, kc / 8 - c);  // chunks of this tap inside the stage
        int si = pi + tap / 3 - 1, sj = pj + tap % 3 - 1;
        const bool v = row_ok && tap < 9 && si >= 0 && si < H && sj >= 0 && sj < W;
        if (in_mode == 1) {
          si >>= 1;
          sj >>= 1;
        }
        const __nv_bfloat16* src = v ? xb + (((long long)pb * Hs + si) * Ws + sj) * Cin + ci0 : xb;
        for (int q = 0; q < run; ++q)
          cp_async16_l1(dst0 + uint32_t((c + q) * (TC_M / 8) * 128), v ? src + 8 * q : xb, v);
        c += run;
      }
    } else
    for (int c = 0; c < kc / 8; ++c) {
      const int k0 = s * TC_KC + c * 8;
      const uint32_t dst = a_s + uint32_t(((c * (TC_M / 8) + (tid >> 3)) * 8 + (tid & 7)) * 16);
      if ((Cin & 7) == 0) {
        const int tap = k0 / Cin, ci0 = k0 - tap * Cin;
        int si = pi + tap / 3 - 1, sj = pj + tap % 3 - 1;
        const bool v = row_ok && k0 < K && si >= 0 && si < H && sj >= 0 && sj < W;
        if (in_mode == 1) {
          si >>= 1;
          sj >>= 1;
        }
        const __nv_bfloat16* src = v ? xb + (((long long)pb * Hs + si) * Ws + sj) * Cin + ci0 : xb;
        cp_async16_l1(dst, src, v);
      } else {  // thin input (the 1-channel network input): element gather
        __align__(16) __nv_bfloat16 e8[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = k0 + e, tap = k / Cin, ci = k - tap * Cin;
          const int si = pi + tap / 3 - 1, sj = pj + tap % 3 - 1;
          const bool v = row_ok && k < K && si >= 0 && si < H && sj >= 0 && sj < W;
          float val = 0.f;
          if (v) {
            if (in_mode == 2) {
              const int ri = si + H / 2 >= H ? si + H / 2 - H : si + H / 2;
              const int rj = sj + W / 2 >= W ? sj + W / 2 - W : sj + W / 2;
              val = in_scale * log1pf(static_cast<const float*>(x)[((long long)pb * H + ri) * W + rj]);
            } else {
              const int ssi = in_mode == 1 ? si >> 1 : si, ssj = in_mode == 1 ? sj >> 1 : sj;
              val = __bfloat162float(xb[(((long long)pb * Hs + ssi) * Ws + ssj) * Cin + ci]);
            }
          }
          e8[e] = __float2bfloat16_rn(val);
        }
        asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(dst),
                     "r"(reinterpret_cast<uint32_t*>(e8)[0]), "r"(reinterpret_cast<uint32_t*>(e8)[1]),
                     "r"(reinterpret_cast<uint32_t*>(e8)[2]), "r"(reinterpret_cast<uint32_t*>(e8)[3])
                     : "memory");
      }
    }
    // the packed weight slice is the stage's shared-memory image: one bulk copy by one thread for wide layers,
    // 16-byte copies by all threads for narrow ones (whose small slices would serialise on the bulk-copy unit)
    const __nv_bfloat16* wsrc = wpk + (size_t)Npad * TC_KC * s;
    if (!b_bulk)
      for (int q = tid; q < Npad * kc / 8; q += TC_THREADS)
        cp_async16_cg(b_s + uint32_t(q * 16), wsrc + size_t(q) * 8);
    cp_async_commit();
    if (b_bulk && tid == 0) {
      const uint32_t fb = (i & 1) ? full1 : full0, bytes = uint32_t(Npad * kc * 2);
      mbar_expect_tx(fb, bytes);
      bulk_g2s(b_s, wsrc, bytes, fb);
    }
  };

  bool ok = true;
  long long issued = 0, loaded = 1;  // items whose MMAs have been committed / whose loads have been issued
  load_item(0);
  for (long long i = 0; i < nitems; ++i) {
    const int s = int(i % nstages);
    const uint32_t bar = (i & 1) ? bar1 : bar0;
    cp_async_wait_all();
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      if (b_bulk && !mbar_wait((i & 1) ? full1 : full0, uint32_t((i >> 1) & 1))) {  // the weight slice of item i
        atomicCAS(err, 0, 3);
        s_abort = 1;
      } else {
        tc_fence_after();
        const uint32_t a_s = sbase + uint32_t((i & 1) * STAGE), b_s = a_s + TcSmem::A_BYTES;
        const int kc = min(TC_KC, Kp - s * TC_KC);
        for (int kk = 0; kk < kc / 16; ++kk) {
          const uint64_t da = umma_desc(a_s + uint32_t(kk * 2 * (TC_M / 8) * 128), uint32_t((TC_M / 8) * 128), 128u);
          const uint64_t db = umma_desc(b_s + uint32_t(kk * 2 * (Npad / 8) * 128), uint32_t((Npad / 8) * 128), 128u);
          umma_bf16(tmem, da, db, idesc, s > 0 || kk > 0);
        }
      }
      umma_commit(bar);  // committed either way, so every barrier keeps one phase per item
    }
    issued = i + 1;
    if (i + 1 < nitems) {
      // buffer (i + 1) & 1 was last read by item i - 1's MMAs
      if (i >= 1 && !mbar_wait(((i - 1) & 1) ? bar1 : bar0, uint32_t(((i - 1) >> 1) & 1))) {
        if (tid == 0) atomicCAS(err, 0, 1);
        ok = false;
      }
      if (__syncthreads_or(!ok || s_abort)) {
        ok = false;
        break;
      }
      load_item(i + 1);
      loaded = i + 2;
    }
    if (s == nstages - 1) {
      if (!mbar_wait(bar, uint32_t((i >> 1) & 1))) {  // this tile's last commit covers all its MMAs
        if (tid == 0) atomicCAS(err, 0, 2);
        ok = false;
      }
      if (__syncthreads_or(!ok || s_abort)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const long long tile = blockIdx.x + (i / nstages) * gridDim.x;
      int pb = 0, pi = 0, pj = 0;
      const bool row_ok = tc_pixel(tile, tid, H, W, Mtot, out_mode == 2, pb, pi, pj);
      const long long m = ((long long)pb * H + pi) * W + pj;
      const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
      for (int c8 = 0; c8 < Npad / 8; ++c8) {
        float v[8];
        tmem_ld8(trow + uint32_t(c8 * 8), v);
        const int co0 = c8 * 8;
        if (out_mode == 2) {
          // 2x2 average of the four lanes of the window (rows of a pooled warp are all valid or all invalid)
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            float r = v[e] + (co0 + e < Cout ? bias[co0 + e] : 0.f);
            if (relu) r = fmaxf(r, 0.f);
            r += __shfl_xor_sync(0xffffffffu, r, 1);
            r += __shfl_xor_sync(0xffffffffu, r, 16);
            v[e] = 0.25f * r;
          }
          if (!row_ok || co0 >= Cout || (tid & 17)) continue;  // lanes with even row and even column write
          __align__(16) __nv_bfloat16 o8[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) o8[e] = __float2bfloat16_rn(v[e]);
          const long long mp = ((long long)pb * (H / 2) + (pi >> 1)) * (W / 2) + (pj >> 1);
          *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + mp * Cout + co0) = *reinterpret_cast<uint4*>(o8);
          continue;
        }
        if (!row_ok || co0 >= Cout) continue;
        if (out_mode == 0) {
          __align__(16) __nv_bfloat16 o8[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            float r = v[e] + bias[co0 + e];
            if (relu) r = fmaxf(r, 0.f);
            o8[e] = __float2bfloat16_rn(r);
          }
          *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(y) + m * Cout + co0) = *reinterpret_cast<uint4*>(o8);
        } else {
          float* yf = static_cast<float*>(y);
          const int p = pi * W + pj;
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int co = co0 + e;
            if (co < Cout) {
              float r = v[e] + bias[co];
              if (relu) r = fmaxf(r, 0.f);
              yf[((long long)pb * Cout + co) * HW + p] = r;
            }
          }
        }
      }
      tc_fence_before();  // TMEM reads done before the next tile's first MMA overwrites the accumulator
    }
  }
  cp_async_wait_all();
  if (!ok && tid == 0) {
    // a wait gave up: give the MMAs and the weight copies already issued one more bounded wait before the
    // accumulator and the shared memory are released
    if (issued > 0) mbar_wait(((issued - 1) & 1) ? bar1 : bar0, uint32_t(((issued - 1) >> 1) & 1));
    if (b_bulk)
      for (long long j = issued > 0 ? issued - 1 : 0; j < loaded; ++j)
        mbar_wait((j & 1) ? full1 : full0, uint32_t((j >> 1) & 1));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---- 3x3 convolution as nine shifted GEMMs (Cin in {16, 32, 64}; the packed weights resident in shared memory) ----
// A CTA tile is 16 rows x 8 columns of output pixels of one image (M = 128, GEMM row m = 8 * row + column).  Its
// input halo (18 x 10 pixels, zero outside the image; for an upsampled input each halo pixel is read from its source
// pixel) is copied into shared memory once, as Cin / 8 planes of 18 x 10 16-byte pixel chunks (8 channels each).  For
// tap (dy, dx) the 128 x 16 A operand of channel chunks (2j, 2j + 1) is then the canonical K-major no-swizzle matrix
// that starts at plane 2j, halo row dy, halo column dx: its 8-row core matrices are 8 consecutive pixels of one halo
// row (128 contiguous bytes), one halo row (160 B) apart, and its two K halves one plane apart.  So the nine taps need
// no im2col copy, only nine descriptors, and the packed weights ([k / 8][n][8], k = tap * Cin + ci) are the B
// operands as they stand.  The halo loads of the next two tiles (cp.async, zero-fill outside the image) overlap the
// current tile's MMAs and epilogue.
constexpr int TAP_ROWS = 16, TAP_COLS = 8, HALO_R = TAP_ROWS + 2, HALO_C = TAP_COLS + 2;
constexpr int HALO_PLANE = HALO_R * HALO_C * 16;  // 2880 B
constexpr int TAP_NBUF = 3;                           // halo buffers: two tiles' loads in flight behind the current
constexpr int TAP_MAX_SMEM = 225 * 1024;  // dynamic shared memory of one CTA (227 KB less the 2 KB of static data)
__host__ __device__ constexpr int tap_smem(int Cin, int Npad) {
  return Npad * 9 * Cin * 2 + TAP_NBUF * (Cin / 8) * HALO_PLANE + 64;  // weights, halo buffers, the mbarrier
}

template <int Cin>
__global__ void __launch_bounds__(TC_THREADS, 4)
    k_conv_tap(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wpk,
               const float* __restrict__ bias, void* __restrict__ y, int B, int H, int W, int Cout, int Npad,
               int relu, int in_mode, int out_mode, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_skip;
  __shared__ float s_bias[TC_MAX_N];
  constexpr int chunks = Cin / 8;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wbytes = Npad * 9 * Cin * 2;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t w_s = sbase, h_s = sbase + uint32_t(wbytes), hsz = uint32_t(chunks * HALO_PLANE);
  const uint32_t bar = h_s + TAP_NBUF * hsz;
  const int tiles_x = W / TAP_COLS, per_img = tiles_x * (H / TAP_ROWS);
  const long long ntiles = (long long)B * per_img;
  const uint32_t ncols = Npad <= 32 ? 32u : (Npad <= 64 ? 64u : (Npad <= 128 ? 128u : 256u));
  const uint32_t idesc = umma_idesc_bf16(TC_M, Npad);
  if (tid == 0) s_skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (s_skip || (long long)blockIdx.x >= ntiles) return;  // uniform across the CTA
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  for (int q = tid; q < Npad; q += TC_THREADS) s_bias[q] = q < Cout ? bias[q] : 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int Hs = in_mode == 1 ? H / 2 : H, Ws = in_mode == 1 ? W / 2 : W;  // stored input size

  auto load_halo = [&](long long tile, uint32_t dst) {
    const int b = int(tile / per_img), rem = int(tile - (long long)b * per_img);
    const int y0 = (rem / tiles_x) * TAP_ROWS - 1, x0 = (rem % tiles_x) * TAP_COLS - 1;
    for (int q = tid; q < HALO_R * HALO_C * chunks; q += TC_THREADS) {
      const int j = q % chunks, pix = q / chunks, hy = pix / HALO_C, hx = pix - hy * HALO_C;
      int sy = y0 + hy, sx = x0 + hx;
      const bool v = sy >= 0 && sy < H && sx >= 0 && sx < W;
      if (in_mode == 1) {
        sy >>= 1;
        sx >>= 1;
      }
      const __nv_bfloat16* src = v ? x + (((long long)b * Hs + sy) * Ws + sx) * Cin + 8 * j : x;
      cp_async16_l1(dst + uint32_t(j * HALO_PLANE + (hy * HALO_C + hx) * 16), src, v);
    }
  };

  const long long my_tiles = (ntiles - 1 - blockIdx.x) / gridDim.x + 1;
  // cp.async groups: weights with tile 0's halo, then one group per tile (empty past the end), so that before tile i
  // exactly TAP_NBUF - 2 younger groups may still be pending
  for (int q = tid; q < wbytes / 16; q += TC_THREADS) cp_async16_cg(w_s + uint32_t(q * 16), wpk + size_t(q) * 8);
  for (int k = 0; k < TAP_NBUF - 1; ++k) {
    if (k < my_tiles) load_halo(blockIdx.x + k * (long long)gridDim.x, h_s + uint32_t(k) * hsz);
    cp_async_commit();
  }
  bool ok = true;
  uint32_t phase = 0;
  for (long long i = 0; i < my_tiles; ++i) {
    const long long tile = blockIdx.x + i * gridDim.x;
    const uint32_t hcur = h_s + uint32_t(i % TAP_NBUF) * hsz;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(TAP_NBUF - 2) : "memory");
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      int mm = 0;
      for (int tap = 0; tap < 9; ++tap) {
        const uint32_t a_tap = hcur + uint32_t(((tap / 3) * HALO_C + tap % 3) * 16);
#pragma unroll
        for (int jj = 0; jj < chunks / 2; ++jj, ++mm) {
          const uint64_t da = umma_desc(a_tap + uint32_t(2 * jj * HALO_PLANE), HALO_PLANE, HALO_C * 16);
          const uint64_t db = umma_desc(w_s + uint32_t((tap * chunks + 2 * jj) * Npad * 16), uint32_t(Npad * 16), 128u);
          umma_bf16(tmem, da, db, idesc, mm > 0);
        }
      }
      umma_commit(bar);
    }
    // tile i + TAP_NBUF - 1 goes into the buffer of tile i - 1, whose MMAs completed before its epilogue
    if (i + TAP_NBUF - 1 < my_tiles)
      load_halo(tile + (TAP_NBUF - 1) * (long long)gridDim.x, h_s + uint32_t((i + TAP_NBUF - 1) % TAP_NBUF) * hsz);
    cp_async_commit();
    // one thread waits for the MMAs (the others do not spin on the barrier) and the block barrier passes it on
    if (tid == 0 && !mbar_wait(bar, phase)) {
      atomicCAS(err, 0, 4);
      ok = false;
    }
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    tc_fence_after();
    const int b = int(tile / per_img), rem = int(tile - (long long)b * per_img);
    const int m = warp * 32 + lane;
    const int py = (rem / tiles_x) * TAP_ROWS + (m >> 3), px = (rem % tiles_x) * TAP_COLS + (m & 7);
    const uint32_t trow = tmem + (uint32_t(warp * 32) << 16);
    for (int c8 = 0; c8 < (Cout + 7) / 8; ++c8) {  // uniform across the warp (tcgen05.ld is warp-collective)
      float v[8];
      tmem_ld8(trow + uint32_t(c8 * 8), v);
      const int co0 = c8 * 8;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        float r = v[e] + s_bias[co0 + e];
        if (relu) r = fmaxf(r, 0.f);
        if (out_mode == 2) {  // 2 x 2 window: lanes l, l ^ 1 (next column), l ^ 8 (next row), l ^ 9
          r += __shfl_xor_sync(0xffffffffu, r, 1);
          r += __shfl_xor_sync(0xffffffffu, r, 8);
          r *= 0.25f;
        }
        v[e] = r;
      }
      if (out_mode == 1) {  // NCHW FP32 (the output layer)
        float* yf = static_cast<float*>(y);
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (co0 + e < Cout) yf[(((long long)b * Cout + co0 + e) * H + py) * W + px] = v[e];
        continue;
      }
      __align__(16) __nv_bfloat16 o8[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) o8[e] = __float2bfloat16_rn(v[e]);
      __nv_bfloat16* yb = static_cast<__nv_bfloat16*>(y);
      if (out_mode == 2) {
        if (lane & 9) continue;
        const long long mp = ((long long)b * (H / 2) + (py >> 1)) * (W / 2) + (px >> 1);
        *reinterpret_cast<uint4*>(yb + mp * Cout + co0) = *reinterpret_cast<uint4*>(o8);
      } else {
        const long long mo = ((long long)b * H + py) * W + px;
        *reinterpret_cast<uint4*>(yb + mo * Cout + co0) = *reinterpret_cast<uint4*>(o8);
      }
    }
    tc_fence_before();  // TMEM reads done before the next tile's first MMA overwrites the accumulator
  }
  cp_async_wait_all();
  if (!ok && tid == 0) mbar_wait(bar, phase ^ 1u);  // one more bounded wait for the MMAs in flight
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---- the shifted-GEMM form for wide inputs (Cin = 128 or 256, N <= 64): channel groups of 64 streamed per tile ----
// The packed weights no longer fit beside the halos, so each tile runs over its Cin / 64 channel groups, and each
// group over three items of three taps: item j = (tile, group, third).  A group's 8 halo planes (cp.async by all
// threads, as in k_conv_tap) land in halo buffer (tile * G + group) & 1 while the previous group's items run; an
// item's three 64-channel weight slices (one-thread bulk copies of 8 x Npad x 16 bytes each, completing on an
// mbarrier) land in weight buffer j & 1 while item j - 1's MMAs run.  3 x 4 MMAs per item accumulate into the tile's
// accumulator (two, alternating by tile, so that a tile's epilogue runs after the next tile's first MMAs have been
// issued).  About 95 KB of shared memory: two CTAs per SM.
constexpr int TAPG_HALO = 8 * HALO_PLANE;  // one group's halo: 8 planes of 8 channels
__host__ __device__ constexpr int tapg_wbytes(int Npad) { return 3 * 8 * Npad * 16; }  // three taps' slices
__host__ __device__ constexpr int tapg_smem(int Npad) { return 2 * TAPG_HALO + 2 * tapg_wbytes(Npad) + 64; }

template <int Cin>
__global__ void __launch_bounds__(TC_THREADS, 2)
    k_conv_tapg(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ wpk,
                const float* __restrict__ bias, void* __restrict__ y, int B, int H, int W, int Cout, int Npad,
                int relu, int in_mode, int out_mode, int* __restrict__ err) {
  constexpr int G = Cin / 64, IPT = 3 * G;  // items per tile
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ int s_skip;
  __shared__ float s_bias[TC_MAX_N];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wbytes = tapg_wbytes(Npad);
  const uint32_t sbase = smem_u32(smem);
  const uint32_t h_s = sbase, w_s = sbase + 2 * TAPG_HALO;
  const uint32_t bars = w_s + 2 * uint32_t(wbytes);  // full0, full1 (weights landed), done0, done1 (MMAs done)
  const int tiles_x = W / TAP_COLS, per_img = tiles_x * (H / TAP_ROWS);
  const long long ntiles = (long long)B * per_img;
  const uint32_t ncols = Npad <= 32 ? 32u : 64u;
  const uint32_t idesc = umma_idesc_bf16(TC_M, Npad);
  if (tid == 0) s_skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (s_skip || (long long)blockIdx.x >= ntiles) return;  // uniform across the CTA
  if (tid == 0) {
    for (int q = 0; q < 4; ++q) mbar_init(bars + 8 * q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(2 * ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  for (int q = tid; q < Npad; q += TC_THREADS) s_bias[q] = q < Cout ? bias[q] : 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int Hs = in_mode == 1 ? H / 2 : H, Ws = in_mode == 1 ? W / 2 : W;  // stored input size
  const long long my_tiles = (ntiles - 1 - blockIdx.x) / gridDim.x + 1, nitems = my_tiles * IPT;

  // all threads: the halo planes of group gi = tile index * G + group (halo buffer gi & 1)
  auto load_halo = [&](long long gi) {
    const long long tile = blockIdx.x + (gi / G) * gridDim.x;
    const int g = int(gi % G);
    const uint32_t hdst = h_s + uint32_t(gi & 1) * TAPG_HALO;
    const int b = int(tile / per_img), rem = int(tile - (long long)b * per_img);
    const int y0 = (rem / tiles_x) * TAP_ROWS - 1, x0 = (rem % tiles_x) * TAP_COLS - 1;
    for (int q = tid; q < HALO_R * HALO_C * 8; q += TC_THREADS) {
      const int c = q & 7, pix = q >> 3, hy = pix / HALO_C, hx = pix - hy * HALO_C;
      int sy = y0 + hy, sx = x0 + hx;
      const bool v = sy >= 0 && sy < H && sx >= 0 && sx < W;
      if (in_mode == 1) {
        sy >>= 1;
        sx >>= 1;
      }
      const __nv_bfloat16* src = v ? x + (((long long)b * Hs + sy) * Ws + sx) * Cin + 64 * g + 8 * c : x;
      cp_async16_l1(hdst + uint32_t(c * HALO_PLANE + (hy * HALO_C + hx) * 16), src, v);
    }
    cp_async_commit();
  };
  // one thread: item j's three weight slices into weight buffer j & 1
  auto load_weights = [&](long long j) {
    const int g = int((j % IPT) / 3), third = int(j % 3);
    const uint32_t full = bars + 8 * uint32_t(j & 1), slice = uint32_t(8 * Npad * 16);
    const uint32_t wdst = w_s + uint32_t(j & 1) * uint32_t(wbytes);
    mbar_expect_tx(full, uint32_t(wbytes));
    for (int t = 0; t < 3; ++t) {
      const int tap = 3 * third + t;
      bulk_g2s(wdst + uint32_t(t) * slice, wpk + size_t(tap * (Cin / 8) + 8 * g) * Npad * 8, slice, full);
    }
  };
  auto epilogue = [&](long long i) {
    const long long tile = blockIdx.x + i * gridDim.x;
    const int b = int(tile / per_img), rem = int(tile - (long long)b * per_img);
    const int m = warp * 32 + lane;
    const int py = (rem / tiles_x) * TAP_ROWS + (m >> 3), px = (rem % tiles_x) * TAP_COLS + (m & 7);
    const uint32_t trow = tmem + uint32_t(i & 1) * ncols + (uint32_t(warp * 32) << 16);
    for (int c8 = 0; c8 < (Cout + 7) / 8; ++c8) {
      float v[8];
      tmem_ld8(trow + uint32_t(c8 * 8), v);
      const int co0 = c8 * 8;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        float r = v[e] + s_bias[co0 + e];
        if (relu) r = fmaxf(r, 0.f);
        if (out_mode == 2) {
          r += __shfl_xor_sync(0xffffffffu, r, 1);
          r += __shfl_xor_sync(0xffffffffu, r, 8);
          r *= 0.25f;
        }
        v[e] = r;
      }
      if (out_mode == 1) {
        float* yf = static_cast<float*>(y);
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (co0 + e < Cout) yf[(((long long)b * Cout + co0 + e) * H + py) * W + px] = v[e];
        continue;
      }
      __align__(16) __nv_bfloat16 o8[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) o8[e] = __float2bfloat16_rn(v[e]);
      __nv_bfloat16* yb = static_cast<__nv_bfloat16*>(y);
      if (out_mode == 2) {
        if (lane & 9) continue;
        const long long mp = ((long long)b * (H / 2) + (py >> 1)) * (W / 2) + (px >> 1);
        *reinterpret_cast<uint4*>(yb + mp * Cout + co0) = *reinterpret_cast<uint4*>(o8);
      } else {
        const long long mo = ((long long)b * H + py) * W + px;
        *reinterpret_cast<uint4*>(yb + mo * Cout + co0) = *reinterpret_cast<uint4*>(o8);
      }
    }
    tc_fence_before();  // TMEM reads done before the MMAs of tile i + 2 overwrite this accumulator
  };

  bool ok = true;
  long long committed = 0, loaded = 1;  // items whose MMAs have been committed / whose weights have been requested
  load_halo(0);
  if (tid == 0) load_weights(0);
  for (long long j = 0; j < nitems && ok; ++j) {
    const long long i = j / IPT, gi = j / 3;
    const int third = int(j % 3), g = int((j % IPT) / 3);
    bool fail = false;
    if (third == 0) cp_async_wait_all();  // this group's halo (the only group in flight)
    fence_async_smem();
    if (tid == 0 && !mbar_wait(bars + 8 * uint32_t(j & 1), uint32_t((j >> 1) & 1))) {  // this item's weights
      atomicCAS(err, 0, 5);
      fail = true;
    }
    if (__syncthreads_or(fail)) {
      ok = false;
      break;
    }
    if (tid == 0) {
      tc_fence_after();
      const uint32_t acc = tmem + uint32_t(i & 1) * ncols, hbuf = h_s + uint32_t(gi & 1) * TAPG_HALO;
      const uint32_t wbuf = w_s + uint32_t(j & 1) * uint32_t(wbytes);
      for (int t = 0; t < 3; ++t) {
        const int tap = 3 * third + t;
        const uint32_t a_tap = hbuf + uint32_t(((tap / 3) * HALO_C + tap % 3) * 16);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const uint64_t da = umma_desc(a_tap + uint32_t(2 * jj * HALO_PLANE), HALO_PLANE, HALO_C * 16);
          const uint64_t db = umma_desc(wbuf + uint32_t((t * 8 + 2 * jj) * Npad * 16), uint32_t(Npad * 16), 128u);
          umma_bf16(acc, da, db, idesc, g > 0 || third > 0 || t > 0 || jj > 0);
        }
      }
      umma_commit(bars + 16 + 8 * uint32_t(j & 1));
    }
    committed = j + 1;
    // weight buffer (j + 1) & 1 was last read by item j - 1's MMAs; at a group's first item, the other halo buffer
    // was last read by the previous group's items, whose MMAs are all done once item j - 1's are
    if (j >= 1 && tid == 0 && !mbar_wait(bars + 16 + 8 * uint32_t((j - 1) & 1), uint32_t(((j - 1) >> 1) & 1))) {
      atomicCAS(err, 0, 6);
      fail = true;
    }
    if (__syncthreads_or(fail)) {
      ok = false;
      break;
    }
    if (j + 1 < nitems) {
      if (tid == 0) load_weights(j + 1);
      loaded = j + 2;
    }
    if (third == 0 && (gi + 1) * 3 < nitems) load_halo(gi + 1);
    // the previous tile's MMAs (item j - 1 was its last) are done: its epilogue overlaps this tile's MMAs
    if (g == 0 && third == 0 && i > 0) {
      tc_fence_after();
      epilogue(i - 1);
    }
  }
  if (ok) {  // the last tile
    bool fail = false;
    if (tid == 0 && !mbar_wait(bars + 16 + 8 * uint32_t((nitems - 1) & 1), uint32_t(((nitems - 1) >> 1) & 1))) {
      atomicCAS(err, 0, 6);
      fail = true;
    }
    if (!__syncthreads_or(fail)) {
      tc_fence_after();
      epilogue(my_tiles - 1);
    } else {
      ok = false;
    }
  }
  cp_async_wait_all();
  if (!ok && tid == 0) {  // bounded waits for the MMAs and weight copies still in flight
    for (long long j = committed > 1 ? committed - 2 : 0; j < committed; ++j)
      mbar_wait(bars + 16 + 8 * uint32_t(j & 1), uint32_t((j >> 1) & 1));
    for (long long j = committed; j < loaded; ++j) mbar_wait(bars + 8 * uint32_t(j & 1), uint32_t((j >> 1) & 1));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * ncols) : "memory");
}

// wpk (stage s, chunk c, 8-row group g, row r, element e) = w[n = 8g + r][k = 64 s + 8 c + e] in BF16, the
// k = tap * Cin + ci order of the GEMM; zero for n >= Cout or k >= 9 Cin.  Weights FP32 (Cout, Cin, 3, 3).
__global__ void k_pack_tc_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wpk, int Cin, int Cout,
                                  int Npad, int Kp) {
  const int K = 9 * Cin;
  const size_t n_all = size_t(Npad) * Kp;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n_all; q += size_t(gridDim.x) * blockDim.x) {
    const int s = int(q / (size_t(Npad) * TC_KC));
    const int rem = int(q - size_t(s) * Npad * TC_KC);
    const int kc = min(TC_KC, Kp - s * TC_KC);
    const int c = rem / (Npad * 8), r2 = rem % (Npad * 8);
    const int n = r2 / 8, e = r2 % 8;  // (g, r) flattened = n
    const int k = s * TC_KC + c * 8 + e;
    float v = 0.f;
    if (c < kc / 8 && n < Cout && k < K) {
      const int tap = k / Cin, ci = k % Cin;
      v = w[(size_t(n) * Cin + ci) * 9 + tap];
    }
    wpk[q] = __float2bfloat16_rn(v);
  }
}

// NHWC BF16 2x2 average pooling to H x W (input 2H x 2W), C channels
__global__ void k_tc_pool2(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, int B, int H, int W,
                           int C) {
  const size_t n = size_t(B) * H * W * C;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int c = int(q % C);
    const size_t pix = q / C;
    const int j = int(pix % W), i = int((pix / W) % H);
    const size_t b = pix / (size_t(W) * H);
    const size_t r0 = ((b * 2 * H + 2 * i) * 2 * W + 2 * j) * C + c, r1 = r0 + size_t(2 * W) * C;
    const float s = __bfloat162float(x[r0]) + __bfloat162float(x[r0 + C]) + __bfloat162float(x[r1]) +
                    __bfloat162float(x[r1 + C]);
    y[q] = __float2bfloat16_rn(0.25f * s);
  }
}
// NHWC BF16 2x nearest upsampling of H x W, C channels
__global__ void k_tc_up2(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y, int B, int H, int W,
                         int C) {
  const size_t n = size_t(B) * 4 * H * W * C;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int c = int(q % C);
    const size_t pix = q / C;
    const int j = int(pix % (2 * W)), i = int((pix / (2 * W)) % (2 * H));
    const size_t b = pix / (size_t(4) * W * H);
    y[q] = x[((b * H + i / 2) * W + j / 2) * C + c];
  }
}
__global__ void k_to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, size_t n) {
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x)
    y[q] = __float2bfloat16_rn(x[q]);
}

// First layer on CUDA cores (K = 9 is too thin for the tensor cores): y = pool2(relu(bias + conv3x3(in_scale *
// log1p(centred amp)))) as NHWC BF16 (B x H/2 x W/2 x C1), C1 output channels.  A CTA owns a 16 x 16 tile of pooled
// pixels (32 x 32 convolution outputs): the 34 x 34 input halo is transformed once into shared memory, each thread
// computes one pooled pixel's 2 x 2 outputs for all channels from a 4 x 4 window.
template <int C1>
__global__ void __launch_bounds__(256, 4) k_tc_first(const float* __restrict__ amp, const float* __restrict__ w,
                                                  const float* __restrict__ bias, __nv_bfloat16* __restrict__ y, int H,
                                                  int W, float in_scale) {
  __shared__ float s_in[34][35];
  __shared__ float s_w[9][C1];
  __shared__ float s_b[C1];
  const int Hp = H / 2, Wp = W / 2;
  const int tiles_x = (Wp + 15) / 16;
  const int ti = blockIdx.x / tiles_x, tj = blockIdx.x % tiles_x, b = blockIdx.y;
  const float* a = amp + (size_t)b * H * W;
  for (int q = threadIdx.x; q < 34 * 34; q += 256) {
    const int r = q / 34, c = q % 34;
    const int gi = 32 * ti + r - 1, gj = 32 * tj + c - 1;
    float v = 0.f;
    if (gi >= 0 && gi < H && gj >= 0 && gj < W) {
      const int ri = gi + H / 2 >= H ? gi + H / 2 - H : gi + H / 2;
      const int rj = gj + W / 2 >= W ? gj + W / 2 - W : gj + W / 2;
      // the BF16 rounding the tensor-core path applies to its inputs
      v = __bfloat162float(__float2bfloat16_rn(in_scale * log1pf(a[(size_t)ri * W + rj])));
    }
    s_in[r][c] = v;
  }
  for (int q = threadIdx.x; q < 9 * C1; q += 256) {
    const int k = q / C1, co = q % C1;
    s_w[k][co] = __bfloat162float(__float2bfloat16_rn(w[co * 9 + k]));
  }
  if (threadIdx.x < C1) s_b[threadIdx.x] = bias[threadIdx.x];
  __syncthreads();
  const int li = threadIdx.x / 16, lj = threadIdx.x % 16;
  const int pi = 16 * ti + li, pj = 16 * tj + lj;
  if (pi >= Hp || pj >= Wp) return;
  float v[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) v[r][c] = s_in[2 * li + r][2 * lj + c];
  __align__(16) __nv_bfloat16 o[C1];
#pragma unroll
  for (int co = 0; co < C1; ++co) {
    float s = 0.f;
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        float acc = s_b[co];
#pragma unroll
        for (int k = 0; k < 9; ++k) acc += s_w[k][co] * v[dy + k / 3][dx + k % 3];
        s += fmaxf(acc, 0.f);
      }
    o[co] = __float2bfloat16_rn(0.25f * s);
  }
  uint4* dst = reinterpret_cast<uint4*>(y + (((size_t)b * Hp + pi) * Wp + pj) * C1);
#pragma unroll
  for (int q = 0; q < C1 / 8; ++q) dst[q] = reinterpret_cast<const uint4*>(o)[q];
}

// Output layer on CUDA cores (N = 3 is too narrow for the tensor cores): y (NCHW FP32) = bias + conv3x3(x) for x NHWC
// BF16 with CIN channels, CO <= 4 outputs; one thread per pixel, weights (BF16-rounded like the tensor-core path) in
// shared memory.
template <int CIN>
__global__ void __launch_bounds__(256) k_tc_last(const __nv_bfloat16* __restrict__ x, const float* __restrict__ w,
                                                 const float* __restrict__ bias, float* __restrict__ y, int B, int H,
                                                 int W, int CO) {
  __shared__ float s_w[4][9][CIN];
  for (int q = threadIdx.x; q < 4 * 9 * CIN; q += 256) {
    const int co = q / (9 * CIN), k = (q / CIN) % 9, ci = q % CIN;
    s_w[co][k][ci] = co < CO ? __bfloat162float(__float2bfloat16_rn(w[((size_t)co * CIN + ci) * 9 + k])) : 0.f;
  }
  __syncthreads();
  const size_t n = (size_t)B * H * W;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int j = int(q % W), i = int((q / W) % H);
    const size_t b = q / ((size_t)H * W);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      const int si = i + k / 3 - 1, sj = j + k % 3 - 1;
      if (si < 0 || si >= H || sj < 0 || sj >= W) continue;
      const uint4* src = reinterpret_cast<const uint4*>(x + ((b * H + si) * W + sj) * CIN);
#pragma unroll
      for (int c8 = 0; c8 < CIN / 8; ++c8) {
        const uint4 u = src[c8];
        const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&u);
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const float xv = __bfloat162float(e[t]);
#pragma unroll
          for (int co = 0; co < 4; ++co) acc[co] += s_w[co][k][8 * c8 + t] * xv;
        }
      }
    }
#pragma unroll
    for (int co = 0; co < 4; ++co)
      if (co < CO) y[(b * CO + co) * H * W + (size_t)i * W + j] = acc[co] + bias[co];
  }
}

// Self-test of the bounded mbarrier wait: out[0] = 1 when a wait on a phase nothing completes gives up after `limit`
// rounds (the expected outcome), out[1] = 0 when the same wait succeeds after one arrival (the control).
__global__ void k_selftest_mbar(int* out, uint32_t limit) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const bool completed = mbar_wait(b, 0, limit);
  __syncthreads();
  if (threadIdx.x == 0) {
    out[0] = completed ? 0 : 1;
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(b) : "memory");
  }
  __syncthreads();
  const bool after = mbar_wait(b, 0, limit);
  if (threadIdx.x == 0) out[1] = after ? 0 : 1;
}

int grid1(size_t n) {
  const size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > 8192 ? 8192 : g));
}

int fail(const std::string& msg, int code) {
  set_last_error(msg);
  return code;
}

int finish(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(std::string(what) + ": " + cudaGetErrorString(e), PTY_ERR_CUDA);
  return PTY_OK;
}

int pad16(int v) { return (v + 15) / 16 * 16; }

}  // namespace
}  // namespace pty

using namespace pty;

extern "C" {

int pty_tc_weights_size(int Cin, int Cout) {
  if (Cin < 1 || Cout < 1 || Cout > TC_MAX_N) return -1;
  return pad16(Cout) * pad16(9 * Cin);
}

int pty_tc_pack_weights(const float* w, int Cin, int Cout, void* wpk, void* stream) {
  if (!w || !wpk || Cin < 1 || Cout < 1 || Cout > TC_MAX_N) return fail("pty_tc_pack_weights: bad argument", PTY_ERR_INVALID);
  const int Npad = pad16(Cout), Kp = pad16(9 * Cin);
  k_pack_tc_weights<<<grid1(size_t(Npad) * Kp), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, static_cast<__nv_bfloat16*>(wpk), Cin, Cout, Npad, Kp);
  return finish(cudaGetLastError(), "pty_tc_pack_weights");
}

int pty_tc_conv3x3(const void* x, const void* wpk, const float* bias, void* y, int B, int Cin, int Cout, int H, int W,
                   int relu, int in_mode, int out_mode, float in_scale, int* err, void* stream) {
  if (!x || !wpk || !bias || !y || !err || B < 1 || H < 1 || W < 1 || Cin < 1 || Cout < 1 || Cout > TC_MAX_N ||
      in_mode < 0 || in_mode > 2 || out_mode < 0 || out_mode > 2)
    return fail("pty_tc_conv3x3: bad argument", PTY_ERR_INVALID);
  if (out_mode != 1 && (Cout % 8)) return fail("pty_tc_conv3x3: NHWC output needs Cout % 8 == 0", PTY_ERR_INVALID);
  if (Cin % 8 && Cin > 8) return fail("pty_tc_conv3x3: Cin must be a multiple of 8 or at most 8", PTY_ERR_INVALID);
  // the shifted-GEMM forms (tiles of 16 x 8 output pixels): thin inputs with the packed weights resident in shared
  // memory, or 128 / 256 input channels streamed in groups of 64 for N <= 64
  const bool tap = (Cin == 16 || Cin == 32 || Cin == 64) && tap_smem(Cin, pad16(Cout)) <= TAP_MAX_SMEM &&
                   H % TAP_ROWS == 0 && W % TAP_COLS == 0 && (in_mode == 0 || in_mode == 1);
  const bool tapg = (Cin == 128 || Cin == 256) && pad16(Cout) <= 64 && H % TAP_ROWS == 0 && W % TAP_COLS == 0 &&
                    (in_mode == 0 || in_mode == 1);
  if (out_mode == 2 && !tap && !tapg && ((H & 1) || (W % 16)))
    return fail("pty_tc_conv3x3: pooled output needs an even H and W a multiple of 16 (or, in the shifted-GEMM "
                "form, H a multiple of 16 and W of 8)", PTY_ERR_INVALID);
  if (in_mode == 1 && ((H & 1) || (W & 1))) return fail("pty_tc_conv3x3: upsampled input needs even H, W", PTY_ERR_INVALID);
  if (in_mode == 2 && (Cin != 1 || (H & 1) || (W & 1)))
    return fail("pty_tc_conv3x3: amplitude input needs Cin = 1 and even H, W", PTY_ERR_INVALID);
  // the kernel's shared-memory limit is a per-device attribute: set it once on every device that launches it
  constexpr int MAX_DEV = 64;
  static std::atomic<bool> attr_set[MAX_DEV];
  int cur = 0;
  cudaError_t ge = cudaGetDevice(&cur);
  if (ge != cudaSuccess || cur < 0 || cur >= MAX_DEV) return finish(ge, "pty_tc_conv3x3: device");
  if (!attr_set[cur].load()) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TcSmem::total(TC_MAX_N));
    const void* taps[5] = {(const void*)k_conv_tap<16>, (const void*)k_conv_tap<32>, (const void*)k_conv_tap<64>,
                           (const void*)k_conv_tapg<128>, (const void*)k_conv_tapg<256>};
    for (const void* f : taps)
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, TAP_MAX_SMEM);
    if (e != cudaSuccess) return finish(e, "pty_tc_conv3x3: shared memory attribute");
    attr_set[cur].store(true);
  }
  const int Npad = pad16(Cout);
  const int smem = tap ? tap_smem(Cin, Npad) : (tapg ? tapg_smem(Npad) : TcSmem::total(Npad));
  // CTAs resident per SM, from the shared-memory budget (1 KB reserved per CTA, plus the kernel's static 1 KB) and
  // the 512 TMEM columns; the runtime's occupancy query reports 1 for this kernel.  Persistent CTAs do not wait on
  // one another, so an estimate that is too high only queues CTAs.
  int dev = 0, sms = 0, smem_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (e != cudaSuccess) return finish(e, "pty_tc_conv3x3: device attributes");
  const int ncols = (Npad <= 32 ? 32 : (Npad <= 64 ? 64 : (Npad <= 128 ? 128 : 256))) * (tapg ? 2 : 1);
  int per_sm = smem_sm / (smem + 2048);
  if (per_sm > 512 / ncols) per_sm = 512 / ncols;  // TMEM columns of one SM
  if (per_sm > 2048 / TC_THREADS) per_sm = 2048 / TC_THREADS;
  {  // registers (allocated per warp in units of 256): persistent CTAs beyond the resident ones would run as a tail
    static int regs[6] = {0, 0, 0, 0, 0, 0};
    const int ki = tap ? (Cin == 16 ? 1 : (Cin == 32 ? 2 : 3)) : (tapg ? (Cin == 128 ? 4 : 5) : 0);
    int& r = regs[ki];
    if (!r) {
      const void* fns[6] = {(const void*)k_conv_tc, (const void*)k_conv_tap<16>, (const void*)k_conv_tap<32>,
                            (const void*)k_conv_tap<64>, (const void*)k_conv_tapg<128>, (const void*)k_conv_tapg<256>};
      cudaFuncAttributes fa{};
      if (cudaFuncGetAttributes(&fa, fns[ki]) == cudaSuccess) r = fa.numRegs;
    }
    if (r > 0) {
      const int per_warp = (r * 32 + 255) / 256 * 256;
      const int by_regs = 65536 / (per_warp * (TC_THREADS / 32));
      if (per_sm > by_regs) per_sm = by_regs;
    }
  }
  if (per_sm < 1) per_sm = 1;
  const long long M = (long long)B * H * W;
  const long long tiles = (M + TC_M - 1) / TC_M;  // both forms: 128 pixels per tile
  const long long resident = (long long)sms * per_sm;
  const unsigned blocks = unsigned(tiles < resident ? tiles : resident);
  if (tap) {
    auto kern = Cin == 16 ? k_conv_tap<16> : (Cin == 32 ? k_conv_tap<32> : k_conv_tap<64>);
    kern<<<blocks, TC_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(wpk), bias, y, B, H, W, Cout, Npad,
        relu, in_mode, out_mode, err);
    return finish(cudaGetLastError(), "pty_tc_conv3x3");
  }
  if (tapg) {
    auto kern = Cin == 128 ? k_conv_tapg<128> : k_conv_tapg<256>;
    kern<<<blocks, TC_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(wpk), bias, y, B, H, W, Cout, Npad,
        relu, in_mode, out_mode, err);
    return finish(cudaGetLastError(), "pty_tc_conv3x3");
  }
  k_conv_tc<<<blocks, TC_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
      x, static_cast<const __nv_bfloat16*>(wpk), bias, y, B, H, W, Cin, Cout, Npad, pad16(9 * Cin), relu, in_mode,
      out_mode, in_scale, err);
  return finish(cudaGetLastError(), "pty_tc_conv3x3");
}

int pty_tc_first_layer(const float* amp, const float* w, const float* bias, void* y, int B, int Cout, int H, int W,
                       float in_scale, void* stream) {
  if (!amp || !w || !bias || !y || B < 1 || B > 65535 || Cout != 16 || (H & 1) || (W & 1) || H < 2 || W < 2)
    return fail("pty_tc_first_layer: bad argument (Cout must be 16, H and W even)", PTY_ERR_INVALID);
  const int tiles = ((H / 2 + 15) / 16) * ((W / 2 + 15) / 16);
  k_tc_first<16><<<dim3(tiles, B), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      amp, w, bias, static_cast<__nv_bfloat16*>(y), H, W, in_scale);
  return finish(cudaGetLastError(), "pty_tc_first_layer");
}

int pty_tc_last_layer(const void* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H,
                      int W, void* stream) {
  if (!x || !w || !bias || !y || B < 1 || Cout < 1 || Cout > 4 || H < 1 || W < 1 || Cin != 32)
    return fail("pty_tc_last_layer: bad argument (Cin must be 32, Cout at most 4)", PTY_ERR_INVALID);
  const size_t n = (size_t)B * H * W;
  k_tc_last<32><<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(x), w,
                                                                          bias, y, B, H, W, Cout);
  return finish(cudaGetLastError(), "pty_tc_last_layer");
}

int pty_selftest_bounded_waits(int* codes) {
  if (!codes) return fail("pty_selftest_bounded_waits: null argument", PTY_ERR_INVALID);
  int* d = nullptr;
  unsigned* bar = nullptr;
  cudaError_t e = cudaMalloc(&d, 8 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&bar, 4 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(d, 0xFF, 8 * sizeof(int));
  if (e == cudaSuccess) {
    k_selftest_mbar<<<1, 64>>>(d, 1u << 12);
    e = cudaGetLastError();
  }
  // grid barrier: 16 CTAs, 64 rounds reaching their count (control), then one round expecting 17 arrivals
  if (e == cudaSuccess) e = selftest_grid_barrier(16, 16, 1u << 16, 64, bar, d + 2, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(codes + 2, d + 2, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = selftest_grid_barrier(16, 17, 1u << 16, 1, bar, d + 3, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(codes, d, 2 * sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(codes + 3, d + 3, sizeof(int), cudaMemcpyDeviceToHost);
  if (d) cudaFree(d);
  if (bar) cudaFree(bar);
  return finish(e, "pty_selftest_bounded_waits");
}

int pty_tc_pool2(const void* x, void* y, int B, int H, int W, int C, void* stream) {
  if (!x || !y || B < 1 || H < 1 || W < 1 || C < 1) return fail("pty_tc_pool2: bad argument", PTY_ERR_INVALID);
  k_tc_pool2<<<grid1(size_t(B) * H * W * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), static_cast<__nv_bfloat16*>(y), B, H, W, C);
  return finish(cudaGetLastError(), "pty_tc_pool2");
}

int pty_tc_up2(const void* x, void* y, int B, int H, int W, int C, void* stream) {
  if (!x || !y || B < 1 || H < 1 || W < 1 || C < 1) return fail("pty_tc_up2: bad argument", PTY_ERR_INVALID);
  k_tc_up2<<<grid1(size_t(B) * 4 * H * W * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), static_cast<__nv_bfloat16*>(y), B, H, W, C);
  return finish(cudaGetLastError(), "pty_tc_up2");
}

int pty_tc_to_bf16(const float* x, void* y, size_t n, void* stream) {
  if (!x || !y || n == 0) return fail("pty_tc_to_bf16: bad argument", PTY_ERR_INVALID);
  k_to_bf16<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, static_cast<__nv_bfloat16*>(y), n);
  return finish(cudaGetLastError(), "pty_tc_to_bf16");
}

}  // extern "C"
