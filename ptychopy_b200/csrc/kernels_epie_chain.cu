// ePIE as a chain of whole-GPU kernels per position (ePIE::iteration, src/ePIE.cpp:65-129): launch variant 3 with FP32
// transforms (fft2_pdl), and the precision = 1 path, whose 2-D transforms run as split-BF16 tensor-core stages
// (fft2_tc, N = 256).  The pointwise steps follow the fused kernel k_epie phase by phase (kernels_epie.cu), so the
// paths compute the same update; the chain spreads every step over the whole GPU, where the fused kernel runs one
// thread-block cluster (it wins with several probe modes).  Per position s of the visiting order:
//   exit      psi_k = bilinear patch (Q2) x P_k, k < Ka                       (get projections, a3/a4)
//   FFT2      Psi_k
//   modulus   d_k = (Psi'_k - Psi_k)/N^2 with the modal modulus and the error metric (a5, a9); by linearity the
//             inverse transform of d_k is psi_new - psi_old
//   IFFT2     dpsi_k
//   object    O += (1/max |P|^2) sum_k conj(P_k) dpsi_k at the rounded position, phase constraint, |O|^2 cache (a6)
//             with the 16 x 16 tile maxima of |O|^2 under the patch, one block per tile (probe update only)
//   probe     object max from the tiles; P_k += (1/max |O|^2) conj(O) dpsi_k; |P_k|^2 cache and the probe maximum
//             (a7): pixel-local, so it runs at the start of the next position's exit kernel, by the threads that
//             then read those probe pixels (the last position's in a final kernel)
// Every kernel is launched with programmatic dependent launch.
#include <algorithm>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels.h"
#include "kernels_epie.h"
#include "fftx.cuh"
#include "kernels_mls.h"
#include "pdl.cuh"

namespace pty {

namespace {

int grid_e(size_t n) {
  size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > 1184 ? 1184 : g));
}

// The object max from TM, reduced by every block (1/max |O|^2, the probe update's step); block 0 records it.
__device__ float ec_object_step(const EpieChainArgs& g) {
  __shared__ float s_om;
  float m = 0.f;
  const int n = g.TX * g.TY;
  const int n4 = (reinterpret_cast<uintptr_t>(g.TM) & 15) ? 0 : n / 4;  // 16-byte vectors, then the tail
  const float4* tm4 = reinterpret_cast<const float4*>(g.TM);
  // the first TMV vectors of each thread are loaded before any is used, so their L2 latencies overlap (a plain
  // strided loop waits for each load before issuing the next)
  constexpr int TMV = 8;
  float4 v[TMV];
#pragma unroll
  for (int u = 0; u < TMV; ++u) {
    const int j = threadIdx.x + u * blockDim.x;
    v[u] = j < n4 ? tm4[j] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
#pragma unroll
  for (int u = 0; u < TMV; ++u) m = fmaxf(m, fmaxf(fmaxf(v[u].x, v[u].y), fmaxf(v[u].z, v[u].w)));
  for (int j = threadIdx.x + TMV * blockDim.x; j < n4; j += blockDim.x) {
    const float4 w = tm4[j];
    m = fmaxf(m, fmaxf(fmaxf(w.x, w.y), fmaxf(w.z, w.w)));
  }
  for (int j = 4 * n4 + threadIdx.x; j < n; j += blockDim.x) m = fmaxf(m, g.TM[j]);
  m = block_reduce_maxf(m);
  if (threadIdx.x == 0) {
    s_om = m;
    if (blockIdx.x == 0) g.sc->objMax = m;
  }
  __syncthreads();
  return 1.0f / s_om;
}

// Probe update of one pixel (a7) for the position at rounded offset (ox, oy): P_k += cP conj(O) dpsi_k, |P_k|^2
// cache, the pixel's contribution to the probe maximum.  Returns the updated mode-0 value.
__device__ __forceinline__ float2 ec_probe_pixel(const EpieChainArgs& g, size_t idx, int x, int y, int ox, int oy,
                                                 float cP, float& pmax) {
  const size_t NN = size_t(g.N) * g.N;
  const float2 oc = g.obj[size_t(x + ox) * g.Y + (y + oy)];
  float modal = 0.f;
  float2 p0 = make_float2(0.f, 0.f);
  for (int k = 0; k < g.K; ++k) {
    float cache;
    if (k < g.Ka) {
      const float2 u = cconjmul(oc, g.psi[k * NN + idx]);
      float2 pv = g.probe[k * NN + idx];
      pv = make_float2(u.x * cP + pv.x, u.y * cP + pv.y);
      const float mg = sqrtf(pv.x * pv.x + pv.y * pv.y);
      g.probe[k * NN + idx] = pv;
      if (k == 0) p0 = pv;
      cache = mg * mg;
      g.pcache[k * NN + idx] = cache;
    } else {
      cache = g.pcache[k * NN + idx];
    }
    if (g.useAll && g.K > 1)
      modal += cache;
    else
      pmax = fmaxf(pmax, cache);
  }
  if (g.useAll && g.K > 1) pmax = fmaxf(pmax, modal);
  return p0;
}

__device__ __forceinline__ void ec_probe_max(const EpieChainArgs& g, int sp, float pmax) {
  pmax = block_reduce_maxf(pmax);
  if (threadIdx.x == 0) atomicMax(reinterpret_cast<int*>(&g.pmax2[sp & 1]), __float_as_int(pmax));
}

// Probe update of position sp over this thread's grid-stride loop (the last position's, after the loop over
// positions).
__device__ void ec_probe_update(const EpieChainArgs& g, int sp) {
  const float cP = ec_object_step(g);
  const float2 q = g.pos[g.order[sp]];
  const int ox = int(roundf(q.x)), oy = int(roundf(q.y));
  const int N = g.N;
  const size_t NN = size_t(N) * N;
  float pmax = 0.f;
  for (size_t idx = blockIdx.x * size_t(blockDim.x) + threadIdx.x; idx < NN; idx += size_t(gridDim.x) * blockDim.x)
    ec_probe_pixel(g, idx, int(idx / N), int(idx % N), ox, oy, cP, pmax);
  ec_probe_max(g, sp, pmax);
}

// The global loads of one pixel of the exit kernel (one mode): the four bilinear taps of the patch and their weights,
// and for the probe update the object at the previous position, the returned dpsi and the probe.
struct ExitLoads {
  float2 v00, v01, v10, v11, oc, ps, pr;
  float wa, wb;
};
__device__ __forceinline__ void ec_exit_loads(const EpieChainArgs& g, float2 q, size_t idx, int pox, int poy,
                                              bool upd, ExitLoads& l) {
  const int x = int(idx / g.N), y = int(idx % g.N);
  int r0, r1, c0, c1;
  tex_axis(q.x, x, g.X, r0, r1, l.wb);
  tex_axis(q.y, y, g.Y, c0, c1, l.wa);
  l.v00 = g.obj[size_t(r0) * g.Y + c0];
  l.v01 = g.obj[size_t(r0) * g.Y + c1];
  l.v10 = g.obj[size_t(r1) * g.Y + c0];
  l.v11 = g.obj[size_t(r1) * g.Y + c1];
  if (upd) {
    l.oc = g.obj[size_t(x + pox) * g.Y + (y + poy)];
    l.ps = g.psi[idx];
  }
  l.pr = g.probe[idx];
}

// Exit waves of position s, with the previous position's probe update of the same pixel first (pixel-local: the
// thread that updates a probe pixel is the one that then multiplies it into the patch).
__global__ void k_ec_exit(EpieChainArgs g, int s) {
  // the visiting order and the positions stay fixed during an iteration (written before it starts): read before the
  // wait for the previous kernel, so their latency overlaps its tail
  const bool upd = g.up && s > 0;
  const float2 q = g.pos[g.order[s]];
  int pox = 0, poy = 0;
  if (upd) {
    const float2 pq = g.pos[g.order[s - 1]];
    pox = int(roundf(pq.x));
    poy = int(roundf(pq.y));
  }
  pdl_enter();
  const int N = g.N;
  const size_t NN = size_t(N) * N;
  const size_t start = blockIdx.x * size_t(blockDim.x) + threadIdx.x, stride = size_t(gridDim.x) * blockDim.x;
  float pmax = 0.f;
  if (g.K == 1 && g.Ka == 1) {
    // one mode: the loop is software-pipelined, the next pixel's loads issued before this pixel's stores (which
    // they would otherwise wait for: the compiler cannot tell that they do not alias); the first pixel's loads go
    // out before the object-maximum reduction, whose latency they then share
    ExitLoads cur{}, nxt{};
    if (start < NN) ec_exit_loads(g, q, start, pox, poy, upd, cur);
    const float cP = upd ? ec_object_step(g) : 0.f;
    if (g.up && blockIdx.x == 0 && threadIdx.x == 0) g.pmax2[s & 1] = 0.f;  // this position's probe maximum
    for (size_t idx = start; idx < NN; idx += stride) {
      if (idx + stride < NN) ec_exit_loads(g, q, idx + stride, pox, poy, upd, nxt);
      float2 pv = cur.pr;
      if (upd) {
        const float2 u = cconjmul(cur.oc, cur.ps);
        pv = make_float2(u.x * cP + pv.x, u.y * cP + pv.y);
        const float mg = sqrtf(pv.x * pv.x + pv.y * pv.y);
        g.probe[idx] = pv;
        g.pcache[idx] = mg * mg;
        pmax = fmaxf(pmax, mg * mg);
      }
      const float wa = cur.wa, wb = cur.wb;
      const float w00 = (1.f - wa) * (1.f - wb), w01 = wa * (1.f - wb), w10 = (1.f - wa) * wb, w11 = wa * wb;
      const float2 patch = make_float2(cur.v00.x * w00 + cur.v01.x * w01 + cur.v10.x * w10 + cur.v11.x * w11,
                                       cur.v00.y * w00 + cur.v01.y * w01 + cur.v10.y * w10 + cur.v11.y * w11);
      g.psi[idx] = cmul(patch, pv);
      cur = nxt;
    }
    if (upd) ec_probe_max(g, s - 1, pmax);
    return;
  }
  const float cP = upd ? ec_object_step(g) : 0.f;
  if (g.up && blockIdx.x == 0 && threadIdx.x == 0) g.pmax2[s & 1] = 0.f;  // this position's probe maximum
  for (size_t idx = start; idx < NN; idx += stride) {
    const int x = int(idx / N), y = int(idx % N);
    // the patch gathers first: the probe update's stores would otherwise hold them back (the compiler cannot move a
    // load of the object above a store through the probe pointers)
    int r0, r1, c0, c1;
    float wb, wa;
    tex_axis(q.x, x, g.X, r0, r1, wb);
    tex_axis(q.y, y, g.Y, c0, c1, wa);
    const float2 v00 = g.obj[size_t(r0) * g.Y + c0], v01 = g.obj[size_t(r0) * g.Y + c1];
    const float2 v10 = g.obj[size_t(r1) * g.Y + c0], v11 = g.obj[size_t(r1) * g.Y + c1];
    float2 p0 = make_float2(0.f, 0.f);
    if (upd) p0 = ec_probe_pixel(g, idx, x, y, pox, poy, cP, pmax);
    const float w00 = (1.f - wa) * (1.f - wb), w01 = wa * (1.f - wb), w10 = (1.f - wa) * wb, w11 = wa * wb;
    const float2 patch = make_float2(v00.x * w00 + v01.x * w01 + v10.x * w10 + v11.x * w11,
                                     v00.y * w00 + v01.y * w01 + v10.y * w10 + v11.y * w11);
    for (int k = 0; k < g.Ka; ++k) g.psi[k * NN + idx] = cmul(patch, (upd && k == 0) ? p0 : g.probe[k * NN + idx]);
  }
  if (upd) ec_probe_max(g, s - 1, pmax);
}

__global__ void k_ec_modulus(EpieChainArgs g, int s) {
  // the order and the amplitudes are fixed during an iteration: the thread's first amplitude and the pattern's sum
  // are loaded before the wait for the previous kernel
  const int i = g.order[s];
  const int N = g.N;
  const size_t NN = size_t(N) * N;
  const float nrm = 1.f / float(NN);
  const float* Ai = g.amp + size_t(i) * NN;  // natural layout, as psi: A(x, y) at [x N + y]
  const size_t start = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
  const float A0 = start < NN ? Ai[start] : 0.f;
  const double sq = g.rms ? double(g.sqsum[i]) : 1.0;
  pdl_enter();
  double err = 0.0;
  for (size_t idx = start; idx < NN; idx += size_t(gridDim.x) * blockDim.x) {
    const float A = idx == start ? A0 : Ai[idx];
    if (g.Ka == 1) {
      const float2 psi = g.psi[idx];
      if (g.rms) err += fabsf(A - sqrtf(psi.x * psi.x + psi.y * psi.y));
      float2 rep;
      if (A - g.saturation >= 0.f)
        rep = make_float2(psi.x * nrm, psi.y * nrm);  // floating pixel: no modulus
      else
        rep = modulus_replace(psi, A * nrm);
      g.psi[idx] = make_float2(rep.x - psi.x * nrm, rep.y - psi.y * nrm);
    } else {
      float tot = 0.f;
      float2 sum = make_float2(0.f, 0.f);
      for (int k = 0; k < g.Ka; ++k) {
        const float2 psi = g.psi[k * NN + idx];
        tot += psi.x * psi.x + psi.y * psi.y;
        sum = cadd(sum, psi);
      }
      if (g.rms) err += fabsf(A - sqrtf(sum.x * sum.x + sum.y * sum.y));
      const float sc = (tot > 0.f) ? ((A - g.saturation >= 0.f) ? 1.f : A) * rsqrtf(tot) * nrm : 0.f;
      for (int k = 0; k < g.Ka; ++k) {
        const float2 psi = g.psi[k * NN + idx];
        g.psi[k * NN + idx] = make_float2(psi.x * (sc - nrm), psi.y * (sc - nrm));
      }
    }
  }
  if (g.rms) {
    const double e = block_reduce_sum(err);
    if (threadIdx.x == 0) atomicAdd(&g.sc->err, e / double(g.Ka) / sq);
  }
}

// Object update and tile maxima in one pass: one block per 16 x 16 object tile under the patch; each thread updates
// its cell when the patch covers it (as k_ec_object), then the block writes the tile's maximum of |O|^2 (cells
// outside the patch unchanged) into TM
__global__ void __launch_bounds__(256) k_ec_object_tiles(EpieChainArgs g, int s) {
  const int i = g.order[s];  // order and positions are fixed during an iteration: read before the wait
  const float2 q = g.pos[i];
  const int ox = int(roundf(q.x)), oy = int(roundf(q.y)), N = g.N;
  const int tr0 = ox / 16, tc0 = oy / 16, ntc = (oy + N - 1) / 16 - tc0 + 1, ntr = (ox + N - 1) / 16 - tr0 + 1;
  pdl_enter();
  if (int(blockIdx.x) >= ntr * ntc) return;  // the grid covers the most tiles a patch can touch
  const int tr = tr0 + int(blockIdx.x) / ntc, tc = tc0 + int(blockIdx.x) % ntc;
  const int xr = tr * 16 + int(threadIdx.x) / 16, yc = tc * 16 + int(threadIdx.x) % 16;
  const size_t NN = size_t(N) * N;
  float m2 = 0.f;
  if (xr < g.X && yc < g.Y) {
    const size_t o_i = size_t(xr) * g.Y + yc;
    const int x = xr - ox, y = yc - oy;
    if (x >= 0 && x < N && y >= 0 && y < N) {
      const float pmax = (g.up && s > 0) ? g.pmax2[(s - 1) & 1] : g.sc->probeMax;
      const float cO = 1.0f / pmax;
      const size_t idx = size_t(x) * N + y;
      float2 inc = make_float2(0.f, 0.f);
      for (int k = 0; k < g.Ka; ++k) inc = cadd(inc, cconjmul(g.probe[k * NN + idx], g.psi[k * NN + idx]));
      float2 o = g.obj[o_i];
      o = make_float2(o.x + inc.x * cO, o.y + inc.y * cO);
      const float mag = sqrtf(o.x * o.x + o.y * o.y);
      if (g.pc) o = constrain_phase(o);
      g.obj[o_i] = o;
      m2 = mag * mag;
      g.ocache[o_i] = m2;
    } else {
      m2 = g.ocache[o_i];
    }
  }
  if (!g.up) return;  // the tile maxima are only consumed by the probe update
  m2 = block_reduce_maxf(m2);
  if (threadIdx.x == 0) g.TM[size_t(tr) * g.TY + tc] = m2;
}

// The last position's probe update and the probe maximum for the next iteration
__global__ void k_ec_finish(EpieChainArgs g) {
  pdl_enter();
  if (!g.up || g.P == 0) return;
  ec_probe_update(g, g.P - 1);
}

// One mode at L = 512: the second pass of the forward transform with the modulus step of k_ec_modulus in its
// epilogue (the same arithmetic per element, so the same result), one launch fewer per position.  The CTA transforms
// rows x0 .. x0 + R - 1 of the transposed work plane and stores columns x0 .. x0 + R - 1 of Psi in its natural layout;
// the amplitudes of those elements are fixed during the iteration, so each thread loads its share before the wait for
// the first pass (in the epilogue each load would wait for the previous element's store, which it might alias).
template <int L, int R>
__global__ void __launch_bounds__(R * FftShape<L>::T) k_ec_fwd2_modulus(EpieChainArgs g, int s) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, NT = R * T, KPT = L * R / NT;
  static_assert(NT % 32 == 0 && NT % R == 0, "whole warps, whole store rows");
  extern __shared__ float4 smem4[];
  float2* s_tw = reinterpret_cast<float2*>(smem4);
  float2* s_x = s_tw + L;
  load_twiddles<L>(s_tw, g.tw);
  const int i = g.order[s];
  const int x0 = int(blockIdx.x) * R;
  const int v = threadIdx.x / T, t = threadIdx.x % T;  // transform: row x0 + v, lane t
  const int vv = threadIdx.x % R, n0 = threadIdx.x / R;  // store: column x0 + vv, rows n0 + T k
  const float* Ai = g.amp + size_t(i) * L * L + x0 + vv;
  float Av[KPT];
#pragma unroll
  for (int k = 0; k < KPT; ++k) Av[k] = Ai[size_t(n0 + k * T) * L];
  const double sq = g.rms ? g.sqsum[i] : 1.0;
  pdl_enter();
  __syncthreads();  // twiddles
  float2 a[E];
  const float2* wrow = g.work + size_t(x0 + v) * L;
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = wrow[t + T * e];
  fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
  __syncthreads();  // the staging tile aliases the exchange buffers of other warps
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    s_x[(t + T * e) * (R + 1) + v] = a[out_slot<L>(e)];
  });
  __syncthreads();
  const float nrm = 1.f / float(L * L);
  double err = 0.0;
#pragma unroll
  for (int k = 0; k < KPT; ++k) {
    const int n = n0 + k * T;
    const float2 psi = s_x[n * (R + 1) + vv];
    const float A = Av[k];
    if (g.rms) err += fabsf(A - sqrtf(psi.x * psi.x + psi.y * psi.y));
    float2 rep;
    if (A - g.saturation >= 0.f)
      rep = make_float2(psi.x * nrm, psi.y * nrm);  // floating pixel: no modulus
    else
      rep = modulus_replace(psi, A * nrm);
    g.psi[size_t(n) * L + x0 + vv] = make_float2(rep.x - psi.x * nrm, rep.y - psi.y * nrm);
  }
  if (g.rms) {
    const double e = block_reduce_sum(err);
    if (threadIdx.x == 0) atomicAdd(&g.sc->err, e / sq);
  }
}

// The forward transform of one mode at 512^2 with the modulus step fused into its second pass (R rows per CTA).
template <int R>
cudaError_t ec_forward_modulus(const EpieChainArgs& g, int s, cudaStream_t st) {
  constexpr int L = 512;
  cudaError_t e = launch_fftx<L, false, R>(g.work, g.tw, 1, ProLoad{g.psi}, EpiStore{}, st);
  if (e != cudaSuccess) return e;
  return launch_pdl(k_ec_fwd2_modulus<L, R>, dim3(L / R), R * FftShape<L>::T, rows_smem_bytes_r<L, R>(), st, g, s);
}

__global__ void k_ec_scalars(EpieChainArgs g) {
  pdl_enter();
  if (threadIdx.x == 0 && blockIdx.x == 0 && g.up && g.P > 0) g.sc->probeMax = g.pmax2[(g.P - 1) & 1];
}

}  // namespace

namespace {
// rows per CTA of the FP32 transform passes (g.frows; 0: 4 at 512^2, where one plane's 512 rows then spread over
// 128 CTAs instead of 64: 35.0 against 36.6 ms per 900-position iteration; the default tile elsewhere)
int ec_rows(const EpieChainArgs& g) { return g.frows > 0 ? g.frows : (g.N == 512 ? 4 : 0); }
// one mode at 512^2 with FP32 transforms of 2, 4 or 8 rows per CTA: the modulus step runs in the second forward pass
bool ec_fused_modulus(const EpieChainArgs& g) {
  const int rows = ec_rows(g);
  return !g.tc && g.K == 1 && g.Ka == 1 && g.N == 512 && (rows == 2 || rows == 4 || rows == 8);
}
}  // namespace

cudaError_t epie_chain_iteration(const EpieChainArgs& g, cudaStream_t st) {
  const size_t NN = size_t(g.N) * g.N;
  const int gb = grid_e(NN);
  const int tiles = ((g.N + 15) / 16 + 1) * ((g.N + 15) / 16 + 1);
  cudaError_t e;
  const int rows = ec_rows(g);
  const bool fused = ec_fused_modulus(g);
  auto fft = [&](bool inv) -> cudaError_t {
    if (g.tc) return fft2_tc(g.psi, g.work, g.Ka, g.N, inv, g.tcerr, st);
    const ProLoad pl{g.psi};
    switch (rows) {
      case 2:
        return inv ? fftx2<true, ProLoad, EpiStore, 2>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st)
                   : fftx2<false, ProLoad, EpiStore, 2>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st);
      case 4:
        return inv ? fftx2<true, ProLoad, EpiStore, 4>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st)
                   : fftx2<false, ProLoad, EpiStore, 4>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st);
      case 8:
        return inv ? fftx2<true, ProLoad, EpiStore, 8>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st)
                   : fftx2<false, ProLoad, EpiStore, 8>(g.N, g.work, g.psi, g.tw, g.Ka, pl, EpiStore{}, st);
      default:
        return fft2_pdl(g.psi, g.work, g.tw, g.Ka, g.N, inv, st);
    }
  };
  // the exit kernel carries the previous position's probe update, whose blocks each reduce the tile maxima of the
  // whole object first: two blocks per SM keep that reduction from dominating its one-pixel-per-thread work
  int sms = 148;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int gx = g.up ? std::min(gb, 2 * sms) : gb;
  for (int s = 0; s < g.P; ++s) {
    if ((e = launch_pdl(k_ec_exit, gx, 256, 0, st, g, s)) != cudaSuccess) return e;
    if (fused) {
      e = rows == 2 ? ec_forward_modulus<2>(g, s, st) : rows == 4 ? ec_forward_modulus<4>(g, s, st)
                                                              : ec_forward_modulus<8>(g, s, st);
      if (e != cudaSuccess) return e;
    } else {
      if ((e = fft(false)) != cudaSuccess) return e;
      if ((e = launch_pdl(k_ec_modulus, gb, 256, 0, st, g, s)) != cudaSuccess) return e;
    }
    if ((e = fft(true)) != cudaSuccess) return e;
    // one block per tile the patch touches: the tile count depends on the position's offset within a tile, so the
    // grid covers the most a patch can touch and blocks past this position's tiles return
    if ((e = launch_pdl(k_ec_object_tiles, tiles, 256, 0, st, g, s)) != cudaSuccess) return e;
  }
  if ((e = launch_pdl(k_ec_finish, gx, 256, 0, st, g)) != cudaSuccess) return e;
  return launch_pdl(k_ec_scalars, 1, 32, 0, st, g);
}

int epie_chain_launches(const EpieChainArgs& g) { return g.P * (ec_fused_modulus(g) ? 6 : 7) + 2; }

}  // namespace pty
