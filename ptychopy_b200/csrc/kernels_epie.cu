// ePIE (src/ePIE.cpp:65-129) as ONE persistent kernel: a single thread-block cluster of C CTAs walks the
// seeded visiting order serially; each position is five phases separated by cluster barriers.  The CTAs split
// rows (row phases) and columns (column phase) of the N x N window; intermediates live in two small global
// buffers that stay in L2 (Ka*N*N complex each).
//
//   A  rows     patch = bilinear O at (x+qx, y+qy) with 1/256-quantised weights (texture fetch,
//               src/SampleKernels.cu:167-178), psi_old_k = patch * P_k (src/CXMath.h:49-58), FFT along y,
//               stored transposed: W1[k][ky][x]
//   B  columns  FFT along x, error term |A - |sum_k Psi_k|| (src/utilitiesKernels.cu:684-712), modulus
//               (d_adjustFFT / d_adjustModalFFT, src/utilitiesKernels.cu:633-682), D_k = Psi'_k - Psi_k/N^2,
//               inverse FFT along x, stored transposed: W2[k][x][ky]
//   C  rows     inverse FFT along y gives dpsi_k = psi_k - psi_old_k; object update at the rounded offset
//               O += (1/probeMax) sum_k conj(P_k) dpsi_k, phase clamp, |O|^2 cache (src/SampleKernels.cu:244-294)
//   D  tiles    16x16 tile maxima of the |O|^2 cache are refreshed where the patch touched them; every CTA
//               then takes the max over all tiles = max |O|^2 over the whole object (src/Sample.cpp:340-345)
//   E  rows     probe update P_k += (1/objMax) conj(O_new) dpsi_k and |P_k|^2 cache (src/ProbeKernels.cu:425-458),
//               per-CTA partial of Probe::getModalDoubleMax, combined after the barrier
//
// Cluster barriers (barrier.cluster arrive.release / wait.acquire) order the global-memory hand-offs at cluster
// scope.  For 512 x 512 windows the same kernel runs as a whole-GPU cooperative launch of 128 CTAs whose phases are
// separated by a device-scope grid barrier with a bounded wait (k_epie<L, R, true>).
#include <cooperative_groups.h>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels_epie.h"

namespace cg = cooperative_groups;

namespace pty {

// barrier.cluster.arrive (release) + barrier.cluster.wait (acquire): cluster-scope ordering of the global and
// shared memory the CTAs hand to each other.  Every hand-off of this kernel stays inside its single cluster, so no
// device-scope fence is needed.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}


// Device-scope barrier over all CTAs of a cooperative launch (the whole-GPU variant): arrival count bar[0],
// generation bar[1].  Thread 0 publishes its CTA's writes (fence), arrives, and the last arrival resets the count and
// advances the generation; the others poll the generation (bounded: after EPIE_GRID_WAIT polls the CTA records
// code 1 in *err and reports failure, so every CTA returns instead of waiting for good).
constexpr unsigned EPIE_GRID_WAIT = 1u << 24;
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err, unsigned expected = 0,
                                             unsigned limit = EPIE_GRID_WAIT) {
  if (expected == 0) expected = gridDim.x;
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    int ok = 1;
    __threadfence();
    if (atomicAdd(bar, 1u) + 1u == expected) {
      bar[0] = 0;
      __threadfence();
      atomicExch(bar + 1, gen + 1u);
    } else {
      unsigned n = 0;
      while (*vgen == gen) {
        if (++n > limit) {
          ok = 0;
          atomicCAS(err, 0, 1);
          break;
        }
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// GRID = false: one thread-block cluster (cluster barriers); GRID = true: all CTAs of a cooperative launch spread
// over the GPU (grid barriers).  The phases, their work split (CTA c of C takes rows / columns [c L/C, (c+1) L/C))
// and the global hand-offs are the same.
template <int L, int R, bool GRID>
__global__ void __launch_bounds__(R* FftShape<L>::T) k_epie(EpieArgs g) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E;
  constexpr float nrm = 1.0f / float(L * L);
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  float2* s_tw = smem;
  float2* s_x = smem + L;                                   // exchange / staging
  float* s_m2 = reinterpret_cast<float*>(s_x + (R * S::XCH > L * (R + 1) ? R * S::XCH : L * (R + 1)));  // R*L
  float2* s_sum = reinterpret_cast<float2*>(s_m2 + R * L);  // R*L (error metric, Ka > 1)
  __shared__ float s_objmax, s_probemax;

  const int c = GRID ? int(blockIdx.x) : int(cg::this_cluster().block_rank());
  const int C = g.C;
  // phase separator; false only when a grid barrier timed out (then every CTA leaves the kernel)
  auto sync_all = [&]() -> bool {
    if constexpr (GRID) {
      return grid_barrier(g.gbar, g.gerr);
    } else {
      cluster_barrier();
      return true;
    }
  };
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  const int rows_cta = L / C, passes = rows_cta / R;
  const int Ka = g.Ka;
  const size_t NN = size_t(L) * L;
  const int nthreads = R * T;
  load_twiddles<L>(s_tw, g.tw);
  if (threadIdx.x == 0) {
    s_objmax = g.sc->objMax;
    s_probemax = g.sc->probeMax;
  }
  __syncthreads();
  double err_acc = 0.0;

  for (int s = 0; s < g.P; ++s) {
    const int i = g.order[s];
    const float2 q = g.pos[i];
    const int ox = int(roundf(q.x)), oy = int(roundf(q.y));
    const float* Ai = g.ampT + size_t(i) * NN;

    // ---------------- A: bilinear patch * probe modes, row FFT, transposed store into W1 -------------------
    for (int ps = 0; ps < passes; ++ps) {
      const int x0 = c * rows_cta + ps * R, x = x0 + v;
      int r0, r1;
      float wb;
      tex_axis(q.x, x, g.X, r0, r1, wb);
      float2 patch[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int y = t + T * e;
        int c0, c1;
        float wa;
        tex_axis(q.y, y, g.Y, c0, c1, wa);
        const float2 v00 = g.obj[size_t(r0) * g.Y + c0], v01 = g.obj[size_t(r0) * g.Y + c1];
        const float2 v10 = g.obj[size_t(r1) * g.Y + c0], v11 = g.obj[size_t(r1) * g.Y + c1];
        const float w00 = (1.f - wa) * (1.f - wb), w01 = wa * (1.f - wb), w10 = (1.f - wa) * wb, w11 = wa * wb;
        patch[e] = make_float2(v00.x * w00 + v01.x * w01 + v10.x * w10 + v11.x * w11,
                               v00.y * w00 + v01.y * w01 + v10.y * w10 + v11.y * w11);
      }
      for (int k = 0; k < Ka; ++k) {
        const float2* prow = g.probe + size_t(k) * NN + size_t(x) * L;
        float2 a[E];
#pragma unroll
        for (int e = 0; e < E; ++e) a[e] = cmul(patch[e], prow[t + T * e]);
        fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
        store_rows_transposed<L, R>(a, g.W1 + size_t(k) * NN, x0, v, t, s_x);
      }
    }
    if (!sync_all()) return;

    // ---------------- B: column FFT, modulus, inverse column FFT, transposed store into W2 -------------------
    for (int ps = 0; ps < passes; ++ps) {
      const int k0 = c * rows_cta + ps * R, ky = k0 + v;
      const float* arow = Ai + size_t(ky) * L;
      if (Ka == 1) {
        float2 a[E];
        const float2* row = g.W1 + size_t(ky) * L;
#pragma unroll
        for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
        fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
        static_for<0, E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          const float A = arow[t + T * e];
          const float2 psi = a[out_slot<L>(e)];
          if (g.rms) err_acc += fabsf(A - sqrtf(psi.x * psi.x + psi.y * psi.y));
          float2 rep;
          if (A - g.saturation >= 0.f)
            rep = make_float2(psi.x * nrm, psi.y * nrm);  // floating pixel: no modulus
          else
            rep = modulus_replace(psi, A * nrm);
          a[out_slot<L>(e)] = make_float2(rep.x - psi.x * nrm, rep.y - psi.y * nrm);
        });
        to_input_order<L>(a);
        fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
        store_rows_transposed<L, R>(a, g.W2, k0, v, t, s_x);
      } else {
        float* m2 = s_m2 + v * L;
        float2* sm = s_sum + v * L;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          m2[t + T * e] = 0.f;
          sm[t + T * e] = make_float2(0.f, 0.f);
        }
        for (int k = 0; k < Ka; ++k) {
          float2 a[E];
          float2* row = g.W1 + size_t(k) * NN + size_t(ky) * L;
#pragma unroll
          for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
          fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
          static_for<0, E>([&](auto ec) {
            constexpr int e = decltype(ec)::value;
            const int n = t + T * e;
            const float2 psi = a[out_slot<L>(e)];
            row[n] = psi;  // spectrum kept in place for the second sweep
            m2[n] += psi.x * psi.x + psi.y * psi.y;
            sm[n] = cadd(sm[n], psi);
          });
        }
        if (g.rms) {
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int n = t + T * e;
            const float2 z = sm[n];
            err_acc += fabsf(arow[n] - sqrtf(z.x * z.x + z.y * z.y));
          }
        }
        for (int k = 0; k < Ka; ++k) {
          float2 a[E];
          const float2* row = g.W1 + size_t(k) * NN + size_t(ky) * L;
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int n = t + T * e;
            const float2 psi = row[n];
            const float A = arow[n];
            const float tot = m2[n];
            const float sc = (tot > 0.f) ? ((A - g.saturation >= 0.f) ? 1.f : A) * rsqrtf(tot) * nrm : 0.f;
            a[e] = make_float2(psi.x * (sc - nrm), psi.y * (sc - nrm));
          }
          fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
          store_rows_transposed<L, R>(a, g.W2 + size_t(k) * NN, k0, v, t, s_x);
        }
      }
    }
    if (g.rms) {
      // per-position error: (sum over pixels)/Ka/sqsum_i, summed over CTAs
      double e = block_reduce_sum(err_acc);
      if (threadIdx.x == 0) atomicAdd(&g.sc->err, e / double(Ka) / double(g.sqsum[i]));
      err_acc = 0.0;
    }
    if (!sync_all()) return;

    // ---------------- C: inverse row FFT -> dpsi; object update; |O|^2 cache ----------------------------
    const float cO = 1.0f / s_probemax;
    for (int ps = 0; ps < passes; ++ps) {
      const int x0 = c * rows_cta + ps * R, x = x0 + v;
      float2 inc[E];
#pragma unroll
      for (int e = 0; e < E; ++e) inc[e] = make_float2(0.f, 0.f);
      for (int k = 0; k < Ka; ++k) {
        float2 a[E];
        const float2* row = g.W2 + size_t(k) * NN + size_t(x) * L;
#pragma unroll
        for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
        fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
        const float2* prow = g.probe + size_t(k) * NN + size_t(x) * L;
        float2* drow = g.W1 + size_t(k) * NN + size_t(x) * L;
        static_for<0, E>([&](auto ec) {
          constexpr int e = decltype(ec)::value;
          const int n = t + T * e;
          const float2 d = a[out_slot<L>(e)];
          if (g.up) drow[n] = d;
          inc[e] = cadd(inc[e], cconjmul(prow[n], d));
        });
      }
      float2* orow = g.obj + size_t(x + ox) * g.Y + oy;
      float* crow = g.ocache + size_t(x + ox) * g.Y + oy;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int n = t + T * e;
        float2 o = orow[n];
        o = make_float2(o.x + inc[e].x * cO, o.y + inc[e].y * cO);
        const float mag = sqrtf(o.x * o.x + o.y * o.y);
        if (g.pc) o = constrain_phase(o);
        orow[n] = o;
        crow[n] = mag * mag;
      }
    }
    if (!sync_all()) return;

    if (!g.up) continue;  // the object max is only consumed by the probe update

    // ---------------- D: refresh tile maxima under the patch, then the global object max ---------------------
    {
      const int tr0 = ox / 16, tr1 = (ox + L - 1) / 16, tc0 = oy / 16, tc1 = (oy + L - 1) / 16;
      const int ntc = tc1 - tc0 + 1, ntiles = (tr1 - tr0 + 1) * ntc;
      const int warps = nthreads / 32, gw = c * warps + int(threadIdx.x / 32), lane = threadIdx.x & 31;
      for (int tile = gw; tile < ntiles; tile += C * warps) {
        const int tr = tr0 + tile / ntc, tc = tc0 + tile % ntc;
        float m = 0.f;
        for (int j = lane; j < 256; j += 32) {
          const int xr = tr * 16 + j / 16, yc = tc * 16 + j % 16;
          if (xr < g.X && yc < g.Y) m = fmaxf(m, g.ocache[size_t(xr) * g.Y + yc]);
        }
        m = warp_reduce_maxf(m);
        if (lane == 0) g.TM[size_t(tr) * g.TY + tc] = m;
      }
    }
    if (!sync_all()) return;
    {
      float m = 0.f;
      const int nt = g.TX * g.TY;
      for (int j = threadIdx.x; j < nt; j += nthreads) m = fmaxf(m, g.TM[j]);
      m = block_reduce_maxf(m);
      if (threadIdx.x == 0) s_objmax = m;
      __syncthreads();
    }

    // ---------------- E: probe update and the modal max of the probe intensity cache -----------------------
    {
      const float cP = 1.0f / s_objmax;
      float pmax = 0.f;
      for (int ps = 0; ps < passes; ++ps) {
        const int x0 = c * rows_cta + ps * R, x = x0 + v;
        const float2* orow = g.obj + size_t(x + ox) * g.Y + oy;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int n = t + T * e;
          const float2 oc = orow[n];
          float modal = 0.f;
          for (int k = 0; k < g.K; ++k) {
            const size_t idx = size_t(k) * NN + size_t(x) * L + n;
            float cache;
            if (k < Ka) {
              const float2 d = g.W1[idx];
              const float2 u = cconjmul(oc, d);
              float2 pv = g.probe[idx];
              pv = make_float2(u.x * cP + pv.x, u.y * cP + pv.y);
              const float mg = sqrtf(pv.x * pv.x + pv.y * pv.y);
              g.probe[idx] = pv;
              cache = mg * mg;
              g.pcache[idx] = cache;
            } else {
              cache = g.pcache[idx];
            }
            if (g.useAll && g.K > 1)
              modal += cache;
            else
              pmax = fmaxf(pmax, cache);
          }
          if (g.useAll && g.K > 1) pmax = fmaxf(pmax, modal);
        }
      }
      // partial maxima double-buffered by position parity: the next position writes the other half, and the one
      // after it cannot reach this half before every CTA has passed the next position's first barrier, i.e. has
      // read it here
      float* pm = g.pm + (s & 1) * 256;
      pmax = block_reduce_maxf(pmax);
      if (threadIdx.x == 0) pm[c] = pmax;
      if (!sync_all()) return;
      if (threadIdx.x == 0) {
        float m = 0.f;
        for (int j = 0; j < C; ++j) m = fmaxf(m, pm[j]);
        s_probemax = m;
      }
      __syncthreads();
    }
  }
  if (c == 0 && threadIdx.x == 0) {
    g.sc->objMax = s_objmax;
    g.sc->probeMax = s_probemax;
  }
}

// ---- shared-memory-resident ePIE for windows of L <= 128 with one probe mode -----------------------------------
// A cluster of C = L/32 CTAs; CTA c owns rows [32c, 32c+32) of the window (and of the probe, which stays in its
// shared memory for the whole launch) and columns [32c, 32c+32) of the column phase.  The row phase writes the row
// spectra into the CTA's own slab; the column phase gathers its columns from every CTA's slab through distributed
// shared memory (row r lives in CTA r/32), transforms, applies the modulus and writes the columns back in place; the inverse row phase reads the slab locally.  The amplitudes of the next position's
// columns are copied into shared memory (cp.async, natural layout) while the current position runs.  Per position:
// A rows -> barrier -> B columns -> barrier -> C rows (object update) -> barrier [-> D tile maxima -> barrier ->
// E probe update in shared memory].  Same equations and order as k_epie (src/ePIE.cpp:65-129).
template <int L>
struct EpieSm {
  static constexpr int T = FftShape<L>::T, E = FftShape<L>::E, R = 32, C = L / 32, NT = R * T;
  static constexpr int XROWS = R * FftShape<L>::XCH, XCOLS = cols_xch_elems<L>();
  static constexpr int XS = XROWS > XCOLS ? XROWS : XCOLS;
  // float2 units: tw | probe | slab | xch, then 2 amplitude buffers (floats)
  static constexpr size_t SMEM = sizeof(float2) * (L + 2 * size_t(R) * L + XS) + sizeof(float) * 2 * size_t(L) * 32;
  static_assert(cols_threads<L>() == NT, "column phase uses the CTA's threads");
  static_assert(cols_per_block<L>() == 32, "32 columns per CTA");
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory"); }

// This CTA's 32 amplitude columns of pattern i (natural layout A[kx][ky]) into dst[kx*32 + cc].
template <int L>
__device__ __forceinline__ void epie_sm_fetch_amp(const float* __restrict__ amp, int i, int c, float* dst) {
  constexpr int CHUNKS = L * 8;  // L rows x 128 bytes
  const float* src = amp + size_t(i) * L * L + 32 * c;
  for (int q = threadIdx.x; q < CHUNKS; q += EpieSm<L>::NT) {
    const int kx = q >> 3, part = q & 7;
    cp_async16(dst + kx * 32 + part * 4, src + size_t(kx) * L + part * 4);
  }
  cp_async_commit();
}

template <int L>
__global__ void __launch_bounds__(EpieSm<L>::NT) k_epie_sm(EpieArgs g) {
  using S = FftShape<L>;
  using Z = EpieSm<L>;
  constexpr int T = Z::T, E = Z::E, R = Z::R;
  constexpr float nrm = 1.0f / float(L * L);
  extern __shared__ float4 smem4[];
  float2* s_tw = reinterpret_cast<float2*>(smem4);
  float2* s_probe = s_tw + L;
  float2* s_slab = s_probe + R * L;
  float2* s_x = s_slab + R * L;
  float* s_amp = reinterpret_cast<float*>(s_x + Z::XS);  // 2 x L x 32
  __shared__ float s_objmax, s_probemax, s_pmpart;

  cg::cluster_group cl = cg::this_cluster();
  const int c = int(cl.block_rank());
  const int v = threadIdx.x / T, t = threadIdx.x % T;  // row phases: local row v, lane t
  int s, cc;                                            // column phase
  cols_thread<L>(threadIdx.x, s, cc);
  const int col = 32 * c + cc;
  const int x = 32 * c + v;

  load_twiddles<L>(s_tw, g.tw);
#pragma unroll
  for (int e = 0; e < E; ++e) s_probe[v * L + t + T * e] = g.probe[size_t(x) * L + t + T * e];
  if (threadIdx.x == 0) {
    s_objmax = g.sc->objMax;
    s_probemax = g.sc->probeMax;
    s_pmpart = 0.f;
  }
  bool pm_valid = false;
  if (g.P > 0) epie_sm_fetch_amp<L>(g.amp, g.order[0], c, s_amp);
  __syncthreads();
  cluster_barrier();  // every CTA of the cluster is running before any distributed shared memory access
  double err_acc = 0.0;
  float2 onew[E];

  for (int si = 0; si < g.P; ++si) {
    const int i = g.order[si];
    const float2 q = g.pos[i];
    const int ox = int(roundf(q.x)), oy = int(roundf(q.y));
    const float* s_A = s_amp + (si & 1) * L * 32;
    if (si + 1 < g.P)
      epie_sm_fetch_amp<L>(g.amp, g.order[si + 1], c, s_amp + ((si + 1) & 1) * L * 32);
    else
      cp_async_commit();  // keep one group per position so the wait below stays uniform

    // ---------------- A: bilinear patch * probe, row FFT into the slab -------------------------------------------
    {
      int r0, r1;
      float wb;
      tex_axis(q.x, x, g.X, r0, r1, wb);
      float2 a[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int y = t + T * e;
        int c0, c1;
        float wa;
        tex_axis(q.y, y, g.Y, c0, c1, wa);
        const float2 v00 = g.obj[size_t(r0) * g.Y + c0], v01 = g.obj[size_t(r0) * g.Y + c1];
        const float2 v10 = g.obj[size_t(r1) * g.Y + c0], v11 = g.obj[size_t(r1) * g.Y + c1];
        const float w00 = (1.f - wa) * (1.f - wb), w01 = wa * (1.f - wb), w10 = (1.f - wa) * wb, w11 = wa * wb;
        const float2 pt = make_float2(v00.x * w00 + v01.x * w01 + v10.x * w10 + v11.x * w11,
                                      v00.y * w00 + v01.y * w01 + v10.y * w10 + v11.y * w11);
        a[e] = cmul(pt, s_probe[v * L + y]);
      }
      fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        s_slab[v * L + t + T * e] = a[out_slot<L>(e)];
      });
    }
    cluster_barrier();

    // ---------------- B: columns through distributed shared memory: FFT, modulus, inverse FFT ----------------
    {
      float2 a[E];
      float2* src[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int r = s + T * e;
        src[e] = cl.map_shared_rank(s_slab, r / 32) + (r % 32) * L + col;
        a[e] = *src[e];
      }
      cp_async_wait<1>();  // this position's amplitudes (the next position's copy may still be in flight)
      fft_cols<L, false>(a, s, cc, s_x, s_tw);  // its first barrier publishes every thread's amplitude copies
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const float A = s_A[(s + T * e) * 32 + cc];
        const float2 psi = a[out_slot<L>(e)];
        if (g.rms) err_acc += fabsf(A - sqrtf(psi.x * psi.x + psi.y * psi.y));
        float2 rep;
        if (A - g.saturation >= 0.f)
          rep = make_float2(psi.x * nrm, psi.y * nrm);  // floating pixel: no modulus
        else
          rep = modulus_replace(psi, A * nrm);
        a[out_slot<L>(e)] = make_float2(rep.x - psi.x * nrm, rep.y - psi.y * nrm);
      });
      to_input_order<L>(a);
      fft_cols<L, true>(a, s, cc, s_x, s_tw);
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        *src[e] = a[out_slot<L>(e)];
      });
      if (g.rms) {
        const double er = block_reduce_sum(err_acc);
        if (threadIdx.x == 0) atomicAdd(&g.sc->err, er / double(g.sqsum[i]));
        err_acc = 0.0;
      }
    }
    cluster_barrier();

    // ---------------- C: inverse row FFT, dpsi, object update (global), |O|^2 cache -------------------------
    {
      if (pm_valid && threadIdx.x == 0) {  // probe maximum after the previous position's probe update
        float m = 0.f;
        for (int r = 0; r < Z::C; ++r) m = fmaxf(m, *cl.map_shared_rank(&s_pmpart, r));
        s_probemax = m;
      }
      float2* orow = g.obj + size_t(x + ox) * g.Y + oy;
      float* crow = g.ocache + size_t(x + ox) * g.Y + oy;
      float2 a[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        onew[e] = orow[t + T * e];
        a[e] = s_slab[v * L + t + T * e];
      }
      fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
      __syncthreads();  // s_probemax
      const float cO = 1.0f / s_probemax;
      static_for<0, E>([&](auto ec) {
        constexpr int e = decltype(ec)::value;
        const int n = t + T * e;
        const float2 pv = s_probe[v * L + n];
        const float2 d = a[out_slot<L>(e)];  // IFFT2(Psi' - Psi/N^2) = psi_new - psi_old
        s_slab[v * L + n] = d;
        const float2 inc = cconjmul(pv, d);
        float2 o = make_float2(onew[e].x + inc.x * cO, onew[e].y + inc.y * cO);
        const float mag = sqrtf(o.x * o.x + o.y * o.y);
        if (g.pc) o = constrain_phase(o);
        orow[n] = o;
        crow[n] = mag * mag;
        onew[e] = o;
      });
    }
    cluster_barrier();  // object writes visible to every CTA (next patch, tile maxima)
    if (!g.up) continue;

    // ---------------- D: refresh tile maxima under the patch, then the global object max ---------------------
    {
      const int tr0 = ox / 16, tr1 = (ox + L - 1) / 16, tc0 = oy / 16, tc1 = (oy + L - 1) / 16;
      const int ntc = tc1 - tc0 + 1, ntiles = (tr1 - tr0 + 1) * ntc;
      const int warps = Z::NT / 32, gw = c * warps + int(threadIdx.x / 32), lane = threadIdx.x & 31;
      for (int tile = gw; tile < ntiles; tile += Z::C * warps) {
        const int tr = tr0 + tile / ntc, tcc = tc0 + tile % ntc;
        float m = 0.f;
        for (int j = lane; j < 256; j += 32) {
          const int xr = tr * 16 + j / 16, yc = tcc * 16 + j % 16;
          if (xr < g.X && yc < g.Y) m = fmaxf(m, g.ocache[size_t(xr) * g.Y + yc]);
        }
        m = warp_reduce_maxf(m);
        if (lane == 0) g.TM[size_t(tr) * g.TY + tcc] = m;
      }
    }
    cluster_barrier();
    {
      float m = 0.f;
      const int nt = g.TX * g.TY;
      for (int j = threadIdx.x; j < nt; j += Z::NT) m = fmaxf(m, g.TM[j]);
      m = block_reduce_maxf(m);
      if (threadIdx.x == 0) s_objmax = m;
      __syncthreads();
    }

    // ---------------- E: probe update in shared memory, partial max of |P|^2 --------------------------------
    {
      const float cP = 1.0f / s_objmax;
      float pmax = 0.f;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int n = t + T * e;
        const float2 u = cconjmul(onew[e], s_slab[v * L + n]);
        float2 pv = s_probe[v * L + n];
        pv = make_float2(u.x * cP + pv.x, u.y * cP + pv.y);
        const float mg = sqrtf(pv.x * pv.x + pv.y * pv.y);
        s_probe[v * L + n] = pv;
        pmax = fmaxf(pmax, mg * mg);
      }
      pmax = block_reduce_maxf(pmax);
      if (threadIdx.x == 0) s_pmpart = pmax;
      pm_valid = true;
    }
  }
  cp_async_wait<0>();
  cluster_barrier();  // last partial maxima written
  if (threadIdx.x == 0 && pm_valid) {
    float m = 0.f;
    for (int r = 0; r < Z::C; ++r) m = fmaxf(m, *cl.map_shared_rank(&s_pmpart, r));
    s_probemax = m;
  }
  __syncthreads();
  // probe rows and their |P|^2 cache back to global memory
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = t + T * e;
    const float2 pv = s_probe[v * L + n];
    const float mg = sqrtf(pv.x * pv.x + pv.y * pv.y);
    g.probe[size_t(x) * L + n] = pv;
    g.pcache[size_t(x) * L + n] = mg * mg;
  }
  if (c == 0 && threadIdx.x == 0) {
    g.sc->objMax = s_objmax;
    g.sc->probeMax = s_probemax;
  }
  cluster_barrier();  // no CTA leaves while another may still read its shared memory
}

bool epie_uses_smem(int N, int K) { return K == 1 && (N == 32 || N == 64 || N == 128); }

template <int L>
static cudaError_t epie_sm_prepare_t() {
  return cudaFuncSetAttribute(k_epie_sm<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(EpieSm<L>::SMEM));
}

template <int L>
static cudaError_t epie_sm_launch_t(const EpieArgs& g, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(EpieSm<L>::C);
  cfg.blockDim = dim3(EpieSm<L>::NT);
  cfg.dynamicSmemBytes = EpieSm<L>::SMEM;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = EpieSm<L>::C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_epie_sm<L>, g);
}

cudaError_t epie_sm_prepare(int N) {
  switch (N) {
    case 32: return epie_sm_prepare_t<32>();
    case 64: return epie_sm_prepare_t<64>();
    case 128: return epie_sm_prepare_t<128>();
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t epie_sm_launch(const EpieArgs& g, cudaStream_t st) {
  switch (g.N) {
    case 32: return epie_sm_launch_t<32>(g, st);
    case 64: return epie_sm_launch_t<64>(g, st);
    case 128: return epie_sm_launch_t<128>(g, st);
    default: return cudaErrorInvalidValue;
  }
}

// Rows per pass of a CTA (blockDim = R * T) for a length-L window; the cluster takes the largest size (<= 16)
// whose CTAs hold whole passes.  Each position is a chain of short latency-bound phases: at L = 128, 4 CTAs of 8
// warps (R = 32) measured no faster than 16 CTAs of 2 warps (3.43 vs 3.21 ms per 100-position iteration).  At
// L = 256 with 5 modes (2601 positions): R = 8 / 16 / 32 measured 415 / 237 / 308 ms per iteration.
template <int L> struct EpieShape;
template <> struct EpieShape<32> { static constexpr int R = 8; };
template <> struct EpieShape<64> { static constexpr int R = 4; };
template <> struct EpieShape<128> { static constexpr int R = 8; };
template <> struct EpieShape<256> { static constexpr int R = 16; };
template <> struct EpieShape<512> { static constexpr int R = 16; };

// Whole-GPU variant: one pass of R rows per CTA, C = L / R CTAs in a cooperative launch (the default at 512; at 256 only
// when the autotuner asks for it).  At 512 (900 positions, 1 mode) R = 2 / 4 / 8 measured 50.6 / 47.4 / 47.0 ms per
// iteration: the phases' latency chains, not the CTA count, bound it.
// Measured per 900-position iteration at 512^2: 47 ms against 74 ms for the 16-CTA cluster.  At 256^2 with 5
// modes (64 CTAs of 4 rows) it measured 245 ms against 239 ms for the cluster: the row split gives both the same
// 128 warps, and the grid barriers cost more than the cluster's, so 256 keeps the cluster.
template <int L> struct EpieGridShape { static constexpr int R = 0; };
template <> struct EpieGridShape<256> { static constexpr int R = 4; };
template <> struct EpieGridShape<512> { static constexpr int R = 4; };

template <int L, int R>
static size_t epie_smem_r() {
  constexpr int XCH = FftShape<L>::XCH;
  constexpr int xs = R * XCH > L * (R + 1) ? R * XCH : L * (R + 1);
  return sizeof(float2) * (L + xs) + sizeof(float) * R * L + sizeof(float2) * R * L;
}
template <int L>
static size_t epie_smem(int) {
  return epie_smem_r<L, EpieShape<L>::R>();
}

// Whole-GPU variant set-up: C = L / R CTAs must be co-resident (cooperative launch); returns C, or 0 if not possible.
template <int L>
static int epie_grid_prepare_t() {
  constexpr int R = EpieGridShape<L>::R;
  if constexpr (R == 0) {
    return 0;
  } else {
    constexpr int T = FftShape<L>::T, C = L / R;
    auto kern = k_epie<L, R, true>;
    const size_t smem = epie_smem_r<L, R>();
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, R * T, smem) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    return (coop && per_sm * sms >= C) ? C : 0;
  }
}

template <int L>
static cudaError_t epie_prepare_t(int* C_out) {
  constexpr int R = EpieShape<L>::R, T = FftShape<L>::T;
  auto kern = k_epie<L, R, false>;
  const size_t smem = epie_smem<L>(0);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  // Largest cluster (<= 16, dividing the rows into whole passes, >= one warp per CTA) that can be resident.
  int best = 0;
  for (int C = 16; C >= 1; C /= 2) {
    if (L % C || (L / C) % R) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(R * T);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n >= 1) {
      best = C;
      break;
    }
    cudaGetLastError();
  }
  if (!best) return cudaErrorInvalidConfiguration;
  *C_out = best;
  return cudaSuccess;
}

int epie_grid_prepare(int N, bool any_size) {
  if (N == 512) return epie_grid_prepare_t<512>();
  if (N == 256 && any_size) return epie_grid_prepare_t<256>();
  return 0;
}

cudaError_t epie_prepare(int N, int* C_out) {
  switch (N) {
    case 32: return epie_prepare_t<32>(C_out);
    case 64: return epie_prepare_t<64>(C_out);
    case 128: return epie_prepare_t<128>(C_out);
    case 256: return epie_prepare_t<256>(C_out);
    case 512: return epie_prepare_t<512>(C_out);
    default: return cudaErrorInvalidValue;
  }
}

template <int L>
static cudaError_t epie_launch_t(const EpieArgs& g, cudaStream_t st) {
  if constexpr (EpieGridShape<L>::R > 0) {
    if (g.grid) {
      constexpr int R = EpieGridShape<L>::R, T = FftShape<L>::T;
      cudaError_t e = cudaMemsetAsync(g.gbar, 0, 2 * sizeof(unsigned), st);
      if (e != cudaSuccess) return e;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(g.C);
      cfg.blockDim = dim3(R * T);
      cfg.dynamicSmemBytes = epie_smem_r<L, R>();
      cfg.stream = st;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      return cudaLaunchKernelEx(&cfg, k_epie<L, R, true>, g);
    }
  }
  constexpr int R = EpieShape<L>::R, T = FftShape<L>::T;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(g.C);
  cfg.blockDim = dim3(R * T);
  cfg.dynamicSmemBytes = epie_smem<L>(0);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = g.C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_epie<L, R, false>, g);
}

cudaError_t epie_launch(const EpieArgs& g, cudaStream_t st) {
  switch (g.N) {
    case 32: return epie_launch_t<32>(g, st);
    case 64: return epie_launch_t<64>(g, st);
    case 128: return epie_launch_t<128>(g, st);
    case 256: return epie_launch_t<256>(g, st);
    case 512: return epie_launch_t<512>(g, st);
    default: return cudaErrorInvalidValue;
  }
}

__global__ void k_tile_max_all(const float* __restrict__ ocache, int X, int Y, float* __restrict__ TM, int TY) {
  const int tr = blockIdx.y, tc = blockIdx.x;
  float m = 0.f;
  for (int j = threadIdx.x; j < 256; j += blockDim.x) {
    const int xr = tr * 16 + j / 16, yc = tc * 16 + j % 16;
    if (xr < X && yc < Y) m = fmaxf(m, ocache[size_t(xr) * Y + yc]);
  }
  m = block_reduce_maxf(m);
  if (threadIdx.x == 0) TM[size_t(tr) * TY + tc] = m;
}

cudaError_t tile_max_all(const float* ocache, int X, int Y, float* TM, int TX, int TY, cudaStream_t st) {
  k_tile_max_all<<<dim3(TY, TX), 64, 0, st>>>(ocache, X, Y, TM, TY);
  return cudaGetLastError();
}

// ---- modal set-up (Probe::initProbeModes / orthogonalize, src/Probe.cpp:229-242,320-330) ---------------
__global__ void k_modes_from_base(float2* __restrict__ probe, float* __restrict__ pcache, int K, size_t NN,
                                  float factor) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < NN; i += size_t(gridDim.x) * blockDim.x) {
    const float2 b = probe[i];
    const float2 v = make_float2(b.x * factor, b.y * factor);
    const float m = sqrtf(v.x * v.x + v.y * v.y);
    for (int k = 1; k < K; ++k) {
      probe[size_t(k) * NN + i] = v;
      pcache[size_t(k) * NN + i] = m * m;
    }
  }
}

// out[0..1] += sum conj(a) * b, out[2] += sum |a|^2 (double accumulation)
__global__ void k_inner(const float2* __restrict__ a, const float2* __restrict__ b, size_t n, double* out) {
  double re = 0, im = 0, aa = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float2 x = a[i], y = b[i];
    re += double(x.x) * y.x + double(x.y) * y.y;
    im += double(x.x) * y.y - double(x.y) * y.x;
    aa += double(x.x) * x.x + double(x.y) * x.y;
  }
  re = block_reduce_sum(re);
  __syncthreads();
  im = block_reduce_sum(im);
  __syncthreads();
  aa = block_reduce_sum(aa);
  if (threadIdx.x == 0) {
    atomicAdd(&out[0], re);
    atomicAdd(&out[1], im);
    atomicAdd(&out[2], aa);
  }
}

// target -= f * u with f = conj(<u, v>) / <u, u> read from ip = {Re<u,v>, Im<u,v>, <u,u>} (h_projectUtoV:
// factor = innerProduct(v, u) / innerProduct(u, u), innerProduct(a, b) = sum conj(a) b).
__global__ void k_project_sub(float2* __restrict__ target, const float2* __restrict__ u, size_t n,
                              const double* __restrict__ ip) {
  const double fr = ip[0] / ip[2], fi = -ip[1] / ip[2];
  const float2 f = make_float2(float(fr), float(fi));
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    target[i] = csub(target[i], cmul(f, u[i]));
}

cudaError_t epie_init_modes(float2* probe, float* pcache, int K, int N, float2* copy, double* scratch3,
                            cudaStream_t st) {
  const size_t NN = size_t(N) * N;
  int grid = int((NN + 255) / 256);
  if (grid > 1184) grid = 1184;
  k_modes_from_base<<<grid, 256, 0, st>>>(probe, pcache, K, NN, 0.05f);
  cudaError_t e = cudaMemcpyAsync(copy, probe, sizeof(float2) * NN * K, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  for (int i = 1; i < K; ++i)
    for (int j = i - 1; j >= 0; --j) {
      e = cudaMemsetAsync(scratch3, 0, 3 * sizeof(double), st);
      if (e != cudaSuccess) return e;
      k_inner<<<grid, 256, 0, st>>>(probe + size_t(j) * NN, copy + size_t(i) * NN, NN, scratch3);
      k_project_sub<<<grid, 256, 0, st>>>(probe + size_t(i) * NN, probe + size_t(j) * NN, NN, scratch3);
    }
  return cudaGetLastError();
}

// Self-test of the bounded grid barrier (failure detection without a GPU fault): a cooperative launch of C CTAs
// passes `rounds` barriers expecting `expected` arrivals with at most `limit` polls each; a barrier whose count
// cannot be reached (expected > C) must time out, set *err and let every CTA return.
__global__ void k_selftest_grid_barrier(unsigned* bar, int* err, unsigned expected, unsigned limit, int rounds) {
  for (int r = 0; r < rounds; ++r)
    if (!grid_barrier(bar, err, expected, limit)) return;
}

cudaError_t selftest_grid_barrier(int ctas, unsigned expected, unsigned limit, int rounds, unsigned* bar, int* err,
                                  cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(64);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_selftest_grid_barrier, bar, err, expected, limit, rounds);
}

}  // namespace pty
