// Reference DM ("difference map" as ptychopy implements it, src/DM.cu:80-128 with the cuFFT callbacks of
// src/SampleKernels.cu:416-490) as three kernels per wave of patterns plus a finalize step:
//
//   rows   u = 2*P*O[x+ox][y+oy] - psi[x][y]  (load callback d_calculatePsi), FFT along y (one warp per row),
//          W1[x][ky] row-major                                                  reads psi once from HBM
//   cols   FFT along x of CB adjacent columns per CTA (fft_cols: coalesced row segments, no transpose),
//          D = Psi' - Psi/N^2 with Psi' = A*Psi/|Psi|/N^2 (store callback d_modulusConstraint), inverse FFT along x,
//          W2[x][ky] row-major                                                  reads A once
//   inv    inverse FFT along y gives psi_new = IFFT2(D) = psi + IFFT2(Psi') - 2*P*O (store callback
//          d_updateObject), writes psi, and accumulates the object / probe increments       writes psi once
//   finalize   O += dO, P += dP, sums of |O|^2 and |P|^2, the hysteresis-cached factors (src/DM.cu:54-73)
//
// psi_new is formed as IFFT2(Psi' - Psi/N^2): by linearity IFFT2(Psi/N^2) = u = 2*P*O - psi, so
// psi + IFFT2(Psi') - 2*P*O = IFFT2(Psi') - u.  This removes the second read of psi the callback form needs,
// leaving 20*N^2 bytes of algorithmic HBM traffic per pattern: psi read + write, A read.  Every global access is a
// coalesced row segment and every plane keeps its natural row-major layout.
//
// The kernels are persistent (grid = resident CTA slots) and stride over the wave's work items (NB per pattern).
//
// Object and probe updates use snapshot semantics: all increments of an iteration are computed from O and P
// as they were at its start and summed (the reference adds them with atomics while other callbacks still read
// O and P, which makes its result order-dependent).
#include <algorithm>
#include <cmath>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels.h"

namespace pty {

// CTAs per SM the DM kernels are compiled for (64 registers).  5 CTAs/SM (48 registers: no spills in the row and
// column kernels) measured slower, 3.30 vs 3.12 ms per 900-pattern iteration at 512^2.
template <int L> struct DMOcc {
  static constexpr int MIN_BLOCKS = 4;
  static constexpr int MIN_BLOCKS_INV = 4;
};

// Row and column work items use the same CTA size and item count per pattern for every supported L.
template <int L>
struct DMShape {
  static constexpr int THREADS = FftShape<L>::THREADS;
  static constexpr int NB = L / FftShape<L>::RC;
  static_assert(cols_threads<L>() == THREADS, "row and column items share the CTA size");
  static_assert(L / cols_per_block<L>() == NB, "row and column items share the item count");
  static constexpr size_t SMEM_ROWS = sizeof(float2) * (L + FftShape<L>::RC * FftShape<L>::XCH);
  static constexpr size_t SMEM_COLS = sizeof(float2) * (L + cols_xch_elems<L>());
  static constexpr size_t SMEM = SMEM_ROWS > SMEM_COLS ? SMEM_ROWS : SMEM_COLS;
};

// Rows x = sub*R .. sub*R + R-1 of pattern p (W slot `slot`).
template <int L>
__device__ __forceinline__ void dm_item_rows(const DMBuffers& b, int p, int slot, int sub, float2* s_x,
                                             const float2* s_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  const int x = sub * R + v;
  const int2 o = b.offs[p];
  const float2* prow = b.probe + size_t(x) * L;
  const float2* orow = b.obj + size_t(x + o.x) * b.Y + o.y;
  const float2* srow = b.psi + (size_t(p) * L + x) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = t + T * e;
    const float2 ph = cmul(prow[n], orow[n]);
    const float2 sv = ld_stream(srow + n);
    a[e] = make_float2(2.f * ph.x - sv.x, 2.f * ph.y - sv.y);
  }
  fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
  float2* wrow = b.W1 + (size_t(slot) * L + x) * L;
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    wrow[t + T * e] = a[out_slot<L>(e)];
  });
}

// Columns sub*CB .. sub*CB + CB-1 of pattern p: forward FFT along x, modulus, inverse FFT along x.
template <int L>
__device__ __forceinline__ void dm_item_cols(const DMBuffers& b, int p, int slot, int slot2, int sub, float2* s_x,
                                             const float2* s_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, CB = cols_per_block<L>();
  int s, c;
  cols_thread<L>(threadIdx.x, s, c);
  const int col = sub * CB + c;
  const float2* w1 = b.W1 + size_t(slot) * L * L + col;
  const float* A = b.amp + size_t(p) * L * L + col;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = w1[size_t(s + T * e) * L];
  fft_cols<L, false>(a, s, c, s_x, s_tw);
  constexpr float nrm = 1.0f / float(L * L);
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const float Av = ld_stream(A + size_t(s + T * e) * L);
    const float2 ps = a[out_slot<L>(e)];
    const float2 rep = modulus_replace(ps, Av * nrm);
    a[out_slot<L>(e)] = make_float2(rep.x - ps.x * nrm, rep.y - ps.y * nrm);
  });
  to_input_order<L>(a);
  fft_cols<L, true>(a, s, c, s_x, s_tw);
  float2* w2 = b.W2 + size_t(slot2) * L * L + col;
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    w2[size_t(s + T * e) * L] = a[out_slot<L>(e)];
  });
}

// Rows of pattern p: inverse FFT along y -> psi_new, psi write, object / probe increments.
template <int L, bool PC, bool UP>
__device__ __forceinline__ void dm_item_inv(const DMBuffers& b, int p, int slot, int sub, float2* s_x,
                                            const float2* s_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  const int x = sub * R + v;
  const float2* row = b.W2 + (size_t(slot) * L + x) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
  fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
  const int2 o = b.offs[p];
  const float2* prow = b.probe + size_t(x) * L;
  const float2* orow = b.obj + size_t(x + o.x) * b.Y + o.y;
  float2* dorow = b.dO + size_t(x + o.x) * b.Y + o.y;
  float2* psrow = b.psi + (size_t(p) * L + x) * L;
  float2* dprow = b.dP + size_t(x) * L;
  // probe (and object) values in batches of DB elements, loaded before the batch's stores and atomics: a load placed
  // after a store it might alias waits for it, which would leave one L2 round trip per element
  constexpr int DB = UP ? 2 : 4;
  static_assert(E % DB == 0, "epilogue batches");
  static_for<0, E / DB>([&](auto bc) {
    constexpr int e0 = decltype(bc)::value * DB;
    float2 pv[DB];
    [[maybe_unused]] float2 ov[DB];
    static_for<0, DB>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      pv[j] = prow[t + T * (e0 + j)];
      if constexpr (UP) ov[j] = orow[t + T * (e0 + j)];
    });
    static_for<0, DB>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      const int n = t + T * (e0 + j);
      const float2 pn = a[out_slot<L>(e0 + j)];
      st_stream(psrow + n, pn);
      // the increments are accumulated unscaled: finalize multiplies the sums by f1 (object) and f0 (probe), which
      // as positive factors commute with the phase clamp
      float2 inc = cconjmul(pv[j], pn);
      if constexpr (PC) inc = constrain_phase(inc);
      atomicAdd(dorow + n, inc);
      if constexpr (UP) atomicAdd(dprow + n, cconjmul(ov[j], pn));
    });
  });
}

template <int L>
__global__ void __launch_bounds__(DMShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS)
    k_dm_rows(const DMBuffers b, const DMWave w) {
  constexpr int NB = DMShape<L>::NB;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  load_twiddles<L>(smem, b.tw);
  __syncthreads();
  for (int item = blockIdx.x; item < NB * w.count; item += gridDim.x)
    dm_item_rows<L>(b, w.slot_pat[item / NB], item / NB, item % NB, smem + L, smem);
}

template <int L>
__global__ void __launch_bounds__(DMShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS)
    k_dm_cols(const DMBuffers b, const DMWave w) {
  constexpr int NB = DMShape<L>::NB;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  load_twiddles<L>(smem, b.tw);  // visible after fft_cols' first barrier
  for (int item = blockIdx.x; item < NB * w.count; item += gridDim.x)
    dm_item_cols<L>(b, w.slot_pat[item / NB], item / NB, item / NB, item % NB, smem + L, smem);
}

template <int L, bool PC, bool UP>
__global__ void __launch_bounds__(DMShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS_INV)
    k_dm_inv(const DMBuffers b, const DMWave w) {
  constexpr int NB = DMShape<L>::NB;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  load_twiddles<L>(smem, b.tw);
  __syncthreads();
  for (int item = blockIdx.x; item < NB * w.count; item += gridDim.x)
    dm_item_inv<L, PC, UP>(b, w.slot_pat[item / NB], item / NB, item % NB, smem + L, smem);
}

// O += dO, P += dP (mode 0), reset the accumulators, and sum |O|^2 and |P|^2 over all stacked probe modes.
__global__ void k_dm_finalize(float2* __restrict__ obj, float2* __restrict__ dO, size_t nobj,
                              float2* __restrict__ probe, float2* __restrict__ dP, size_t nprobe0, size_t nprobe,
                              int updateProbe, double* __restrict__ sums, const double* __restrict__ fac) {
  double so = 0, sp = 0;
  const float f0 = float(fac[0]), f1 = float(fac[1]);
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nobj; i += stride) {
    float2 v = obj[i], d = dO[i];
    v = cadd(v, cscale(d, f1));
    obj[i] = v;
    dO[i] = make_float2(0.f, 0.f);
    float m = sqrtf(v.x * v.x + v.y * v.y);
    so += double(m * m);
  }
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nprobe; i += stride) {
    float2 v = probe[i];
    if (updateProbe && i < nprobe0) {
      v = cadd(v, cscale(dP[i], f0));
      probe[i] = v;
      dP[i] = make_float2(0.f, 0.f);
    }
    float m = sqrtf(v.x * v.x + v.y * v.y);
    sp += double(m * m);
  }
  so = block_reduce_sum(so);
  __syncthreads();
  sp = block_reduce_sum(sp);
  if (threadIdx.x == 0) {
    atomicAdd(&sums[0], so);
    atomicAdd(&sums[1], sp);
  }
}

// checkCache (src/DM.cu:54-73): factor j moves to its new value only if it changed by more than EPS = 1e-3.
__global__ void k_dm_factors(double* __restrict__ sums, double* __restrict__ fac) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double objMax = sums[0], probeMax = sums[1];
    const double passed[2] = {1.0 / objMax, 1.0 / probeMax};
    for (int j = 0; j < 2; ++j)
      if (fabs(fac[j] - passed[j]) > 1e-3) fac[j] = passed[j];
    fac[2] = objMax;
    fac[3] = probeMax;
    sums[0] = 0;
    sums[1] = 0;
  }
}

template <int L>
static int dm_slots_rows();
template <int L>
static int dm_slots_cols();
template <int L>
static int dm_slots_inv();

template <int L>
static cudaError_t dm_prepare_t() {
  const int sm = int(DMShape<L>::SMEM);
  const void* fns[6] = {(const void*)k_dm_rows<L>, (const void*)k_dm_cols<L>, (const void*)k_dm_inv<L, false, false>,
                        (const void*)k_dm_inv<L, false, true>, (const void*)k_dm_inv<L, true, false>,
                        (const void*)k_dm_inv<L, true, true>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
  }
  // the resident-slot counts, queried here, outside any stream capture
  dm_slots_rows<L>();
  dm_slots_cols<L>();
  dm_slots_inv<L>();
  return cudaGetLastError();
}

cudaError_t dm_prepare(int N) {
  switch (N) {
    case 32: return dm_prepare_t<32>();
    case 64: return dm_prepare_t<64>();
    case 128: return dm_prepare_t<128>();
    case 256: return dm_prepare_t<256>();
    case 512: {
      const cudaError_t e = dm_prepare_t<512>();
      return e != cudaSuccess ? e : dm_cols_tc_prepare();
    }
    default: return cudaErrorInvalidValue;
  }
}

// Resident CTA slots of a DM kernel (once per kernel and size; first asked by dm_prepare, outside stream capture).
template <typename K>
static int resident_slots(K kern, int threads, size_t smem) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess) cudaGetLastError();
  return sms * (per > 0 ? per : 1);
}
template <int L>
static int dm_slots_rows() {
  static const int s = resident_slots(k_dm_rows<L>, DMShape<L>::THREADS, DMShape<L>::SMEM);
  return s;
}
template <int L>
static int dm_slots_cols() {
  static const int s = resident_slots(k_dm_cols<L>, DMShape<L>::THREADS, DMShape<L>::SMEM);
  return s;
}
template <int L>
static int dm_slots_inv() {
  static const int s = resident_slots(k_dm_inv<L, true, true>, DMShape<L>::THREADS, DMShape<L>::SMEM);
  return s;
}

template <int L>
static cudaError_t dm_wave_t(const DMBuffers& b, const DMWave& w, bool pc, bool up, cudaStream_t st,
                             int64_t* launches) {
  constexpr int NT = DMShape<L>::THREADS, NB = DMShape<L>::NB;
  constexpr size_t SM = DMShape<L>::SMEM;
  const int items = NB * w.count;
  const int grid = std::min(dm_slots_inv<L>(), items);
  k_dm_rows<L><<<std::min(dm_slots_rows<L>(), items), NT, SM, st>>>(b, w);
  if constexpr (L == 512) {
    if (b.tc) {
      const cudaError_t e = dm_cols_tc(b, w, st);
      if (e != cudaSuccess) return e;
    } else {
      k_dm_cols<L><<<std::min(dm_slots_cols<L>(), items), NT, SM, st>>>(b, w);
    }
  } else {
    k_dm_cols<L><<<std::min(dm_slots_cols<L>(), items), NT, SM, st>>>(b, w);
  }
  if (pc && up)
    k_dm_inv<L, true, true><<<grid, NT, SM, st>>>(b, w);
  else if (pc)
    k_dm_inv<L, true, false><<<grid, NT, SM, st>>>(b, w);
  else if (up)
    k_dm_inv<L, false, true><<<grid, NT, SM, st>>>(b, w);
  else
    k_dm_inv<L, false, false><<<grid, NT, SM, st>>>(b, w);
  if (launches) *launches += 3;
  return cudaGetLastError();
}

template <int L>
static int dm_wave_size_t(int P) {
  const size_t bytes_per_pattern = 2 * sizeof(float2) * size_t(L) * L;
  const int maxwave = int(std::max<size_t>(1, (size_t(1) << 29) / bytes_per_pattern));
  int nw = (P + maxwave - 1) / maxwave;
  const int by_items = int(size_t(P) * DMShape<L>::NB / (2 * size_t(dm_slots_inv<L>())));
  nw = std::max(nw, std::min(8, by_items));
  nw = std::max(1, std::min(nw, P));
  return (P + nw - 1) / nw;
}

// Patterns per wave: balanced waves, at least eight where each still holds two persistent grids' worth of items, and
// W1 + W2 of the two lanes of waves in flight within 1 GiB.  The kernels are bound by their on-chip work (shared
// memory, L1, issue), not by the W1 / W2 traffic: with one lane, waves small enough for W1 + W2 to stay in L2 lost
// more to the per-wave tails of three dependent launches than they saved (25 / 50 / 75 / 225 patterns: 3.55 / 3.35 /
// 3.25 / 3.11 ms per 900 x 512^2 iteration); with two lanes each wave's kernels fill the other's tails.
int dm_wave_size(int N, int P) {
  switch (N) {
    case 32: return dm_wave_size_t<32>(P);
    case 64: return dm_wave_size_t<64>(P);
    case 128: return dm_wave_size_t<128>(P);
    case 256: return dm_wave_size_t<256>(P);
    case 512: return dm_wave_size_t<512>(P);
    default: return std::max(1, P);
  }
}

cudaError_t dm_wave(const DMBuffers& b, const DMWave& w, bool pc, bool up, cudaStream_t st, int64_t* launches) {
  switch (b.N) {
    case 32: return dm_wave_t<32>(b, w, pc, up, st, launches);
    case 64: return dm_wave_t<64>(b, w, pc, up, st, launches);
    case 128: return dm_wave_t<128>(b, w, pc, up, st, launches);
    case 256: return dm_wave_t<256>(b, w, pc, up, st, launches);
    case 512: return dm_wave_t<512>(b, w, pc, up, st, launches);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t dm_finalize(const DMBuffers& b, bool up, cudaStream_t st, int64_t* launches) {
  const size_t nobj = size_t(b.X) * b.Y, np0 = size_t(b.N) * b.N, np = np0 * b.K;
  int grid = int((nobj + 255) / 256);
  if (grid > 1184) grid = 1184;
  k_dm_finalize<<<grid, 256, 0, st>>>(b.obj, b.dO, nobj, b.probe, b.dP, np0, np, up ? 1 : 0, b.sums, b.fac);
  k_dm_factors<<<1, 32, 0, st>>>(b.sums, b.fac);
  if (launches) *launches += 2;
  return cudaGetLastError();
}

// psi_p[x][y] = P[x][y] * O[x + ox_p][y + oy_p] for every pattern: the exit waves of the current object and probe
// (mode 0), the usual start of the difference map for a given object.
__global__ void k_dm_psi_from_object(const DMBuffers b, int P) {
  const size_t NN = size_t(b.N) * b.N, n = size_t(P) * NN;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int p = int(q / NN), k = int(q % NN), x = k / b.N, y = k % b.N;
    const int2 o = b.offs[p];
    b.psi[q] = cmul(b.probe[k], b.obj[size_t(x + o.x) * b.Y + o.y + y]);
  }
}

cudaError_t dm_psi_from_object(const DMBuffers& b, int P, cudaStream_t st) {
  const size_t n = size_t(P) * b.N * b.N;
  const int grid = int(std::min<size_t>((n + 255) / 256, 148 * 16));
  k_dm_psi_from_object<<<grid, 256, 0, st>>>(b, P);
  return cudaGetLastError();
}

}  // namespace pty
