// Reference DM ("difference map" as ptychopy implements it, src/DM.cu:80-128 with the cuFFT callbacks of
// src/SampleKernels.cu:416-490) as a three-kernel pipeline per wave of patterns plus a finalize step:
//
//   fwd_rows   u = 2*P*O[x+ox][y+oy] - psi[x][y]  (load callback d_calculatePsi), FFT along y,
//              stored transposed into W1[ky][x]                                   reads psi once from HBM
//   cols       FFT along x (now contiguous), D = Psi' - Psi/N^2 with Psi' = A*Psi/|Psi|/N^2 (store callback
//              d_modulusConstraint), inverse FFT along x, stored transposed into W2[x][ky]  reads A once
//   inv_rows   inverse FFT along y gives psi_new = IFFT2(D) = psi + IFFT2(Psi') - 2*P*O (store callback
//              d_updateObject), writes psi, and accumulates the object / probe increments   writes psi once
//   finalize   O += dO, P += dP, sums of |O|^2 and |P|^2, the hysteresis-cached factors (src/DM.cu:54-73)
//
// psi_new is formed as IFFT2(Psi' - Psi/N^2): by linearity IFFT2(Psi/N^2) = u = 2*P*O - psi, so
// psi + IFFT2(Psi') - 2*P*O = IFFT2(Psi') - u.  This removes the second read of psi the callback form needs,
// leaving the algorithmic minimum of HBM traffic, 20*N^2 bytes per pattern: psi read + write, A read.
// W1/W2 hold one wave (a few tens of MB) and stay in L2 between the kernels.
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

// CTAs per SM the DM kernels are compiled for (caps registers so that many fit next to their shared memory).
template <int L> struct DMOcc { static constexpr int MIN_BLOCKS = 4; };

// Work items of a wave: (row block, slot) pairs; CTAs are persistent and stride over them (grid <= resident
// slots), so a launch has no partially filled last round and CTAs drift out of lock-step (load / FFT overlap).
template <int L>
__global__ void __launch_bounds__(FftShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS)
    k_dm_fwd_rows(const float2* __restrict__ psi, const float2* __restrict__ obj, int objY,
                  const float2* __restrict__ probe, const int2* __restrict__ offs, const int* __restrict__ slot_pat,
                  int count, float2* __restrict__ W1, const float2* __restrict__ g_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC, NB = L / S::RC;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  float2* s_tw = smem;
  float2* s_x = smem + L;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  load_twiddles<L>(s_tw, g_tw);
  for (int item = blockIdx.x; item < NB * count; item += gridDim.x) {
  const int slot = item / NB;
  const int p = slot_pat[slot];
  const int x0 = (item % NB) * R, x = x0 + v;
  const int2 o = offs[p];
  const float2* prow = probe + size_t(x) * L;
  const float2* orow = obj + size_t(x + o.x) * objY + o.y;
  const float2* srow = psi + (size_t(p) * L + x) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = t + T * e;
    const float2 ph = cmul(prow[n], orow[n]);
    const float2 sv = ld_stream(srow + n);
    a[e] = make_float2(2.f * ph.x - sv.x, 2.f * ph.y - sv.y);
  }
  __syncthreads();  // twiddles loaded; previous item's staging reads done
  fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
  store_rows_transposed<L, R>(a, W1 + size_t(slot) * L * L, x0, v, t, s_x);
  }
}

template <int L>
__global__ void __launch_bounds__(FftShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS)
    k_dm_cols(const float2* __restrict__ W1, const float* __restrict__ ampT, const int* __restrict__ slot_pat,
              int count, float2* __restrict__ W2, const float2* __restrict__ g_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC, NB = L / S::RC;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  float2* s_tw = smem;
  float2* s_x = smem + L;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  load_twiddles<L>(s_tw, g_tw);
  for (int item = blockIdx.x; item < NB * count; item += gridDim.x) {
  const int slot = item / NB;
  const int p = slot_pat[slot];
  const int k0 = (item % NB) * R, ky = k0 + v;
  const float2* row = W1 + (size_t(slot) * L + ky) * L;
  const float* arow = ampT + (size_t(p) * L + ky) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
  __syncthreads();
  fft_vec<L, false>(a, t, s_x + v * S::XCH, s_tw);
  constexpr float nrm = 1.0f / float(L * L);
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const float A = ld_stream(arow + t + T * e);
    const float2 psi = a[out_slot<L>(e)];
    const float2 rep = modulus_replace(psi, A * nrm);
    a[out_slot<L>(e)] = make_float2(rep.x - psi.x * nrm, rep.y - psi.y * nrm);
  });
  to_input_order<L>(a);
  fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
  store_rows_transposed<L, R>(a, W2 + size_t(slot) * L * L, k0, v, t, s_x);
  }
}

template <int L>
__global__ void __launch_bounds__(FftShape<L>::THREADS, DMOcc<L>::MIN_BLOCKS)
    k_dm_inv_rows(const float2* __restrict__ W2, float2* __restrict__ psi, const float2* __restrict__ obj, int objY,
                  const float2* __restrict__ probe, const int2* __restrict__ offs, const int* __restrict__ slot_pat,
                  int count, float2* __restrict__ dO, float2* __restrict__ dP, const double* __restrict__ fac,
                  int phaseConstraint, int updateProbe, const float2* __restrict__ g_tw) {
  using S = FftShape<L>;
  constexpr int T = S::T, E = S::E, R = S::RC, NB = L / S::RC;
  extern __shared__ float4 smem4[];
  float2* smem = reinterpret_cast<float2*>(smem4);
  float2* s_tw = smem;
  float2* s_x = smem + L;
  const int v = threadIdx.x / T, t = threadIdx.x % T;
  load_twiddles<L>(s_tw, g_tw);
  for (int item = blockIdx.x; item < NB * count; item += gridDim.x) {
  const int slot = item / NB;
  const int p = slot_pat[slot];
  const int x = (item % NB) * R + v;
  const float2* row = W2 + (size_t(slot) * L + x) * L;
  float2 a[E];
#pragma unroll
  for (int e = 0; e < E; ++e) a[e] = row[t + T * e];
  __syncthreads();
  fft_vec<L, true>(a, t, s_x + v * S::XCH, s_tw);
  const float f0 = float(fac[0]), f1 = float(fac[1]);
  const int2 o = offs[p];
  const float2* prow = probe + size_t(x) * L;
  const float2* orow = obj + size_t(x + o.x) * objY + o.y;
  float2* dorow = dO + size_t(x + o.x) * objY + o.y;
  float2* psrow = psi + (size_t(p) * L + x) * L;
  float2* dprow = dP + size_t(x) * L;
  static_for<0, E>([&](auto ec) {
    constexpr int e = decltype(ec)::value;
    const int n = t + T * e;
    const float2 pn = a[out_slot<L>(e)];
    st_stream(psrow + n, pn);
    const float2 pv = prow[n];
    float2 inc = cconjmul(pv, pn);
    inc = make_float2(inc.x * f1, inc.y * f1);
    if (phaseConstraint) inc = constrain_phase(inc);
    atomicAdd(dorow + n, inc);
    if (updateProbe) {
      const float2 ov = orow[n];
      float2 pi = cconjmul(ov, pn);
      atomicAdd(dprow + n, make_float2(pi.x * f0, pi.y * f0));
    }
  });
  }
}

// O += dO, P += dP (mode 0), reset the accumulators, and sum |O|^2 and |P|^2 over all stacked probe modes.
__global__ void k_dm_finalize(float2* __restrict__ obj, float2* __restrict__ dO, size_t nobj,
                              float2* __restrict__ probe, float2* __restrict__ dP, size_t nprobe0, size_t nprobe,
                              int updateProbe, double* __restrict__ sums) {
  double so = 0, sp = 0;
  const size_t stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nobj; i += stride) {
    float2 v = obj[i], d = dO[i];
    v = cadd(v, d);
    obj[i] = v;
    dO[i] = make_float2(0.f, 0.f);
    float m = sqrtf(v.x * v.x + v.y * v.y);
    so += double(m * m);
  }
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < nprobe; i += stride) {
    float2 v = probe[i];
    if (updateProbe && i < nprobe0) {
      v = cadd(v, dP[i]);
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
static cudaError_t dm_prepare_t() {
  const int smem = int(rows_smem_bytes<L>());
  cudaError_t e = cudaFuncSetAttribute(k_dm_fwd_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_dm_cols<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_dm_inv_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return e;
}

cudaError_t dm_prepare(int N) {
  switch (N) {
    case 32: return dm_prepare_t<32>();
    case 64: return dm_prepare_t<64>();
    case 128: return dm_prepare_t<128>();
    case 256: return dm_prepare_t<256>();
    case 512: return dm_prepare_t<512>();
    default: return cudaErrorInvalidValue;
  }
}

template <int L>
static int dm_grid(int items) {
  static int slots = 0;
  if (!slots) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dm_fwd_rows<L>, FftShape<L>::THREADS, rows_smem_bytes<L>());
    slots = sms * (per > 0 ? per : 1);
  }
  return items < slots ? items : slots;
}

template <int L>
static cudaError_t dm_wave_t(const DMBuffers& b, const DMWave& w, bool pc, bool up, cudaStream_t st,
                             int64_t* launches) {
  constexpr int NT = FftShape<L>::THREADS, NB = L / FftShape<L>::RC;
  const size_t smem = rows_smem_bytes<L>();
  const int grid = dm_grid<L>(NB * w.count);
  k_dm_fwd_rows<L><<<grid, NT, smem, st>>>(b.psi, b.obj, b.Y, b.probe, b.offs, w.slot_pat, w.count, b.W1, b.tw);
  k_dm_cols<L><<<grid, NT, smem, st>>>(b.W1, b.ampT, w.slot_pat, w.count, b.W2, b.tw);
  k_dm_inv_rows<L><<<grid, NT, smem, st>>>(b.W2, b.psi, b.obj, b.Y, b.probe, b.offs, w.slot_pat, w.count, b.dO, b.dP,
                                           b.fac, pc ? 1 : 0, up ? 1 : 0, b.tw);
  if (launches) *launches += 3;
  return cudaGetLastError();
}

// Patterns per wave: the largest balanced wave with W1 + W2 within 1 GiB.  The three kernels are bound by their
// on-chip (L1/shared) traffic, so fewer, larger waves (less launch and tail overhead) beat L2-resident small ones.
template <int L>
static int dm_wave_size_t(int P) {
  const size_t bytes_per_pattern = 2 * sizeof(float2) * size_t(L) * L;
  const int maxwave = int(std::max<size_t>(1, (size_t(1) << 30) / bytes_per_pattern));
  const int nwaves = (P + maxwave - 1) / maxwave;
  return (P + nwaves - 1) / nwaves;
}

int dm_wave_size(int N, int P) {
  switch (N) {
    case 32: return dm_wave_size_t<32>(P);
    case 64: return dm_wave_size_t<64>(P);
    case 128: return dm_wave_size_t<128>(P);
    case 256: return dm_wave_size_t<256>(P);
    case 512: return dm_wave_size_t<512>(P);
    default: return 1;
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
  k_dm_finalize<<<grid, 256, 0, st>>>(b.obj, b.dO, nobj, b.probe, b.dP, np0, np, up ? 1 : 0, b.sums);
  k_dm_factors<<<1, 32, 0, st>>>(b.sums, b.fac);
  if (launches) *launches += 2;
  return cudaGetLastError();
}

}  // namespace pty
