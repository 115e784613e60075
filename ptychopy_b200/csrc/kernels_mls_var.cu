// MLs with the reference's defaults (src/Parameters.h:162-163: variable_probe, variable_intensity,
// apply_subpix_shift on, probe_pos_search = PPS): one probe mode, one object, one extra (variable) probe mode.
//
// Per iteration (MLS::iteration, src/MLS.cpp:74-116):
//   windows   from iteration 1 and PPS on: window starts and sub-pixel remainders from the current positions
//             (find_reconstruction_ROI, src/IPtychoScanMesh.cpp:122-171); group boxes from the windows
//   norm      calc_object_norm scales P, the extra mode E and O (src/Probe.cpp:671-699)
//   recentre  positions lose their mean drift from the originals (updateScanPositionsDiff,
//             src/IPtychoScanMesh.cpp:340-368)
//   remove    from iteration 2: E to unit RMS, its weights carry the norm; the intensity weights' regularisation
//             (remove_extra_degree, src/Probe.cpp:615-669)
//   illum     p_object running average (updated_cached_illumination), and its maximum
// Per group of G positions:
//   probes    vp_j = P evo0_j + E evo1_j, shifted by the sub-pixel remainder: IFFT2(FFT2(vp) e^{-2 pi i s.f})/N^2
//             (get_illumination_probe, shift_probe, src/Probe.cpp:887-954,1261-1337)
//   exit      psi = O[window] vp_j; FFT2, modulus with error, IFFT2 -> chi   (kernels_mls.cu)
//   dirs      pu_j = chi conj(O[window]) shifted back; pum = sum_j W pu_j; S += chi conj(vp_j) at the window
//             (src/MLS.cpp:232-347)
//   lsq/solve/update  as the core, with the position's own probe vp_j in dOP
//   search    from PPS: Fourier gradients of the window, least-squares shift per position clamped to 0.2 px
//             (gradient_position_solver, src/Probe.cpp:956-1118)
//   variable  from iteration 3: extra-mode step on the weighted residual of the probe directions, then the
//             extra-mode and intensity weights of the group's positions (update_variable_probe, src/Probe.cpp:1366-1516)
// Scalar bookkeeping (2x2 solves, position and weight updates) runs in one thread on the device, so the iteration
// is one CUDA graph with no host round trip.
#include <algorithm>
#include <cmath>

#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels_mls.h"
#include "pdl.cuh"
#include "fftx.cuh"

namespace pty {

namespace {

constexpr float kTwoPi = 6.283185307179586f;

// Offsets into MlsBuffers::vs (doubles).
struct VsLayout {
  int G;
  __host__ __device__ size_t pos() const { return 0; }             // 4 G: position-search sums
  __host__ __device__ size_t proj() const { return 4 * size_t(G); }  // G: residual projections
  __host__ __device__ size_t evs() const { return 5 * size_t(G); }   // 4 G: weight-update sums
  __host__ __device__ size_t sc() const { return 9 * size_t(G); }    // 8 scalars
};
enum { SC_ESUM = 0, SC_USUM = 1, SC_ENEW = 2, SC_EFAC = 3, SC_PFAC = 4 };

__device__ __forceinline__ float fft_freq(int k, int N) {
  return k < N / 2 ? float(k) / float(N) : float(k) / float(N) - 1.f;
}

__global__ void k_var_windows(const float* __restrict__ pos, int P, int N, int X, int Y, float cvx, float cvy,
                              int2* __restrict__ win, float2* __restrict__ sub) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float p1 = pos[2 * i] + cvx, p2 = pos[2 * i + 1] + cvy;
  const float t1 = roundf(p1), t2 = roundf(p2);
  sub[i] = make_float2(p2 - t2, p1 - t1);
  win[i] = make_int2(min(max(int(t1) - 1, 0), X - N), min(max(int(t2) - 1, 0), Y - N));
}

// Positions minus their mean drift from the originals (one block).
__global__ void k_var_recentre(float* __restrict__ pos, const float* __restrict__ pos_o, int P) {
  pdl_enter();
  double s[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    s[0] += pos[2 * i];
    s[1] += pos[2 * i + 1];
    s[2] += pos_o[2 * i];
    s[3] += pos_o[2 * i + 1];
  }
  __shared__ float d[2];
  block_reduce_sum_n(s);
  if (threadIdx.x == 0) {
    d[0] = float(s[0] / P) - float(s[2] / P);
    d[1] = float(s[1] / P) - float(s[3] / P);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    pos[2 * i] -= d[0];
    pos[2 * i + 1] -= d[1];
  }
}

// out += sum |a|^2 (FP64)
__global__ void k_var_sumsq(const float2* __restrict__ a, size_t n, double* __restrict__ out) {
  pdl_enter();
  double s = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    s += double(a[i].x) * a[i].x + double(a[i].y) * a[i].y;
  s = block_reduce_sum(s);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

// remove_extra_degree's scalars (one thread).  Its mean and norm loops run over m_probe_evolution.size() = 2 entries,
// so only positions 0 and 1 are re-centred; kept as written.
__global__ void k_var_remove(double* __restrict__ sc, double* __restrict__ evo, int P, int NN) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  double* e0 = evo;
  double* e1 = evo + P;
  const double vn = sqrt(sc[SC_ESUM] / NN);
  for (int i = 0; i < P; ++i) e1[i] *= vn;
  const int len = P < 2 ? P : 2;
  double a0 = 0, a1 = 0;
  for (int i = 0; i < len; ++i) {
    a0 += e0[i];
    a1 += e1[i];
  }
  const float m0 = float(a0 / len), m1 = float(a1 / len);
  double sq = 0;
  for (int i = 0; i < len; ++i) {
    e0[i] = (e0[i] - m0) * 0.99 + 1;
    e1[i] = e1[i] - m1;
    sq += e0[i] * e0[i];
  }
  const double cn = sqrt(sq / len);
  for (int i = 0; i < len; ++i) e0[i] /= cn;
  sc[SC_EFAC] = 1.0 / vn;
  sc[SC_PFAC] = cn;
  sc[SC_ESUM] = 0.0;
}

__global__ void k_var_scale(float2* __restrict__ a, size_t n, const double* __restrict__ f) {
  pdl_enter();
  const float s = float(*f);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = cscale(a[i], s);
}

// objp = O[window], vp = P evo0 + E evo1 (zeros past the group's size)
__global__ void k_var_exit(const float2* __restrict__ obj, const float2* __restrict__ probe,
                           const float2* __restrict__ E, const double* __restrict__ evo, int P,
                           const int2* __restrict__ win, const int* __restrict__ members,
                           const int* __restrict__ gsize, int N, int Y, float2* __restrict__ objp,
                           float2* __restrict__ vp) {
  pdl_enter();
  const int k = blockIdx.y;
  const size_t NN = size_t(N) * N;
  const bool live = k < *gsize;
  const int j = live ? members[k] : 0;
  const int2 s = live ? win[j] : make_int2(0, 0);
  const float f0 = live ? float(evo[j]) : 0.f, f1 = live ? float(evo[P + j]) : 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    float2 o = make_float2(0.f, 0.f), v = make_float2(0.f, 0.f);
    if (live) {
      o = obj[size_t(s.x + i / N) * Y + (s.y + i % N)];
      v = cadd(cscale(probe[i], f0), cscale(E[i], f1));
    }
    objp[k * NN + i] = o;
    vp[k * NN + i] = v;
  }
}

// a_k *= e^{-2 pi i sign (s.x f[c] + s.y f[r])} / N^2 on the spectra of the group's windows (shift_probe)
__global__ void k_var_phase(float2* __restrict__ a, const float2* __restrict__ sub, const int* __restrict__ members,
                            const int* __restrict__ gsize, int N, float sign) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N;
  const float2 s = sub[members[k]];
  const float sx = sign * s.x, sy = sign * s.y, nrm = 1.f / float(NN);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float t = sx * fft_freq(i % N, N) + sy * fft_freq(i / N, N);
    float sn, cs;
    sincosf(-kTwoPi * t, &sn, &cs);
    a[k * NN + i] = cmul(a[k * NN + i], make_float2(cs * nrm, sn * nrm));
  }
}

__global__ void k_var_psi(const float2* __restrict__ objp, const float2* __restrict__ vp, float2* __restrict__ psi,
                          size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    psi[i] = cmul(objp[i], vp[i]);
}

// pu = chi conj(objp); S += chi conj(vp) at the window
__global__ void k_var_dirs(const float2* __restrict__ chi, const float2* __restrict__ objp,
                           const float2* __restrict__ vp, const int2* __restrict__ win,
                           const int* __restrict__ members, const int* __restrict__ gsize, int N, int Y,
                           float2* __restrict__ pu, float2* __restrict__ S) {
  pdl_enter();
  const int k = blockIdx.y;
  const size_t NN = size_t(N) * N;
  if (k >= *gsize) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x)
      pu[k * NN + i] = make_float2(0.f, 0.f);
    return;
  }
  const int2 s = win[members[k]];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 c = chi[k * NN + i];
    pu[k * NN + i] = cmulc(c, objp[k * NN + i]);
    atomicAdd(&S[size_t(s.x + i / N) * Y + (s.y + i % N)], cmulc(c, vp[k * NN + i]));
  }
}

// pum = sum_j W_j pu_j, W = p/(p + 0.01 MAX_ILLUM) at the window (a sum over the group per pixel: no atomics)
__global__ void k_var_pum(const float2* __restrict__ pu, const float* __restrict__ pobj,
                          const float* __restrict__ maxIllum, const int2* __restrict__ win,
                          const int* __restrict__ members, const int* __restrict__ gsize, int N, int Y,
                          float2* __restrict__ pum) {
  pdl_enter();
  const int G = *gsize;
  const size_t NN = size_t(N) * N;
  const float damp = 0.01f * *maxIllum;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int k = 0; k < G; ++k) {
      const int2 s = win[members[k]];
      const float w = pobj[size_t(s.x + i / N) * Y + (s.y + i % N)];
      acc = cadd(acc, cscale(pu[k * NN + i], w / (w + damp)));
    }
    pum[i] = acc;
  }
}

// Gradient spectra of the windows: from FFT2(objp) in aux[k], dX -> aux[k] (column frequencies), dY -> aux[Gmax + k]
__global__ void k_var_grad(float2* __restrict__ aux, int Gmax, int N) {
  pdl_enter();
  const int k = blockIdx.y;
  const size_t NN = size_t(N) * N;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 v = aux[k * NN + i];
    const float2 d = cmul(v, make_float2(0.f, kTwoPi));
    aux[(Gmax + k) * NN + i] = cscale(d, fft_freq(i / N, N));
    aux[k * NN + i] = cscale(d, fft_freq(i % N, N));
  }
}

// Per window: sum |dX vp|^2, Re(chi conj(dX vp)), the same for dY (gradient images still unnormalised by N^2)
__global__ void k_var_possums(const float2* __restrict__ aux, const float2* __restrict__ vp,
                              const float2* __restrict__ chi, const int* __restrict__ gsize, int Gmax, int N,
                              double* __restrict__ out) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N;
  const float nrm = 1.f / float(NN);
  double v[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 p = vp[k * NN + i], c = chi[k * NN + i];
    const float2 gx = cmul(cscale(aux[k * NN + i], nrm), p);
    const float2 gy = cmul(cscale(aux[(Gmax + k) * NN + i], nrm), p);
    v[0] += double(gx.x) * gx.x + double(gx.y) * gx.y;
    v[1] += double(c.x) * gx.x + double(c.y) * gx.y;  // Re(chi conj(g))
    v[2] += double(gy.x) * gy.x + double(gy.y) * gy.y;
    v[3] += double(c.x) * gy.x + double(c.y) * gy.y;
  }
  block_reduce_sum_n(v);
  if (threadIdx.x == 0)
    for (int m = 0; m < 4; ++m) atomicAdd(&out[4 * k + m], v[m]);
}

// Position updates (one thread): shift = clamp(num/den, +-0.2); the column-gradient shift moves x (the row
// coordinate) and the row-gradient one y, as gradient_position_solver pairs them.
__global__ void k_var_posupd(double* __restrict__ s, const int* __restrict__ members, const int* __restrict__ gsize,
                             float* __restrict__ pos) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  const int G = *gsize;
  for (int k = 0; k < G; ++k) {
    const double dx = s[4 * k + 1] / s[4 * k], dy = s[4 * k + 3] / s[4 * k + 2];
    const double shx = fmin(fabs(dx), 0.2) * double((0.0 < dx) - (dx < 0.0));
    const double shy = fmin(fabs(dy), 0.2) * double((0.0 < dy) - (dy < 0.0));
    const int j = members[k];
    pos[2 * j] = float(double(pos[2 * j]) + shx);
    pos[2 * j + 1] = float(double(pos[2 * j + 1]) + shy);
    for (int m = 0; m < 4; ++m) s[4 * k + m] = 0.0;
  }
}

// Residual of window k at pixel i: (pu_k - pum/G) p/max(p)
__device__ __forceinline__ float2 var_resid(const float2* pu, const float2* pum, const float* pobj, float inv_pmax,
                                            int2 s, int k, int i, int N, int Y, float invG) {
  const float w = pobj[size_t(s.x + i / N) * Y + (s.y + i % N)] * inv_pmax;
  const float2 r = make_float2(pu[size_t(k) * N * N + i].x - pum[i].x * invG, pu[size_t(k) * N * N + i].y - pum[i].y * invG);
  return cscale(r, w);
}

// proj_k += sum Re(E conj(resid_k))
__global__ void k_var_proj(const float2* __restrict__ pu, const float2* __restrict__ pum,
                           const float* __restrict__ pobj, const float* __restrict__ pmax,
                           const float2* __restrict__ E, const int2* __restrict__ win, const int* __restrict__ members,
                           const int* __restrict__ gsize, int N, int Y, double* __restrict__ proj) {
  pdl_enter();
  const int k = blockIdx.y;
  const int G = *gsize;
  if (k >= G) return;
  const int2 s = win[members[k]];
  const float ip = 1.f / *pmax, invG = 1.f / float(G);
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 r = var_resid(pu, pum, pobj, ip, s, k, i, N, Y, invG);
    const float2 e = E[i];
    acc += double(e.x) * r.x + double(e.y) * r.y;
  }
  acc = block_reduce_sum(acc);
  if (threadIdx.x == 0) atomicAdd(&proj[k], acc);
}

// upd = sum_k resid_k prj_k / N^2 with prj_k = (mean_pixels Re(E conj(resid_k)) + evo1_k) / sum_group evo1^2 (each
// block computes the group's prj into shared memory); usum += sum |upd|^2
__global__ void k_var_upd(const float2* __restrict__ pu, const float2* __restrict__ pum,
                          const float* __restrict__ pobj, const float* __restrict__ pmax,
                          const double* __restrict__ proj, const double* __restrict__ evo, int P,
                          const int2* __restrict__ win, const int* __restrict__ members,
                          const int* __restrict__ gsize, int N, int Y, float2* __restrict__ upd,
                          double* __restrict__ usum) {
  pdl_enter();
  extern __shared__ float s_prj[];
  const int G = *gsize;
  if (threadIdx.x == 0) {
    double evn = 0;
    for (int k = 0; k < G; ++k) evn += evo[P + members[k]] * evo[P + members[k]];
    for (int k = 0; k < G; ++k) s_prj[k] = float((proj[k] / (double(N) * N) + evo[P + members[k]]) / evn);
  }
  __syncthreads();
  const float ip = 1.f / *pmax, invG = 1.f / float(G), nrm = 1.f / float(N * N);
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    float2 u = make_float2(0.f, 0.f);
    for (int k = 0; k < G; ++k) {
      const float2 r = var_resid(pu, pum, pobj, ip, win[members[k]], k, i, N, Y, invG);
      u = cadd(u, cscale(r, s_prj[k]));
    }
    u = cscale(u, nrm);
    upd[i] = u;
    acc += double(u.x) * u.x + double(u.y) * u.y;
  }
  acc = block_reduce_sum(acc);
  if (threadIdx.x == 0) atomicAdd(usum, acc);
}

// u <- E + u relax_U / max(1, rms(u)) (the new extra mode before its normalisation, kept in the update buffer);
// enew += sum |E_new|^2; clears the residual projections
__global__ void k_var_eapply(const float2* __restrict__ E, float2* __restrict__ upd, int NN,
                             const int* __restrict__ gsize, int P, const double* __restrict__ usum,
                             double* __restrict__ enew, double* __restrict__ proj) {
  pdl_enter();
  const double rms = sqrt(*usum / NN);
  const float us = float((double(*gsize) / P) / (rms > 1.0 ? rms : 1.0));
  if (blockIdx.x == 0 && threadIdx.x < *gsize) proj[threadIdx.x] = 0.0;
  double acc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NN; i += gridDim.x * blockDim.x) {
    const float2 e = cadd(E[i], cscale(upd[i], us));
    upd[i] = e;
    acc += double(e.x) * e.x + double(e.y) * e.y;
  }
  acc = block_reduce_sum(acc);
  if (threadIdx.x == 0) atomicAdd(enew, acc);
}

// E = E_new / rms(E_new) (stored by window 0's blocks); per window: sum |objp E|^2, Re(chi conj(objp E)),
// |objp P|^2, Re(chi conj(objp P))
__global__ void k_var_evosums(const float2* __restrict__ objp, const float2* __restrict__ Enew,
                              float2* __restrict__ E, const double* __restrict__ enew,
                              const float2* __restrict__ probe, const float2* __restrict__ chi,
                              const int* __restrict__ gsize, int N, double* __restrict__ out) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N;
  const float f = float(1.0 / sqrt(*enew / double(NN)));
  double v[4] = {0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 e = cscale(Enew[i], f);
    if (k == 0) E[i] = e;
    const float2 o = objp[k * NN + i], c = chi[k * NN + i];
    const float2 a = cmul(o, e), b = cmul(o, probe[i]);
    v[0] += double(a.x) * a.x + double(a.y) * a.y;
    v[1] += double(c.x) * a.x + double(c.y) * a.y;
    v[2] += double(b.x) * b.x + double(b.y) * b.y;
    v[3] += double(c.x) * b.x + double(c.y) * b.y;
  }
  block_reduce_sum_n(v);
  if (threadIdx.x == 0)
    for (int m = 0; m < 4; ++m) atomicAdd(&out[4 * k + m], v[m]);
}

// evo1 += mean num / (mean den + 0.1 group mean of mean den); evo0 += 0.1 sum num / sum den (one thread);
// clears the sums of this group's variable update
__global__ void k_var_evoupd(double* __restrict__ s, double* __restrict__ sc, double* __restrict__ evo, int P,
                             const int* __restrict__ members, const int* __restrict__ gsize, int NN) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  const int G = *gsize;
  double dm = 0;
  for (int k = 0; k < G; ++k) dm += s[4 * k] / NN;
  dm /= G;
  for (int k = 0; k < G; ++k) {
    const int j = members[k];
    evo[P + j] += (s[4 * k + 1] / NN) / (s[4 * k] / NN + 0.1 * dm);
    evo[j] += 0.1 * s[4 * k + 3] / s[4 * k + 2];
    for (int m = 0; m < 4; ++m) s[4 * k + m] = 0.0;
  }
  sc[SC_USUM] = 0.0;
  sc[SC_ENEW] = 0.0;
}

// Zone-plate probe start (initMLH, src/Probe.cpp:376-420 with d_initProbeMLH, src/ProbeKernels.cu:220-315):
// kern = C(r <= D_FZP/2) H(r >= D_H/2) e^{i lens r^2} e^{i kdz r^2} on the linspace(-dx N/2, dx N/2, N) grid of the
// zone plate, written fftshifted; pf = e^{ikz} e^{i kdz (u^2 + v^2)} on the detector frequencies in ifftshifted order.
// FP64 phases (the lens and propagation phases reach ~1e3 rad and nearly cancel).
struct ZonePlate {
  double start, step, lens, rC, rH, fu, startFU, fustep, kdz, kzc, kzs;
};

__global__ void k_fzp_start(float2* __restrict__ probe, float2* __restrict__ pf, int N, ZonePlate z) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const int r = i / N, c = i % N;
    const double x = z.start + z.step * c, y = z.start + z.step * r;
    const double s2 = x * x + y * y, rad = sqrt(s2);
    const double on = (rad <= z.rC ? 1.0 : 0.0) * (rad >= z.rH ? 1.0 : 0.0);
    double s1, c1, s3, c3;
    sincos(z.lens * s2, &s1, &c1);
    sincos(z.kdz * s2, &s3, &c3);
    const double kr = on * (c1 * c3 - s1 * s3), ki = on * (c1 * s3 + s1 * c3);
    probe[size_t((r + N / 2) % N) * N + (c + N / 2) % N] = make_float2(float(kr), float(ki));
    const double u = c < N / 2 ? z.startFU + z.fustep * c : -z.fu / 2 + z.fustep * (c - N / 2);
    const double v = r < N / 2 ? z.startFU + z.fustep * r : -z.fu / 2 + z.fustep * (r - N / 2);
    double sp, cp;
    sincos(z.kdz * (u * u + v * v), &sp, &cp);
    pf[i] = make_float2(float(z.kzc * cp - z.kzs * sp), float(z.kzc * sp + z.kzs * cp));
  }
}

// pf = FFT2(kern) pf
__global__ void k_fzp_mul(const float2* __restrict__ spec, float2* __restrict__ pf, int n) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pf[i] = cmul(spec[i], pf[i]);
}

// probe = fftshift(pf)
__global__ void k_fzp_shift(const float2* __restrict__ pf, float2* __restrict__ probe, int N) {
  pdl_enter();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const int r = i / N, c = i % N;
    probe[size_t((r + N / 2) % N) * N + (c + N / 2) % N] = pf[i];
  }
}

// Exit waves of modes 1..K-1: psik[m-1][k] = P_m objp_k
__global__ void k_var_psik(const float2* __restrict__ probe, const float2* __restrict__ objp, float2* __restrict__ psik,
                           int K, int Gmax, size_t NN) {
  pdl_enter();
  const size_t n = size_t(K - 1) * Gmax * NN;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < n; t += size_t(gridDim.x) * blockDim.x) {
    const size_t i = t % NN, k = (t / NN) % Gmax, m = t / (NN * Gmax) + 1;
    psik[t] = cmul(probe[m * NN + i], objp[k * NN + i]);
  }
}

// Modal modulus: |Psi| = sqrt(sum_m |Psi_m|^2) over all modes, every mode scaled by (A/(|Psi| + 1e-9) - 1)/N^2,
// Fourier error from |Psi| (modulus_constraint, get_fourier_error)
__global__ void k_var_modulus(float2* __restrict__ spec, float2* __restrict__ psik, const float* __restrict__ amp,
                              const int* __restrict__ members, const int* __restrict__ gsize, int N, int K, int Gmax,
                              double* __restrict__ err) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N, GN = size_t(Gmax) * NN;
  const float* A = amp + size_t(members[k]) * NN;
  const float nrm = 1.f / float(NN);
  double e = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 v = spec[k * NN + i];
    float a2 = v.x * v.x + v.y * v.y;
    for (int m = 0; m < K - 1; ++m) {
      const float2 w = psik[m * GN + k * NN + i];
      a2 += w.x * w.x + w.y * w.y;
    }
    const float ap = sqrtf(a2);
    const float a = A[i];
    e += double(a - ap) * double(a - ap) * 0.25;
    const float r = (a / (ap + 1e-9f) - 1.f) * nrm;
    spec[k * NN + i] = cscale(v, r);
    for (int m = 0; m < K - 1; ++m) psik[m * GN + k * NN + i] = cscale(psik[m * GN + k * NN + i], r);
  }
  e = block_reduce_sum(e);
  if (threadIdx.x == 0) atomicAdd(&err[k], e);
}

// Mode m >= 1: P_m += beta_p mean_j W chi_m,j conj(objp_j) (no sub-pixel shift for modes past the first)
__global__ void k_var_mode_update(const float2* __restrict__ chim, const float2* __restrict__ objp,
                                  const float* __restrict__ pobj, const float* __restrict__ maxIllum,
                                  const int2* __restrict__ win, const int* __restrict__ members,
                                  const int* __restrict__ gsize, int N, int Y, const double* __restrict__ betas,
                                  float2* __restrict__ mode) {
  pdl_enter();
  const int G = *gsize;
  const size_t NN = size_t(N) * N;
  const float damp = 0.01f * *maxIllum, invG = 1.f / float(G);
  const float2 b = make_float2(float(betas[2]), float(betas[3]));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    float2 acc = make_float2(0.f, 0.f);
    for (int k = 0; k < G; ++k) {
      const int2 s = win[members[k]];
      const float w = pobj[size_t(s.x + i / N) * Y + (s.y + i % N)];
      acc = cadd(acc, cscale(cmulc(chim[k * NN + i], objp[k * NN + i]), w / (w + damp)));
    }
    mode[i] = cadd(mode[i], cmul(b, cscale(acc, invG)));
  }
}

// ortho_modes (src/Probe.cpp:244-294) in one block: Gram-Schmidt in mode order with powers taken before each mode's
// projections, then modes 1..K-1 take the modes ranked 1..K-1 by that power (mode 0 stays, as written)
__global__ void k_var_ortho(float2* __restrict__ modes, float2* __restrict__ tmp, int K, int NN) {
  pdl_enter();
  __shared__ double pw[64];
  __shared__ float2 proj;
  __shared__ int rank[64];
  for (int i = 0; i < K; ++i) {
    float2* mi = modes + size_t(i) * NN;
    double p = 0;
    for (int t = threadIdx.x; t < NN; t += blockDim.x) p += double(mi[t].x) * mi[t].x + double(mi[t].y) * mi[t].y;
    p = block_reduce_sum(p);
    if (threadIdx.x == 0) pw[i] = p;
    __syncthreads();
    for (int j = 0; j < i; ++j) {
      const float2* mj = modes + size_t(j) * NN;
      double nj = 0, sr = 0, si = 0;
      for (int t = threadIdx.x; t < NN; t += blockDim.x) {
        const float2 a = mi[t], b = mj[t];
        nj += double(b.x) * b.x + double(b.y) * b.y;
        sr += double(a.x) * b.x + double(a.y) * b.y;  // a conj(b)
        si += double(a.y) * b.x - double(a.x) * b.y;
      }
      nj = block_reduce_sum(nj);
      __syncthreads();
      sr = block_reduce_sum(sr);
      __syncthreads();
      si = block_reduce_sum(si);
      if (threadIdx.x == 0) proj = make_float2(float(sr / nj), float(si / nj));
      __syncthreads();
      const float2 pr = proj;
      for (int t = threadIdx.x; t < NN; t += blockDim.x) mi[t] = make_float2(mi[t].x - (pr.x * mj[t].x - pr.y * mj[t].y),
                                                                             mi[t].y - (pr.x * mj[t].y + pr.y * mj[t].x));
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {  // order by power, descending; ties by index
    for (int i = 0; i < K; ++i) rank[i] = i;
    for (int i = 1; i < K; ++i)
      for (int j = i; j > 0 && pw[rank[j]] > pw[rank[j - 1]]; --j) {
        const int t = rank[j];
        rank[j] = rank[j - 1];
        rank[j - 1] = t;
      }
  }
  for (size_t t = threadIdx.x; t < size_t(K) * NN; t += blockDim.x) tmp[t] = modes[t];
  __syncthreads();
  for (int i = 1; i < K; ++i)
    for (int t = threadIdx.x; t < NN; t += blockDim.x) modes[size_t(i) * NN + t] = tmp[size_t(rank[i]) * NN + t];
}

// m_k = m_0 e^{-2 pi i (t1 (c/N - 0.5) + t2 (r/N - 0.5))}, k >= 1 (FP64 phase)
__global__ void k_mode_tilts(float2* __restrict__ probe, int K, int N, const double* __restrict__ tilts) {
  pdl_enter();
  const size_t NN = size_t(N) * N;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < size_t(K - 1) * NN;
       t += size_t(gridDim.x) * blockDim.x) {
    const int k = int(t / NN) + 1;
    const int i = int(t % NN), r = i / N, c = i % N;
    const double t1 = double(float(tilts[2 * (k - 1)])), t2 = double(float(tilts[2 * (k - 1) + 1]));
    double sn, cs;
    sincos(-2 * M_PI * (t1 * (double(c) / N - 0.5) + t2 * (double(r) / N - 0.5)), &sn, &cs);
    const float2 p = probe[i];
    probe[size_t(k) * NN + i] = make_float2(float(p.x * cs - p.y * sn), float(p.x * sn + p.y * cs));
  }
}

// gram[i K + j] = sum conj(m_i) m_j, one block per pair
__global__ void k_mode_gram(const float2* __restrict__ probe, int K, int NN, double2* __restrict__ gram) {
  pdl_enter();
  const int i = blockIdx.x / K, j = blockIdx.x % K;
  double sr = 0, si = 0;
  for (int t = threadIdx.x; t < NN; t += blockDim.x) {
    const float2 a = probe[size_t(i) * NN + t], b = probe[size_t(j) * NN + t];
    sr += double(a.x) * b.x + double(a.y) * b.y;
    si += double(a.x) * b.y - double(a.y) * b.x;
  }
  sr = block_reduce_sum(sr);
  __syncthreads();
  si = block_reduce_sum(si);
  if (threadIdx.x == 0) gram[blockIdx.x] = make_double2(sr, si);
}

// tmp_i = sum_q V(q, i) m_q, then copied back
__global__ void k_mode_combine(const float2* __restrict__ probe, float2* __restrict__ tmp, int K, int NN,
                               const double2* __restrict__ V) {
  pdl_enter();
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < size_t(K) * NN; t += size_t(gridDim.x) * blockDim.x) {
    const int i = int(t / NN);
    const size_t p = t % NN;
    double re = 0, im = 0;
    for (int q = 0; q < K; ++q) {
      const double2 v = V[size_t(q) * K + i];
      const float2 m = probe[size_t(q) * NN + p];
      re += m.x * v.x - m.y * v.y;
      im += m.x * v.y + m.y * v.x;
    }
    tmp[t] = make_float2(float(re), float(im));
  }
}

// Batched 2-D FFT in natural layout like fft2, both passes launched with programmatic dependent launch.
cudaError_t fft2_pdl_impl(float2* data, float2* work, const float2* tw, int batch, int N, bool inverse, cudaStream_t st) {
  return inverse ? fftx2<true>(N, work, data, tw, batch, ProLoad{data}, EpiStore{}, st)
                 : fftx2<false>(N, work, data, tw, batch, ProLoad{data}, EpiStore{}, st);
}

// Prologue of the probes' forward transform: objp_b = O[window_b] (stored on the side) and vp_b = P evo0 + E evo1
struct ProExit {
  const float2 *obj, *probe, *E;
  const double* evo;
  const int2* win;
  const int *members, *gsize;
  float2* objp;
  int P, Y;
  __device__ float2 operator()(int b, int x, int y, int L) const {
    const size_t i = size_t(x) * L + y, k = size_t(b) * L * L + i;
    if (b >= *gsize) {
      objp[k] = make_float2(0.f, 0.f);
      return make_float2(0.f, 0.f);
    }
    const int j = members[b];
    const int2 s = win[j];
    objp[k] = obj[size_t(s.x + x) * Y + (s.y + y)];
    return cadd(cscale(probe[i], float(evo[j])), cscale(E[i], float(evo[P + j])));
  }
};

// Spectrum times e^{-2 pi i sign (s.x f[y] + s.y f[x])} / N^2 (shift_probe)
struct EpiPhase {
  const float2* sub;
  const int *members, *gsize;
  float sign;
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    if (b >= *gsize) return v;
    const float2 s = sub[members[b]];
    const float tt = sign * (s.x * fft_freq(y, L) + s.y * fft_freq(x, L));
    float sn, cs;
    sincosf(-kTwoPi * tt, &sn, &cs);
    const float nrm = 1.f / float(L * L);
    return cmul(v, make_float2(cs * nrm, sn * nrm));
  }
  __device__ void finish(int) {}
};

// The shifted probe is stored; the exit wave psi = objp vp goes on the side
struct EpiVpPsi {
  const float2* objp;
  float2* psi;
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    const size_t k = (size_t(b) * L + x) * L + y;
    psi[k] = cmul(objp[k], v);
    return v;
  }
  __device__ void finish(int) {}
};

// Modulus (one probe mode): Psi (A/(|Psi| + 1e-9) - 1)/N^2 and the Fourier error of the window
struct EpiModulus {
  const float* amp;
  const int *members, *gsize;
  double* err;
  double e;
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    if (b >= *gsize) return v;
    const float ap = sqrtf(v.x * v.x + v.y * v.y);
    const float A = amp[size_t(members[b]) * L * L + size_t(x) * L + y];
    e += double(A - ap) * double(A - ap) * 0.25;
    return cscale(v, (A / (ap + 1e-9f) - 1.f) * (1.f / float(L * L)));
  }
  __device__ void finish(int b) {
    const double r = block_reduce_sum(e);
    if (threadIdx.x == 0 && b < *gsize) atomicAdd(&err[b], r);
  }
};

// chi is stored; pu = chi conj(objp) and S += chi conj(vp) at the window go on the side
struct EpiChi {
  const float2 *objp, *vp;
  const int2* win;
  const int *members, *gsize;
  float2 *pu, *S;
  int Y;
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    const size_t k = (size_t(b) * L + x) * L + y;
    if (b >= *gsize) {
      pu[k] = make_float2(0.f, 0.f);
      return v;
    }
    pu[k] = cmulc(v, objp[k]);
    const int2 s = win[members[b]];
    atomicAdd(&S[size_t(s.x + x) * Y + (s.y + y)], cmulc(v, vp[k]));
    return v;
  }
  __device__ void finish(int) {}
};

// Gradient spectra: d = 2 pi i FFT2(objp); dX = d f[y] stored, dY = d f[x] into plane Gmax + b
struct EpiGrad {
  float2* dy;  // aux + Gmax N^2
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    const float2 d = cmul(v, make_float2(0.f, kTwoPi));
    dy[(size_t(b) * L + x) * L + y] = cscale(d, fft_freq(x, L));
    return cscale(d, fft_freq(y, L));
  }
  __device__ void finish(int) {}
};

// Position-search sums of the gradient images (planes b < Gmax: dX of window b, else dY of window b - Gmax)
struct EpiPosSums {
  const float2 *vp, *chi;
  const int* gsize;
  double* out;
  int Gmax;
  double s0, s1;
  __device__ float2 operator()(int b, int x, int y, int L, float2 v) {
    const int k = b < Gmax ? b : b - Gmax;
    if (k >= *gsize) return v;
    const size_t i = (size_t(k) * L + x) * L + y;
    const float2 g = cmul(cscale(v, 1.f / float(L * L)), vp[i]), c = chi[i];
    s0 += double(g.x) * g.x + double(g.y) * g.y;
    s1 += double(c.x) * g.x + double(c.y) * g.y;
    return v;
  }
  __device__ void finish(int b) {
    double r[2] = {s0, s1};
    block_reduce_sum_n(r);
    const double r0 = r[0], r1 = r[1];
    const int k = b < Gmax ? b : b - Gmax, m = b < Gmax ? 0 : 2;
    if (threadIdx.x == 0 && k < *gsize) {
      atomicAdd(&out[4 * k + m], r0);
      atomicAdd(&out[4 * k + m + 1], r1);
    }
  }
};

// The group's six FP32 2-D transforms with one probe mode, from the exit waves to the shifted-back probe direction,
// as one launch: a thread-block cluster per window runs the twelve row passes with the pointwise steps in their loads
// and stores (the same functors as the separate passes) and cluster barriers between the passes.  Every step of the
// chain reads only its own window, so no hand-off leaves the cluster.
struct VarFront {
  ProExit exit;
  EpiPhase shift;
  EpiVpPsi vpsi;
  EpiModulus modulus;
  EpiChi chi;
  EpiPhase unshift;
  float2 *work, *vp, *psi, *pu;
  const float2* tw;
};

template <int L>
__global__ void __launch_bounds__(FftShape<L>::THREADS) k_var_front(VarFront a) {
  pdl_enter();
  extern __shared__ float4 smem4[];
  float2* s_tw = reinterpret_cast<float2*>(smem4);
  float2* s_x = s_tw + L;
  load_twiddles<L>(s_tw, a.tw);  // each row block starts with a CTA barrier
  const int b = blockIdx.y, rank = blockIdx.x, C = gridDim.x;
  fftx2_cluster<L, false>(a.work, a.vp, b, rank, C, s_tw, s_x, a.exit, a.shift);         // shifted probe
  fftx2_cluster<L, true>(a.work, a.vp, b, rank, C, s_tw, s_x, ProLoad{a.vp}, a.vpsi);    // vp, psi = objp vp
  fftx2_cluster<L, false>(a.work, a.psi, b, rank, C, s_tw, s_x, ProLoad{a.psi}, a.modulus);
  fftx2_cluster<L, true>(a.work, a.psi, b, rank, C, s_tw, s_x, ProLoad{a.psi}, a.chi);   // chi, pu, S
  fftx2_cluster<L, false>(a.work, a.pu, b, rank, C, s_tw, s_x, ProLoad{a.pu}, a.unshift);
  fftx2_cluster<L, true>(a.work, a.pu, b, rank, C, s_tw, s_x, ProLoad{a.pu}, EpiStore{});
}

// chosen once per process (the first session sets it up outside any graph capture, mls_var_prepare)
template <int L>
int front_cluster() {
  static const int C = fit_cluster(k_var_front<L>, L / FftShape<L>::RC, FftShape<L>::THREADS, rows_smem_bytes<L>());
  return C;
}

template <int L>
cudaError_t launch_var_front(const VarFront& a, int planes, cudaStream_t st) {
  return launch_cluster_pdl(k_var_front<L>, front_cluster<L>(), planes, FftShape<L>::THREADS, rows_smem_bytes<L>(),
                            st, a);
}

cudaError_t var_front(const VarFront& a, int N, int planes, cudaStream_t st) {
  switch (N) {
    case 32: return launch_var_front<32>(a, planes, st);
    case 64: return launch_var_front<64>(a, planes, st);
    case 128: return launch_var_front<128>(a, planes, st);
    case 256: return launch_var_front<256>(a, planes, st);
    default: return cudaErrorInvalidValue;
  }
}

int grid_n(size_t n, int cap = 1184) {
  size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > size_t(cap) ? cap : g));
}

}  // namespace

// The one-launch group transforms pay where a window's row blocks fill its cluster (one per CTA, N <= 256); at
// 512^2 a 16-CTA cluster per window leaves most SMs idle (measured 2.2x slower with one window per group), and the
// separate passes, 64 CTAs per window, stay.  Beside other scans' kernels (MLS_SEPARATE) the separate passes stay
// too: 16 scans of the batched workload measured 163.5 K patterns/s with the cluster launches, 193.3 K without.
bool mls_var_fused(int N, int K, bool tc) { return !tc && K == 1 && N <= 256; }

// Per session, on its device: the cluster size is chosen once per process, the kernel's attributes are set on every
// device that runs it
cudaError_t mls_var_prepare(int N) {
  int C = 0;
  cudaError_t e = cudaErrorInvalidValue;
#define PTY_FRONT(L)                                                          \
  case L:                                                                     \
    C = front_cluster<L>();                                                   \
    e = set_cluster_attributes(k_var_front<L>, rows_smem_bytes<L>());         \
    break;
  switch (N) {
    PTY_FRONT(32)
    PTY_FRONT(64)
    PTY_FRONT(128)
    PTY_FRONT(256)
    default:
      break;
  }
#undef PTY_FRONT
  cudaGetLastError();
  if (e != cudaSuccess) return e;
  return C >= 1 ? cudaSuccess : cudaErrorInvalidConfiguration;
}

size_t mls_var_scratch_doubles(int Gmax) { return 9 * size_t(Gmax) + 8; }

cudaError_t fft2_pdl(float2* data, float2* work, const float2* tw, int batch, int N, bool inverse, cudaStream_t st) {
  return fft2_pdl_impl(data, work, tw, batch, N, inverse, st);
}

cudaError_t mls_mode_tilts(float2* probe, int K, int N, const double* tilts, cudaStream_t st) {
  if (K < 2) return cudaSuccess;
  launch_pdl(k_mode_tilts, grid_n(size_t(K - 1) * N * N), 256, 0, st, probe, K, N, tilts);
  return cudaGetLastError();
}

cudaError_t mls_mode_gram(const float2* probe, int K, int N, double2* gram, cudaStream_t st) {
  launch_pdl(k_mode_gram, K * K, 256, 0, st, probe, K, N * N, gram);
  return cudaGetLastError();
}

cudaError_t mls_mode_combine(float2* probe, float2* tmp, int K, int N, const double2* V, cudaStream_t st) {
  const size_t n = size_t(K) * N * N;
  launch_pdl(k_mode_combine, grid_n(n), 256, 0, st, probe, tmp, K, N * N, V);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(probe, tmp, n * sizeof(float2), cudaMemcpyDeviceToDevice, st);
}

cudaError_t mls_zone_plate_probe(float2* probe, float2* pf, float2* work, const float2* tw, int N, double lambda,
                                 double dx_recon, double beamSize, cudaStream_t st) {
  const double Rn = 90e-6, dRn = 50e-9, D_FZP = 180e-6, D_H = 60e-6;
  const double fl = 2 * Rn * dRn / lambda;
  const double dx_fzp = lambda * fl / (N * dx_recon);
  const double k = 2 * M_PI / lambda, zz = fl + beamSize;
  ZonePlate z;
  z.step = dx_fzp * N / (N - 1);
  z.start = -dx_fzp * N / 2;
  z.lens = -2 / (lambda * 2 * fl) * M_PI;
  z.rC = D_FZP / 2;
  z.rH = D_H / 2;
  z.fu = lambda * (fl + beamSize) / dx_fzp;
  z.fustep = z.fu / (N - 1);
  z.startFU = -z.fu / 2 + z.fustep * (N / 2);
  z.kdz = k / (2 * zz);
  z.kzc = std::cos(k * zz);
  z.kzs = std::sin(k * zz);
  const int NN = N * N;
  launch_pdl(k_fzp_start, grid_n(NN), 256, 0, st, probe, pf, N, z);
  cudaError_t e = fft2(probe, work, tw, 1, N, false, st);
  if (e != cudaSuccess) return e;
  launch_pdl(k_fzp_mul, grid_n(NN), 256, 0, st, probe, pf, NN);
  launch_pdl(k_fzp_shift, grid_n(NN), 256, 0, st, pf, probe, N);
  return cudaGetLastError();
}

int mls_var_launches_per_iteration(int ngroups, unsigned flags, int K, bool tc, int N) {
  int pre = 1 + 4 + 1 + 2 + 1;  // boxes, norm (sums + 3 scales), recentre, illumination (2), max
  if (flags & MLS_WINDOWS) ++pre;
  if (flags & MLS_REMOVE) pre += 4;
  // per group: six 2-D transforms of two passes; FP32 fuses exit, both phase ramps, psi, the one-mode modulus and
  // the directions into them (one mode up to 256^2: all twelve passes in one cluster launch), the tensor-core path
  // runs them as 6 kernels (the modulus only for one mode); then pum, lsq with the solves, and the two updates
  int per = (mls_var_fused(N, K, tc) && !(flags & MLS_SEPARATE) ? 1 : 12) + 4 + (tc ? 6 + (K == 1 ? 1 : 0) : 0);
  if (flags & MLS_POSSEARCH) per += tc ? 2 + 1 + 2 + 1 + 1 : 2 + 2 + 1;
  if (flags & MLS_VARUPD) per += 5;
  // other modes: exit waves, forward and inverse 2-D transforms, the modal modulus, one update each
  if (K > 1) per += 1 + 2 + 1 + 2 + (K - 1);
  return pre + ngroups * per + (K > 1 ? 1 : 0);
}

cudaError_t mls_iteration_var(const MlsBuffers& b, int ngroups, unsigned flags, cudaStream_t st) {
  const int N = b.N, NN = N * N, P = b.P;
  const size_t XY = size_t(b.X) * b.Y, GN = size_t(b.Gmax) * NN;
  const VsLayout L{b.Gmax};
  double* sc = b.vs + L.sc();
  cudaError_t e;
  auto fft = [&](float2* d, int batch, bool inv) {
    return b.tc ? fft2_tc(d, b.work, batch, N, inv, b.tc_err, st) : fft2_pdl(d, b.work, b.tw, batch, N, inv, st);
  };
  if (flags & MLS_WINDOWS)
    launch_pdl(k_var_windows, (P + 255) / 256, 256, 0, st, b.pos, P, N, b.X, b.Y, b.cvx, b.cvy, b.win, b.sub);
  if ((e = mls_group_boxes(b.win, b.members, b.gsize, ngroups, b.Gmax, N, b.boxw, st)) != cudaSuccess) return e;
  // calc_object_norm over the object ROI with the current illumination weights: P, E scaled by on, O by 1/on
  if ((e = mls_norm_sums(b.pobj, b.obj, b.Y, b.roi[0], b.roi[1], b.roi[2], b.roi[3], 1, b.normsums, st)) != cudaSuccess)
    return e;
  if ((e = scale_by_norm(b.probe, size_t(b.K) * NN, b.normsums, 0, st)) != cudaSuccess) return e;
  if ((e = scale_by_norm(b.E, NN, b.normsums, 0, st)) != cudaSuccess) return e;
  if ((e = scale_by_norm(b.obj, XY, b.normsums, 1, st)) != cudaSuccess) return e;
  launch_pdl(k_var_recentre, 1, 256, 0, st, b.pos, b.pos_o, P);
  if (flags & MLS_REMOVE) {
    launch_pdl(k_var_sumsq, grid_n(NN, 64), 256, 0, st, b.E, NN, sc + SC_ESUM);
    launch_pdl(k_var_remove, 1, 32, 0, st, sc, b.evo, P, NN);
    launch_pdl(k_var_scale, grid_n(NN), 256, 0, st, b.E, NN, sc + SC_EFAC);
    launch_pdl(k_var_scale, grid_n(NN), 256, 0, st, b.probe, NN, sc + SC_PFAC);
  }
  // updated_cached_illumination: p = (p + sum |P|^2 at the windows) / 2; its maximum for the variable update
  if ((e = scale_real(b.pobj, XY, 0.5f, st)) != cudaSuccess) return e;
  if ((e = mls_illum_add(b.pobj, b.probe, b.win, P, N, b.Y, 0.5f, st)) != cudaSuccess) return e;
  if ((e = max_real(b.pobj, XY, b.pmax, st)) != cudaSuccess) return e;
  const int gb = (NN + 255) / 256 > 64 ? 64 : (NN + 255) / 256;
  const dim3 grid(gb, b.Gmax);
  const bool fused = mls_var_fused(N, b.K, b.tc) && !(flags & MLS_SEPARATE);
  for (int g = 0; g < ngroups; ++g) {
    const int* mem = b.members + size_t(g) * b.Gmax;
    const int* gs = b.gsize + g;
    // the position search needs this group's windows, probes and chi only, and writes positions that no kernel
    // reads before the next iteration: it runs on the side stream while the group goes on, and joins before the
    // next group rewrites those buffers
    auto possearch_fork = [&]() -> cudaError_t {
      cudaError_t r;
      if ((r = cudaEventRecord(b.ev_fork, st)) != cudaSuccess) return r;
      if ((r = cudaStreamWaitEvent(b.side, b.ev_fork, 0)) != cudaSuccess) return r;
      if ((r = fftx2<false>(N, b.work2, b.aux, b.tw, b.Gmax, ProLoad{b.objp}, EpiGrad{b.aux + GN}, b.side)) !=
          cudaSuccess)
        return r;
      const EpiPosSums ps{b.vp, b.psi, gs, b.vs + L.pos(), b.Gmax, 0.0, 0.0};
      if ((r = fftx2<true>(N, b.work2, b.aux, b.tw, 2 * b.Gmax, ProLoad{b.aux}, ps, b.side)) != cudaSuccess) return r;
      launch_pdl(k_var_posupd, 1, 32, 0, b.side, b.vs + L.pos(), mem, gs, b.pos);
      return cudaEventRecord(b.ev_join, b.side);
    };
    if (fused) {  // FP32, one mode: the six transforms and their pointwise steps in one cluster launch
      const VarFront a{ProExit{b.obj, b.probe, b.E, b.evo, b.win, mem, gs, b.objp, P, b.Y},
                       EpiPhase{b.sub, mem, gs, 1.f},
                       EpiVpPsi{b.objp, b.psi},
                       EpiModulus{b.amp, mem, gs, b.errk, 0.0},
                       EpiChi{b.objp, b.vp, b.win, mem, gs, b.pu, b.S, b.Y},
                       EpiPhase{b.sub, mem, gs, -1.f},
                       b.work, b.vp, b.psi, b.pu, b.tw};
      if ((e = var_front(a, N, b.Gmax, st)) != cudaSuccess) return e;
      if ((flags & MLS_POSSEARCH) && (e = possearch_fork()) != cudaSuccess) return e;
    } else {
      if (b.tc) {  // tensor-core transforms: separate pointwise kernels around fft2_tc
        launch_pdl(k_var_exit, grid, 256, 0, st, b.obj, b.probe, b.E, b.evo, P, b.win, mem, gs, N, b.Y, b.objp, b.vp);
        if ((e = fft(b.vp, b.Gmax, false)) != cudaSuccess) return e;
        launch_pdl(k_var_phase, grid, 256, 0, st, b.vp, b.sub, mem, gs, N, 1.f);
        if ((e = fft(b.vp, b.Gmax, true)) != cudaSuccess) return e;
        launch_pdl(k_var_psi, grid_n(GN), 256, 0, st, b.objp, b.vp, b.psi, GN);
        if ((e = fft(b.psi, b.Gmax, false)) != cudaSuccess) return e;
      } else {  // FP32 transforms with the pointwise steps fused into their loads and stores
        const ProExit pe{b.obj, b.probe, b.E, b.evo, b.win, mem, gs, b.objp, P, b.Y};
        if ((e = fftx2<false>(N, b.work, b.vp, b.tw, b.Gmax, pe, EpiPhase{b.sub, mem, gs, 1.f}, st)) != cudaSuccess)
          return e;
        if ((e = fftx2<true>(N, b.work, b.vp, b.tw, b.Gmax, ProLoad{b.vp}, EpiVpPsi{b.objp, b.psi}, st)) !=
            cudaSuccess)
          return e;
        if (b.K == 1) {
          if ((e = fftx2<false>(N, b.work, b.psi, b.tw, b.Gmax, ProLoad{b.psi},
                                EpiModulus{b.amp, mem, gs, b.errk, 0.0}, st)) != cudaSuccess)
            return e;
        } else if ((e = fft(b.psi, b.Gmax, false)) != cudaSuccess) {
          return e;
        }
      }
      if (b.K > 1) {
        launch_pdl(k_var_psik, grid_n(size_t(b.K - 1) * GN), 256, 0, st, b.probe, b.objp, b.psik, b.K, b.Gmax, NN);
        if ((e = fft(b.psik, (b.K - 1) * b.Gmax, false)) != cudaSuccess) return e;
        launch_pdl(k_var_modulus, grid, 256, 0, st, b.psi, b.psik, b.amp, mem, gs, N, b.K, b.Gmax, b.errk);
        if ((e = fft(b.psik, (b.K - 1) * b.Gmax, true)) != cudaSuccess) return e;
      } else if (b.tc && (e = mls_modulus(b, mem, gs, st)) != cudaSuccess) {
        return e;
      }
      if (b.tc) {
        if ((e = fft(b.psi, b.Gmax, true)) != cudaSuccess) return e;
        launch_pdl(k_var_dirs, grid, 256, 0, st, b.psi, b.objp, b.vp, b.win, mem, gs, N, b.Y, b.pu, b.S);
        if ((e = fft(b.pu, b.Gmax, false)) != cudaSuccess) return e;
        launch_pdl(k_var_phase, grid, 256, 0, st, b.pu, b.sub, mem, gs, N, -1.f);
      } else {
        const EpiChi ec{b.objp, b.vp, b.win, mem, gs, b.pu, b.S, b.Y};
        if ((e = fftx2<true>(N, b.work, b.psi, b.tw, b.Gmax, ProLoad{b.psi}, ec, st)) != cudaSuccess) return e;
        if ((flags & MLS_POSSEARCH) && (e = possearch_fork()) != cudaSuccess) return e;
        if ((e = fftx2<false>(N, b.work, b.pu, b.tw, b.Gmax, ProLoad{b.pu}, EpiPhase{b.sub, mem, gs, -1.f}, st)) !=
            cudaSuccess)
          return e;
      }
      if ((e = fft(b.pu, b.Gmax, true)) != cudaSuccess) return e;
    }
    launch_pdl(k_var_pum, grid_n(NN, 256), 256, 0, st, b.pu, b.pobj, b.maxIllum, b.win, mem, gs, N, b.Y, b.pum);
    if ((e = mls_lsq(b, b.vp, NN, mem, gs, st)) != cudaSuccess) return e;
    if ((e = mls_solve_update(b, mem, gs, b.boxw + 4 * size_t(g), 0, st)) != cudaSuccess) return e;
    if ((flags & MLS_POSSEARCH) && b.tc) {
      if ((e = cudaMemcpyAsync(b.aux, b.objp, GN * sizeof(float2), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return e;
      if ((e = fft(b.aux, b.Gmax, false)) != cudaSuccess) return e;
      launch_pdl(k_var_grad, grid, 256, 0, st, b.aux, b.Gmax, N);
      if ((e = fft(b.aux, 2 * b.Gmax, true)) != cudaSuccess) return e;
      launch_pdl(k_var_possums, grid, 256, 0, st, b.aux, b.vp, b.psi, gs, b.Gmax, N, b.vs + L.pos());
      launch_pdl(k_var_posupd, 1, 32, 0, st, b.vs + L.pos(), mem, gs, b.pos);
    }
    if (flags & MLS_VARUPD) {
      launch_pdl(k_var_proj, grid, 256, 0, st, b.pu, b.pum, b.pobj, b.pmax, b.E, b.win, mem, gs, N, b.Y, b.vs + L.proj());
      launch_pdl(k_var_upd, grid_n(NN, 256), 256, sizeof(float) * b.Gmax, st, b.pu, b.pum, b.pobj, b.pmax,
                 b.vs + L.proj(), b.evo, P, b.win, mem, gs, N, b.Y, b.vupd, sc + SC_USUM);
      launch_pdl(k_var_eapply, grid_n(NN, 256), 256, 0, st, b.E, b.vupd, NN, gs, P, sc + SC_USUM, sc + SC_ENEW,
                 b.vs + L.proj());
      launch_pdl(k_var_evosums, grid, 256, 0, st, b.objp, b.vupd, b.E, sc + SC_ENEW, b.probe, b.psi, gs, N,
                 b.vs + L.evs());
      launch_pdl(k_var_evoupd, 1, 32, 0, st, b.vs + L.evs(), sc, b.evo, P, mem, gs, NN);
    }
    for (int m = 1; m < b.K; ++m)  // modes past the first: their directions with the group's probe step
      launch_pdl(k_var_mode_update, grid_n(NN, 256), 256, 0, st, b.psik + size_t(m - 1) * GN, b.objp, b.pobj, b.maxIllum,
                                                          b.win, mem, gs, N, b.Y, b.betas, b.probe + size_t(m) * NN);
    if ((flags & MLS_POSSEARCH) && !b.tc && (e = cudaStreamWaitEvent(st, b.ev_join, 0)) != cudaSuccess) return e;
  }
  if (b.K > 1) launch_pdl(k_var_ortho, 1, 1024, 0, st, b.probe, b.mtmp, b.K, NN);
  return cudaGetLastError();
}

}  // namespace pty
