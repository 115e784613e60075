// MLs core (LSQ-ML with random sparse groups; src/MLS.cpp:74-490 and its callees) for one probe mode and one
// object.  Per group of G positions (G = max(1, P/100)):
//   exit      obj_proj = O[window], psi = P * obj_proj                      (get_projections, get_illumination_probe)
//   FFT2      Psi
//   modulus   chi-spectrum = Psi * (A/(|Psi| + 1e-9) - 1) / N^2, Fourier error (modulus_constraint,
//             get_fourier_error, src/Diffractions.cpp:255-310)
//   IFFT2     chi
//   dirs      probe direction  sum_j W[window] chi conj(obj_proj), W = p/(p + 0.01 MAX_ILLUM)
//             object direction S += chi conj(P) at the windows                (src/MLS.cpp:249-347)
//   lsq       per-window sums of |dOP|^2, |dPO|^2, dOP conj(dPO), Re(conj(dOP) chi), Re(conj(dPO) chi) with the
//             preconditioned object step S/(p + delta_p MAX_ILLUM)  (d_get_optimal_step_lsq,
//             src/utilitiesKernels.cu:444-466), FP64
//   solve     regularised 2x2 Hermitian systems (src/MLS.cpp:379-417), group-mean steps
//   update    O += beta_o S/(p + delta_p MAX_ILLUM) over the group's bounding box, P += beta_p * mean direction
//             (Sample::update_object, Probe::update_probe)
// The whole iteration (calc_object_norm, cached illumination, all groups) is one CUDA graph; the random group
// tables live in device memory and are rewritten before each replay.  This is the fixed-probe core; the reference's
// default path (variable probe, sub-pixel shift, position search) is kernels_mls_var.cu, built on the same kernels.
#include "fft_core.cuh"
#include "kernel_util.cuh"
#include "kernels_mls.h"
#include "pdl.cuh"

namespace pty {

// p[r0+x][c0+y] += scale * |P[x][y]|^2 for every window (set_projections of |P|^2).
__global__ void k_mls_illum_add(float* __restrict__ pobj, const float2* __restrict__ probe,
                                const int2* __restrict__ starts, int N, int Y, float scale) {
  pdl_enter();
  const int j = blockIdx.y;
  const int2 s = starts[j];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const int x = i / N, y = i % N;
    const float2 v = probe[i];
    const float m = sqrtf(v.x * v.x + v.y * v.y);
    atomicAdd(&pobj[size_t(s.x + x) * Y + (s.y + y)], scale * m * m);
  }
}

__global__ void k_scale_real(float* __restrict__ a, size_t n, float s) {
  pdl_enter();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] *= s;
}

// out[0] += sum w^q, out[1] += sum w^q |O|^2 over the rectangle [x0, x0+nx) x [y0, y0+ny), q = 2 (squared) or 1
__global__ void k_mls_norm_sums(const float* __restrict__ w, const float2* __restrict__ obj, int Y, int x0, int y0,
                                int nx, int ny, int squared, double* __restrict__ out) {
  pdl_enter();
  double sw = 0, so = 0;
  const int n = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t k = size_t(x0 + i / ny) * Y + (y0 + i % ny);
    const double ww = squared ? double(w[k]) * w[k] : double(w[k]);
    const float2 o = obj[k];
    sw += ww;
    so += ww * (double(o.x) * o.x + double(o.y) * o.y);
  }
  sw = block_reduce_sum(sw);
  __syncthreads();
  so = block_reduce_sum(so);
  if (threadIdx.x == 0) {
    atomicAdd(&out[0], sw);
    atomicAdd(&out[1], so);
  }
}

// calc_object_norm: on = sqrt(sum w^2|O|^2 / sum w^2); P *= on, O /= on (mode 0: multiply a by on, 1: divide).
// An empty or unlit ROI (sum w^2 = 0, e.g. a single scan line) leaves both unscaled.
__global__ void k_scale_by_norm(float2* __restrict__ a, size_t n, const double* __restrict__ sums, int divide) {
  pdl_enter();
  const double on = sums[0] > 0.0 ? sqrt(sums[1]) / sqrt(sums[0]) : 1.0;
  const float s = divide ? float(1.0 / on) : float(on);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = cscale(a[i], s);
}

__global__ void k_mls_exit(const float2* __restrict__ obj, const float2* __restrict__ probe,
                           const int2* __restrict__ starts, const int* __restrict__ members,
                           const int* __restrict__ gsize, int N, int Y, float2* __restrict__ objp,
                           float2* __restrict__ psi) {
  pdl_enter();
  const int k = blockIdx.y;
  const size_t NN = size_t(N) * N;
  const bool live = k < *gsize;
  const int2 s = live ? starts[members[k]] : make_int2(0, 0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    float2 o = make_float2(0.f, 0.f), e = make_float2(0.f, 0.f);
    if (live) {
      o = obj[size_t(s.x + i / N) * Y + (s.y + i % N)];
      e = cmul(probe[i], o);
    }
    objp[k * NN + i] = o;
    psi[k * NN + i] = e;
  }
}

__global__ void k_mls_modulus(float2* __restrict__ spec, const float* __restrict__ amp,
                              const int* __restrict__ members, const int* __restrict__ gsize, int N,
                              double* __restrict__ err) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N;
  const float* A = amp + size_t(members[k]) * NN;
  const float nrm = 1.f / float(NN);
  double e = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 v = spec[k * NN + i];
    const float ap = sqrtf(v.x * v.x + v.y * v.y);
    const float a = A[i];
    e += double(a - ap) * double(a - ap) * 0.25;
    const float r = (a / (ap + 1e-9f) - 1.f) * nrm;
    spec[k * NN + i] = cscale(v, r);
  }
  e = block_reduce_sum(e);
  if (threadIdx.x == 0) atomicAdd(&err[k], e);
}

__global__ void k_mls_dirs(const float2* __restrict__ chi, const float2* __restrict__ objp,
                           const float2* __restrict__ probe, const float* __restrict__ pobj,
                           const float* __restrict__ maxIllum, const int2* __restrict__ starts,
                           const int* __restrict__ members, const int* __restrict__ gsize, int N, int Y,
                           float2* __restrict__ pum, float2* __restrict__ S) {
  pdl_enter();
  const int k = blockIdx.y;
  if (k >= *gsize) return;
  const size_t NN = size_t(N) * N;
  const int2 s = starts[members[k]];
  const float damp = 0.01f * *maxIllum;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const float2 c = chi[k * NN + i];
    const size_t o = size_t(s.x + i / N) * Y + (s.y + i % N);
    const float w = pobj[o];
    const float2 pu = cmulc(c, objp[k * NN + i]);
    atomicAdd(&pum[i], cscale(pu, w / (w + damp)));
    atomicAdd(&S[o], cmulc(c, probe[i]));
  }
}

// Regularised 2x2 solves, group-mean steps, Fourier error; clears the per-group accumulators (one thread; sums and
// errk read from L2, where the atomics of the group's blocks landed).
__device__ void mls_solve_group(double* sums, double* errk, int G, int N, double beta_obj, double beta_probe,
                                double* betas, double* err_total) {
  double m1 = 0, m4 = 0;
  for (int k = 0; k < G; ++k) {
    m1 += __ldcg(&sums[k * 6 + 0]);
    m4 += __ldcg(&sums[k * 6 + 1]);
  }
  m1 = 0.1 * m1 / G;
  m4 = 0.1 * m4 / G;
  double bor = 0, boi = 0, bpr = 0, bpi = 0, e = 0;
  for (int k = 0; k < G; ++k) {
    const double A11 = __ldcg(&sums[k * 6 + 0]) + m1, A22 = __ldcg(&sums[k * 6 + 1]) + m4;
    const double cr = __ldcg(&sums[k * 6 + 2]), ci = __ldcg(&sums[k * 6 + 3]);  // A12 = c, A21 = conj(c)
    const double b1 = __ldcg(&sums[k * 6 + 4]), b2 = __ldcg(&sums[k * 6 + 5]);
    const double det = A11 * A22 - (cr * cr + ci * ci);      // real for a Hermitian 2x2
    // x0 = (b1 A22 - c b2)/det, x1 = (A11 b2 - conj(c) b1)/det
    bor += (b1 * A22 - cr * b2) / det;
    boi += (-ci * b2) / det;
    bpr += (A11 * b2 - cr * b1) / det;
    bpi += (ci * b1) / det;
    e += sqrt(__ldcg(&errk[k]) / (double(N) * N));
    for (int m = 0; m < 6; ++m) sums[k * 6 + m] = 0.0;
    errk[k] = 0.0;
  }
  betas[0] = beta_obj * bor / G;
  betas[1] = beta_obj * boi / G;
  betas[2] = beta_probe * bpr / G;
  betas[3] = beta_probe * bpi / G;
  *err_total += e;
}

// LSQ sums of window k of the group (its blocks' share), added into sums[k * 6 ..]
__device__ __forceinline__ void lsq_window_sums(const float2* __restrict__ chi, const float2* __restrict__ objp,
                                                const float2* __restrict__ probe, size_t pstride,
                                                const float2* __restrict__ pum, const float2* __restrict__ S,
                                                const float* __restrict__ pobj, const float* __restrict__ maxIllum,
                                                float delta_p, const int2* __restrict__ starts,
                                                const int* __restrict__ members, int G, int k, int N, int Y,
                                                double* sums) {
  const size_t NN = size_t(N) * N;
  const int2 s = starts[members[k]];
  const float dmax = *maxIllum * delta_p, invG = 1.f / float(G);
  const float lam = 1.1920928955078125e-07f / float(NN);  // FLT_EPSILON / N^2
  double a1 = 0, a4 = 0, a2r = 0, a2i = 0, b1 = 0, b2 = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N * N; i += gridDim.x * blockDim.x) {
    const size_t o = size_t(s.x + i / N) * Y + (s.y + i % N);
    const float2 oup = cscale(S[o], 1.f / (pobj[o] + dmax));
    const float2 dOP = cmul(oup, probe[k * pstride + i]);
    const float2 dPO = cmul(cscale(pum[i], invG), objp[k * NN + i]);
    const float2 c = chi[k * NN + i];
    a1 += double(dOP.x * dOP.x + dOP.y * dOP.y + lam);
    a4 += double(dPO.x * dPO.x + dPO.y * dPO.y + lam);
    const float2 x2 = cmulc(dOP, dPO);
    a2r += x2.x;
    a2i += x2.y;
    b1 += double(dOP.x * c.x + dOP.y * c.y);  // Re(conj(dOP) chi)
    b2 += double(dPO.x * c.x + dPO.y * c.y);
  }
  double v[6] = {a1, a4, a2r, a2i, b1, b2};
  block_reduce_sum_n(v);
  if (threadIdx.x == 0)
    for (int m = 0; m < 6; ++m) atomicAdd(&sums[k * 6 + m], v[m]);
}

// probe: one N x N probe for every window (pstride 0) or one per window (pstride N^2).
__global__ void k_mls_lsq(const float2* __restrict__ chi, const float2* __restrict__ objp,
                          const float2* __restrict__ probe, size_t pstride, const float2* __restrict__ pum,
                          const float2* __restrict__ S, const float* __restrict__ pobj,
                          const float* __restrict__ maxIllum, float delta_p, const int2* __restrict__ starts,
                          const int* __restrict__ members, const int* __restrict__ gsize, int N, int Y,
                          double* __restrict__ sums, unsigned* __restrict__ done, double* __restrict__ errk,
                          double beta_obj, double beta_probe, double* __restrict__ betas,
                          double* __restrict__ err_total) {
  pdl_enter();
  const int k = blockIdx.y;
  const int G = *gsize;
  if (k < G) lsq_window_sums(chi, objp, probe, pstride, pum, S, pobj, maxIllum, delta_p, starts, members, G, k, N, Y,
                             sums);
  // the last block to finish solves the group on the completed sums (no separate one-thread launch)
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x * gridDim.y - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    *done = 0u;
    mls_solve_group(sums, errk, G, N, beta_obj, beta_probe, betas, err_total);
  }
}

__global__ void k_mls_update_object(float2* __restrict__ obj, float2* __restrict__ S, const float* __restrict__ pobj,
                                    const float* __restrict__ maxIllum, float delta_p, const double* __restrict__ betas,
                                    const int* __restrict__ bbox, int Y) {
  pdl_enter();
  const int x0 = bbox[0], y0 = bbox[1], nx = bbox[2], ny = bbox[3];
  const float2 b = make_float2(float(betas[0]), float(betas[1]));
  const float dmax = *maxIllum * delta_p;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx * ny; i += gridDim.x * blockDim.x) {
    const size_t o = size_t(x0 + i / ny) * Y + (y0 + i % ny);
    const float2 sv = S[o];
    if (sv.x != 0.f || sv.y != 0.f) {
      obj[o] = cadd(obj[o], cmul(b, cscale(sv, 1.f / (pobj[o] + dmax))));
      S[o] = make_float2(0.f, 0.f);
    }
  }
}

// P += beta_p * pum / G; clear = 1 zeroes the accumulator for the next group's atomics.
__global__ void k_mls_update_probe(float2* __restrict__ probe, float2* __restrict__ pum, const double* __restrict__ betas,
                                   const int* __restrict__ gsize, int n, int clear) {
  pdl_enter();
  const float2 b = make_float2(float(betas[2]), float(betas[3]));
  const float invG = 1.f / float(*gsize);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    probe[i] = cadd(probe[i], cmul(b, cscale(pum[i], invG)));
    if (clear) pum[i] = make_float2(0.f, 0.f);
  }
}

// Bounding box (x0, y0, nx, ny) of each group's windows.
__global__ void k_mls_bbox(const int2* __restrict__ starts, const int* __restrict__ members,
                           const int* __restrict__ gsize, int ngroups, int Gmax, int N, int* __restrict__ bbox) {
  pdl_enter();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  int x0 = 1 << 30, y0 = 1 << 30, x1 = 0, y1 = 0;
  for (int m = 0; m < gsize[g]; ++m) {
    const int2 s = starts[members[size_t(g) * Gmax + m]];
    x0 = min(x0, s.x);
    y0 = min(y0, s.y);
    x1 = max(x1, s.x + N);
    y1 = max(y1, s.y + N);
  }
  bbox[4 * g] = x0;
  bbox[4 * g + 1] = y0;
  bbox[4 * g + 2] = x1 - x0;
  bbox[4 * g + 3] = y1 - y0;
}

static int grid_for(size_t n, int cap = 1184) {
  size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > size_t(cap) ? cap : g));
}

cudaError_t mls_illum_add(float* pobj, const float2* probe, const int2* starts, int P, int N, int Y, float scale,
                          cudaStream_t st) {
  dim3 grid((N * N + 255) / 256, P);
  launch_pdl(k_mls_illum_add, grid, 256, 0, st, pobj, probe, starts, N, Y, scale);
  return cudaGetLastError();
}

cudaError_t scale_real(float* a, size_t n, float s, cudaStream_t st) {
  launch_pdl(k_scale_real, grid_for(n), 256, 0, st, a, n, s);
  return cudaGetLastError();
}

cudaError_t scale_by_norm(float2* a, size_t n, const double* sums, int divide, cudaStream_t st) {
  launch_pdl(k_scale_by_norm, grid_for(n), 256, 0, st, a, n, sums, divide);
  return cudaGetLastError();
}

cudaError_t mls_norm_sums(const float* w, const float2* obj, int Y, int x0, int y0, int nx, int ny, int squared,
                          double* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(double), st);
  if (e != cudaSuccess) return e;
  launch_pdl(k_mls_norm_sums, grid_for(size_t(nx) * ny), 256, 0, st, w, obj, Y, x0, y0, nx, ny, squared, out);
  return cudaGetLastError();
}

__global__ void k_sqrt_inplace(float* __restrict__ a, size_t n) {
  pdl_enter();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = sqrtf(a[i]);
}

cudaError_t sqrt_inplace(float* a, size_t n, cudaStream_t st) {
  launch_pdl(k_sqrt_inplace, grid_for(n), 256, 0, st, a, n);
  return cudaGetLastError();
}

__global__ void k_max_real(const float* __restrict__ a, size_t n, float* out) {
  pdl_enter();
  float m = 0.f;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    m = fmaxf(m, a[i]);
  m = block_reduce_maxf(m);
  if (threadIdx.x == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(m));
}

cudaError_t max_real(const float* a, size_t n, float* out, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float), st);
  if (e != cudaSuccess) return e;
  launch_pdl(k_max_real, grid_for(n), 256, 0, st, a, n, out);
  return cudaGetLastError();
}

cudaError_t mls_iteration(const MlsBuffers& b, int ngroups, cudaStream_t st) {
  const int N = b.N, NN = N * N;
  const size_t XY = size_t(b.X) * b.Y;
  cudaError_t e;
  // calc_object_norm over the object ROI with the current illumination weights
  if ((e = cudaMemsetAsync(b.normsums, 0, 2 * sizeof(double), st)) != cudaSuccess) return e;
  launch_pdl(k_mls_norm_sums, grid_for(size_t(b.roi[2]) * b.roi[3]), 256, 0, st, b.pobj, b.obj, b.Y, b.roi[0], b.roi[1],
                                                                           b.roi[2], b.roi[3], 1, b.normsums);
  launch_pdl(k_scale_by_norm, grid_for(NN), 256, 0, st, b.probe, NN, b.normsums, 0);
  launch_pdl(k_scale_by_norm, grid_for(XY), 256, 0, st, b.obj, XY, b.normsums, 1);
  // updated_cached_illumination: p = (p + sum |P|^2 at the windows) / 2
  launch_pdl(k_scale_real, grid_for(XY), 256, 0, st, b.pobj, XY, 0.5f);
  dim3 gi((NN + 255) / 256, b.P);
  launch_pdl(k_mls_illum_add, gi, 256, 0, st, b.pobj, b.probe, b.starts, N, b.Y, 0.5f);
  const int gb = (NN + 255) / 256 > 64 ? 64 : (NN + 255) / 256;
  for (int g = 0; g < ngroups; ++g) {
    const int* mem = b.members + size_t(g) * b.Gmax;
    const int* gs = b.gsize + g;
    dim3 grid(gb, b.Gmax);
    launch_pdl(k_mls_exit, grid, 256, 0, st, b.obj, b.probe, b.starts, mem, gs, N, b.Y, b.objp, b.psi);
    if ((e = b.tc ? fft2_tc(b.psi, b.work, b.Gmax, N, false, b.tc_err, st)
                  : fft2_pdl(b.psi, b.work, b.tw, b.Gmax, N, false, st)) != cudaSuccess)
      return e;
    launch_pdl(k_mls_modulus, grid, 256, 0, st, b.psi, b.amp, mem, gs, N, b.errk);
    if ((e = b.tc ? fft2_tc(b.psi, b.work, b.Gmax, N, true, b.tc_err, st)
                  : fft2_pdl(b.psi, b.work, b.tw, b.Gmax, N, true, st)) != cudaSuccess)
      return e;
    launch_pdl(k_mls_dirs, grid, 256, 0, st, b.psi, b.objp, b.probe, b.pobj, b.maxIllum, b.starts, mem, gs, N, b.Y, b.pum,
                                     b.S);
    if ((e = mls_lsq(b, b.probe, 0, mem, gs, st)) != cudaSuccess) return e;
    if ((e = mls_solve_update(b, mem, gs, b.bbox + 4 * size_t(g), 1, st)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

int mls_launches_per_iteration(int ngroups) { return 5 + ngroups * 10; }

cudaError_t mls_group_boxes(const int2* starts, const int* members, const int* gsize, int ngroups, int Gmax, int N,
                            int* bbox, cudaStream_t st) {
  launch_pdl(k_mls_bbox, (ngroups + 127) / 128, 128, 0, st, starts, members, gsize, ngroups, Gmax, N, bbox);
  return cudaGetLastError();
}

cudaError_t mls_modulus(const MlsBuffers& b, const int* members, const int* gsize, cudaStream_t st) {
  const int NN = b.N * b.N;
  dim3 grid((NN + 255) / 256 > 64 ? 64 : (NN + 255) / 256, b.Gmax);
  launch_pdl(k_mls_modulus, grid, 256, 0, st, b.psi, b.amp, members, gsize, b.N, b.errk);
  return cudaGetLastError();
}

cudaError_t mls_lsq(const MlsBuffers& b, const float2* probe, size_t pstride, const int* members, const int* gsize,
                    cudaStream_t st) {
  const int NN = b.N * b.N;
  dim3 grid((NN + 255) / 256 > 64 ? 64 : (NN + 255) / 256, b.Gmax);
  launch_pdl(k_mls_lsq, grid, 256, 0, st, b.psi, b.objp, probe, pstride, b.pum, b.S, b.pobj, b.maxIllum, b.delta_p, b.starts,
                                  members, gsize, b.N, b.Y, b.sums, b.lsq_done, b.errk, b.beta_obj, b.beta_probe, b.betas,
                                  b.err);
  return cudaGetLastError();
}

// Object update over the group box, probe update (the 2x2 solves ran at the end of mls_lsq).
cudaError_t mls_solve_update(const MlsBuffers& b, const int* members, const int* gsize, const int* bbox,
                             int clear_pum, cudaStream_t st) {
  (void)members;
  const int NN = b.N * b.N;
  launch_pdl(k_mls_update_object, grid_for(size_t(2) * NN), 256, 0, st, b.obj, b.S, b.pobj, b.maxIllum, b.delta_p, b.betas,
                                                                 bbox, b.Y);
  launch_pdl(k_mls_update_probe, grid_for(NN), 256, 0, st, b.probe, b.pum, b.betas, gsize, NN, clear_pum);
  return cudaGetLastError();
}

}  // namespace pty
