// MLs core kernels (kernels_mls.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "kernels.h"

namespace pty {

struct MlsBuffers {
  float2* obj;            // X x Y
  float2* probe;          // N x N (one mode)
  const float* amp;       // P x N x N, sqrt of the intensities (natural layout)
  float* pobj;            // X x Y illumination weights (p_object)
  float2* S;              // X x Y object-direction accumulator (zero between groups)
  float2* pum;            // N x N probe-direction accumulator (zero between groups)
  float2* objp;           // Gmax x N x N object windows
  float2* psi;            // Gmax x N x N exit waves / chi
  float2* work;           // Gmax x N x N FFT work
  const int2* starts;     // P window starts
  const int* members;     // ngroups x Gmax (position indices, -1 padded)
  const int* gsize;       // ngroups
  const int* bbox;        // ngroups x 4 (x0, y0, nx, ny)
  double* sums;           // Gmax x 6 LSQ sums
  double* errk;           // Gmax Fourier-error sums
  double* betas;          // 4: group-mean object step (re, im), probe step (re, im)
  double* err;            // iteration error accumulator
  double* normsums;       // 2
  const float* maxIllum;  // Probe::MAX_ILLUM (set-up value)
  const float2* tw;
  int roi[4];             // calc_object_norm ROI: x0, y0, nx, ny
  int N, P, X, Y, Gmax;
  float delta_p;
  double beta_obj, beta_probe;  // beta_object * beta_LSQ, beta_probe * beta_LSQ
  int tc;                 // 1: the group FFTs run as split-BF16 tensor-core stages (fft2_tc)
  int* tc_err;            // their wait-timeout flag
};

cudaError_t mls_illum_add(float* pobj, const float2* probe, const int2* starts, int P, int N, int Y, float scale,
                          cudaStream_t st);
cudaError_t scale_real(float* a, size_t n, float s, cudaStream_t st);
cudaError_t mls_norm_sums(const float* w, const float2* obj, int Y, int x0, int y0, int nx, int ny, int squared,
                          double* out, cudaStream_t st);
// a *= sqrt(sums[1]/sums[0]) (divide = 0) or a /= it (divide = 1)
cudaError_t scale_by_norm(float2* a, size_t n, const double* sums, int divide, cudaStream_t st);
cudaError_t sqrt_inplace(float* a, size_t n, cudaStream_t st);
cudaError_t max_real(const float* a, size_t n, float* out, cudaStream_t st);
// One MLs iteration over `ngroups` groups (tables in b.members / b.gsize / b.bbox), enqueued on st.
cudaError_t mls_iteration(const MlsBuffers& b, int ngroups, cudaStream_t st);
int mls_launches_per_iteration(int ngroups);

}  // namespace pty
