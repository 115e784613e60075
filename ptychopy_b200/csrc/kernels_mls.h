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
  unsigned* lsq_done;     // blocks of the LSQ launch that have finished (the last one solves and resets it)
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
  // the reference-default path (kernels_mls_var.cu): variable probe and intensity, sub-pixel probe shift,
  // position search
  float2* E;              // N x N extra probe mode
  double* evo;            // 2 x P probe evolution: intensity weights (evo0) | extra-mode weights (evo1)
  float* pos;             // 2 x P current positions (x = rows)
  const float* pos_o;     // 2 x P original positions
  float2* sub;            // P sub-pixel shifts (x = column remainder, y = row remainder)
  int2* win;              // P window starts, rewritten from pos (same array as `starts`)
  int* boxw;              // ngroups x 4 group boxes, written on the device (same array as `bbox`)
  float2* vp;             // Gmax x N x N probes of the group's positions
  float2* pu;             // Gmax x N x N probe directions, shifted back
  float2* aux;            // 2 Gmax x N x N gradient images of the position search; N x N extra-mode update
  double* vs;             // scratch sums (mls_var_scratch_doubles(Gmax))
  float* pmax;            // max of p_object in this iteration
  float cvx, cvy;         // ceil(X/2 - N/2), ceil(Y/2 - N/2)
  float2* vupd;           // N x N extra-mode update
  float2* work2;          // 2 Gmax x N x N FFT work of the position search
  cudaStream_t side;      // the position search runs on this stream beside the rest of its group
  cudaEvent_t ev_fork, ev_join;
  int K;                  // probe modes (probe holds K x N x N)
  float2* psik;           // (K-1) x Gmax x N x N exit waves of modes 1..K-1
  float2* mtmp;           // K x N x N scratch of the mode orthogonalisation
};

// Parts of one iteration of the reference-default path that depend on the iteration number.
enum MlsVarFlags : unsigned {
  MLS_WINDOWS = 1u,     // windows and sub-pixel shifts from the positions (iteration 1 and from PPS)
  MLS_REMOVE = 2u,      // remove_extra_degree (from iteration 2)
  MLS_VARUPD = 4u,      // update_variable_probe (from iteration 3)
  MLS_POSSEARCH = 8u,   // gradient_position_solver (from PPS)
  MLS_SEPARATE = 16u,   // separate transform passes even where one cluster launch per window would serve (the
                        // step shares the GPU with other scans, whose kernels hold SMs the clusters wait for)
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
// fft2 with both passes launched by programmatic dependent launch (kernels_mls_var.cu)
cudaError_t fft2_pdl(float2* data, float2* work, const float2* tw, int batch, int N, bool inverse, cudaStream_t st);
cudaError_t mls_iteration(const MlsBuffers& b, int ngroups, cudaStream_t st);
int mls_launches_per_iteration(int ngroups);
// One iteration of the reference-default path (kernels_mls_var.cu); flags from MlsVarFlags.
cudaError_t mls_iteration_var(const MlsBuffers& b, int ngroups, unsigned flags, cudaStream_t st);
int mls_var_launches_per_iteration(int ngroups, unsigned flags, int K, bool tc, int N);
size_t mls_var_scratch_doubles(int Gmax);
// One mode in FP32 up to 256^2: the group's six 2-D transforms run as one cluster launch; mls_var_prepare sets that
// launch up for N x N windows (outside graph capture).
bool mls_var_fused(int N, int K, bool tc);
cudaError_t mls_var_prepare(int N);
// MLs probe modes 1..K-1 from mode 0 (initMLH): phase tilts (2 (K-1) values, device), then the Gram matrix
// G_ij = sum conj(m_i) m_j (K x K double2, device) for the host's eigen-decomposition, then modes <- modes V
// (V: K x K double2 on the device, column i = combination i); tmp holds K x N x N.
cudaError_t mls_mode_tilts(float2* probe, int K, int N, const double* tilts, cudaStream_t st);
cudaError_t mls_mode_gram(const float2* probe, int K, int N, double2* gram, cudaStream_t st);
cudaError_t mls_mode_combine(float2* probe, float2* tmp, int K, int N, const double2* V, cudaStream_t st);
// MLs probe start without a given probe: the zone-plate guess of initMLH (N x N into probe; pf and work N x N each).
cudaError_t mls_zone_plate_probe(float2* probe, float2* pf, float2* work, const float2* tw, int N, double lambda,
                                 double dx_recon, double beamSize, cudaStream_t st);
// Kernels the two paths share (kernels_mls.cu).
cudaError_t mls_group_boxes(const int2* starts, const int* members, const int* gsize, int ngroups, int Gmax, int N,
                            int* bbox, cudaStream_t st);
cudaError_t mls_modulus(const MlsBuffers& b, const int* members, const int* gsize, cudaStream_t st);
cudaError_t mls_lsq(const MlsBuffers& b, const float2* probe, size_t pstride, const int* members, const int* gsize,
                    cudaStream_t st);
cudaError_t mls_solve_update(const MlsBuffers& b, const int* members, const int* gsize, const int* bbox,
                             int clear_pum, cudaStream_t st);

}  // namespace pty
