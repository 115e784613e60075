// Host-side launch wrappers for the engine's CUDA kernels.  All take the stream to launch on and return the
// cudaError_t of the launch.  Complex data is float2 (interleaved complex64).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace pty {

// True when N is a transform size this build has kernels for.
bool fft_size_supported(int N);

// Stage-1 twiddle table for length-N transforms (N float2), filled on the host in double precision.
cudaError_t make_twiddles(int N, float2** d_tw, cudaStream_t st);

// Batched 2-D FFT in natural layout: data (batch x N x N) -> work (transposed) -> data.  Unnormalised.
cudaError_t fft2(float2* data, float2* work, const float2* tw, int batch, int N, bool inverse, cudaStream_t st);
// Split-BF16 tensor-core 2-D FFT (N = 256, kernels_fft_tc.cu): prepare once per device outside stream capture;
// *err receives a non-zero code if a tensor-core wait timed out.
cudaError_t fft2_tc_prepare();
cudaError_t fft2_tc(float2* data, float2* work, int batch, int N, bool inverse, int* err, cudaStream_t st);

// Transposes each N x N float plane: out[b][y][x] = in[b][x][y].
cudaError_t transpose_planes(const float* in, float* out, int batch, int N, cudaStream_t st);

// ---- probe guess (src/Probe.cpp:360-372) -------------------------------------------------------------
// mean amplitude over P patterns (avg N*N), the sinc*Gaussian start in mode 0, FFT-domain projection onto avg,
// normalisation to max|P| = 1 over all K modes, and the intensity cache |P|^2.
cudaError_t mean_amplitude(const float* amp, int P, int N, float* avg, cudaStream_t st);
cudaError_t probe_start(float2* probe0, int N, float window, float factor, cudaStream_t st);
cudaError_t modulus_project(float2* spec, const float* avg, int n, float scale, cudaStream_t st);
// Reductions over complex arrays into device doubles: out[0] = max |a|, or sum |a|^2.
cudaError_t reduce_abs_max(const float2* a, size_t n, double* out, cudaStream_t st);
cudaError_t reduce_sum_sq(const float2* a, size_t n, double* out, cudaStream_t st);
cudaError_t scale_by_inverse(float2* a, size_t n, const double* denom, cudaStream_t st);
cudaError_t abs2(const float2* a, float* out, size_t n, cudaStream_t st);
// Forward model: amp[i] = |FFT2(bilinear O at pos[i] * probe)| for `count` positions (psi, work: count*N*N).
cudaError_t simulate_patterns(const float2* obj, int X, int Y, const float2* probe, int N, const float2* pos,
                              int count, float2* psi, float2* work, const float2* tw, float* amp, cudaStream_t st);
cudaError_t scale_complex(float2* a, size_t n, float s, cudaStream_t st);
cudaError_t fill_complex(float2* a, size_t n, float2 v, cudaStream_t st);
// out[p] = sum of plane p (P planes of NN floats), in double: Diffractions::fillSquaredSums.
cudaError_t plane_sums(const float* a, int P, size_t NN, double* out, cudaStream_t st);
// Probe::getModalDoubleMax over an intensity cache (K x NN): modal sum when useAll && K>1, else stacked max.
cudaError_t probe_modal_max(const float* cache, int K, size_t NN, int useAll, float* out, cudaStream_t st);

// ---- reference DM (src/DM.cu:80-128) -------------------------------------------------------------------
struct DMWave {
  const int* slot_pat;  // pattern index of each slot of this wave (device)
  int count;            // patterns in this wave
};
struct DMBuffers {
  float2* psi;          // P x N x N exit waves
  const float* amp;     // P x N x N amplitudes, natural layout ([kx][ky])
  float2* obj;          // X x Y
  float2* probe;        // K x N x N (mode 0 used)
  float2* dO;           // X x Y increment accumulator
  float2* dP;           // N x N increment accumulator
  float2* W1;           // wave x N x N
  float2* W2;           // wave x N x N
  const int2* offs;     // rounded offsets per pattern
  const float2* tw;     // twiddles for N
  double* sums;         // [0] sum|O|^2, [1] sum|P|^2 (accumulated by finalize)
  double* fac;          // [0] 1/objMax, [1] 1/probeMax (hysteresis-cached), [2] objMax, [3] probeMax
  int* err = nullptr;   // wait-timeout flag of the tensor-core column pass
  int N, K, X, Y;
  int tc = 0;           // column pass on the tensor cores (N = 512)
};
// Sets the shared-memory attributes of the DM kernels for size N (call once, outside graph capture).
cudaError_t dm_prepare(int N);
// The DM column pass at N = 512 with its 32-point DFT stages as FP16-split tcgen05 GEMMs (b.tc, b.err set).
cudaError_t dm_cols_tc_prepare();
cudaError_t dm_cols_tc(const DMBuffers& b, const DMWave& w, cudaStream_t st);
// Patterns per pipeline wave for size N (balanced waves, at least eight for large scans; two lanes of W1 + W2 <= 1 GiB).
int dm_wave_size(int N, int P);
cudaError_t dm_wave(const DMBuffers& b, const DMWave& w, bool phaseConstraint, bool updateProbe, cudaStream_t st,
                    int64_t* launches);
cudaError_t dm_finalize(const DMBuffers& b, bool updateProbe, cudaStream_t st, int64_t* launches);

// psi_p = P * O at every pattern's rounded offset (P patterns).
cudaError_t dm_psi_from_object(const DMBuffers& b, int P, cudaStream_t st);

}  // namespace pty
