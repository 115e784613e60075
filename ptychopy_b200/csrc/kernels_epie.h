// Persistent ePIE kernel interface (kernels_epie.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace pty {

// Device-resident scalars carried between positions and iterations.
struct EpieScalars {
  float objMax;    // Sample::m_maxObjectIntensity (max of the |O|^2 cache)
  float probeMax;  // Probe::m_maxIntensity
  double err;      // iteration error accumulator
};

struct EpieArgs {
  const float* ampT;      // P x N x N amplitudes, each plane transposed ([ky][kx]) (k_epie)
  const float* amp;       // P x N x N amplitudes, natural layout (k_epie_sm)
  float2* obj;            // X x Y
  float* ocache;          // X x Y |O|^2 cache
  float2* probe;          // K x N x N
  float* pcache;          // K x N x N |P_k|^2 cache
  const float2* pos;      // P fractional positions (pixels)
  const int* order;       // P visiting order of this iteration
  float2* W1;             // Ka x N x N
  float2* W2;             // Ka x N x N
  float* TM;              // TX x TY tile maxima of ocache (16 x 16 tiles)
  float* pm;              // C partial probe maxima
  EpieScalars* sc;
  const float2* tw;
  const double* sqsum;    // per-pattern amplitude sums (error normaliser)
  float saturation;       // pixels with A >= saturation float (no modulus)
  unsigned* gbar;         // 2: grid-barrier count and generation (whole-GPU variant)
  int* gerr;              // grid-barrier timeout flag (whole-GPU variant)
  int N, K, Ka, P, X, Y, TX, TY, C;
  int pc, up, rms, useAll;
  int grid;               // 1: whole-GPU variant (C CTAs, cooperative launch); 0: one cluster of C CTAs
};

// ePIE as a chain of whole-GPU kernels per position (kernels_epie_chain.cu): the precision = 1 path, whose 2-D
// transforms run as split-BF16 tensor-core stages (tc = 1, N = 256).  Same update as k_epie.
struct EpieChainArgs {
  const float* amp;       // P x N x N amplitudes in their natural layout (A(x, y) at [x N + y])
  float2* obj;
  float* ocache;
  float2* probe;
  float* pcache;
  const float2* pos;
  const int* order;
  float2* psi;            // Ka x N x N exit waves, spectra, updates
  float2* work;           // Ka x N x N FFT work
  float* TM;
  EpieScalars* sc;
  const double* sqsum;
  float* pmax2;           // 2: probe maximum after each position (position parity)
  int* tcerr;             // tensor-core wait-timeout flag
  const float2* tw;       // twiddles of the FP32 transforms (tc = 0)
  float saturation;
  int N, K, Ka, P, X, Y, TX, TY, pc, up, rms, useAll, tc;
  int frows;              // rows per CTA of the FP32 transform passes (0: automatic; 2, 4, 8: capped by the default)
};
cudaError_t epie_chain_iteration(const EpieChainArgs& g, cudaStream_t st);
int epie_chain_launches(const EpieChainArgs& g);

// Sets kernel attributes and picks the cluster size (largest resident of 16, 8, ...); returns it in C_out.
cudaError_t epie_prepare(int N, int* C_out);
// Whole-GPU variant (N = 512, and N = 256 when any_size): the CTA count if a cooperative launch of it fits on this
// device, else 0.
int epie_grid_prepare(int N, bool any_size = false);
cudaError_t epie_launch(const EpieArgs& g, cudaStream_t st);
// Shared-memory-resident variant for small windows with one probe mode (N = 32, 64, 128; K = 1): cluster of
// N/32 CTAs, probe and window in (distributed) shared memory, natural-layout amplitudes.
bool epie_uses_smem(int N, int K);
cudaError_t epie_sm_prepare(int N);
cudaError_t epie_sm_launch(const EpieArgs& g, cudaStream_t st);
// Modes 1..K-1 = 0.05 * mode 0, then Gram-Schmidt against the original copies.
cudaError_t epie_init_modes(float2* probe, float* pcache, int K, int N, float2* copy, double* scratch3,
                            cudaStream_t st);
// Self-test of the bounded grid barrier: `ctas` CTAs, `rounds` barriers expecting `expected` arrivals, at most
// `limit` polls per wait; *err = 1 if a wait ran out.
cudaError_t selftest_grid_barrier(int ctas, unsigned expected, unsigned limit, int rounds, unsigned* bar, int* err,
                                  cudaStream_t st);
// Tile maxima of the whole |O|^2 cache.
cudaError_t tile_max_all(const float* ocache, int X, int Y, float* TM, int TX, int TY, cudaStream_t st);

}  // namespace pty
