// Warm start of the object from the network's per-position predictions: the network input built from the measured
// amplitudes, the stitching of the predicted patches into probe-weighted object sums, the least-squares
// integration of the stitched phase differences (an FFT Poisson solve), and the energy match of the assembled
// object to the data.  No counterpart in the reference, which starts from a constant object
// (src/Sample.cpp:216-220) or a user-supplied one (objectNP); the C ABI is in include/ptychopy_b200.h.
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>

#include "../../include/ptychopy_b200.h"
#include "kernel_util.cuh"
#include "kernels.h"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

namespace {

// x[b][i][j] = scale * log1p(amp[b][(i + N/2) % N][(j + N/2) % N]): the zero frequency moved to the centre
__global__ void k_warm_input(const float* __restrict__ amp, float* __restrict__ x, size_t B, int N, float scale) {
  const size_t NN = size_t(N) * N, n = B * NN;
  const int h = N / 2;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t b = q / NN;
    const int p = int(q % NN), i = p / N, j = p % N;
    const int si = i + h >= N ? i + h - N : i + h, sj = j + h >= N ? j + h - N : j + h;
    x[q] = scale * log1pf(amp[b * NN + size_t(si) * N + sj]);
  }
}

constexpr int ST = 16;  // object tile side of one stitching CTA

// acc (4 planes of X x Y): sum_p w(x - r_p) A_p, sum_p w gx_p, sum_p w gy_p, sum_p w, over the positions p whose
// S x S output patch covers the pixel; r_p = round(pos_p) + off.  A CTA owns a 16 x 16 tile and visits the positions
// in order, so the sums are deterministic: per chunk of 256 positions each thread tests one against the tile, an
// order-preserving compaction (warp ballots and a scan over the warps) lists the ones whose patch meets the tile, and
// only those are visited.  Network outputs are in scaled units: A = amp_mean + o0 * amp_scale, g = o * grad_scale.
__global__ void __launch_bounds__(ST* ST) k_warm_stitch(const float* __restrict__ out, const float* __restrict__ pos,
                                                       int P, const float* __restrict__ wgt, int S, int off,
                                                       float amp_mean, float amp_scale, float grad_scale,
                                                       float* __restrict__ acc, int X, int Y) {
  constexpr int NW = ST * ST / 32;
  __shared__ int s_r[ST * ST], s_c[ST * ST], s_p[ST * ST];
  __shared__ int s_wcount[NW];
  const int tilesY = (Y + ST - 1) / ST;
  const int ti = blockIdx.x / tilesY, tj = blockIdx.x % tilesY;
  const int i = ti * ST + threadIdx.x / ST, j = tj * ST + threadIdx.x % ST;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t SS = size_t(S) * S;
  float a = 0.f, gx = 0.f, gy = 0.f, ws = 0.f;
  for (int p0 = 0; p0 < P; p0 += ST * ST) {
    const int p = p0 + threadIdx.x;
    int r0 = 0, c0 = 0;
    bool hit = false;
    if (p < P) {
      r0 = int(rintf(pos[2 * size_t(p)])) + off;
      c0 = int(rintf(pos[2 * size_t(p) + 1])) + off;
      hit = !(r0 >= ti * ST + ST || r0 + S <= ti * ST || c0 >= tj * ST + ST || c0 + S <= tj * ST);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_wcount[warp] = __popc(bal);
    __syncthreads();
    int base = 0, cnt = 0;
    for (int w = 0; w < NW; ++w) {
      base += w < warp ? s_wcount[w] : 0;
      cnt += s_wcount[w];
    }
    if (hit) {
      const int k = base + __popc(bal & ((1u << lane) - 1u));
      s_r[k] = r0;
      s_c[k] = c0;
      s_p[k] = p;
    }
    __syncthreads();
    for (int q = 0; q < cnt; ++q) {
      const int rq = s_r[q], cq = s_c[q];
      const int li = i - rq, lj = j - cq;
      if (li >= 0 && li < S && lj >= 0 && lj < S) {
        const float wv = wgt[li * S + lj];
        const float* o = out + size_t(s_p[q]) * 3 * SS + size_t(li) * S + lj;
        a += wv * (amp_mean + o[0] * amp_scale);
        gx += wv * (o[SS] * grad_scale);
        gy += wv * (o[2 * SS] * grad_scale);
        ws += wv;
      }
    }
    __syncthreads();
  }
  if (i < X && j < Y) {
    const size_t XY = size_t(X) * Y, k = size_t(i) * Y + j;
    acc[k] = a;
    acc[XY + k] = gx;
    acc[2 * XY + k] = gy;
    acc[3 * XY + k] = ws;
  }
}

// z (M x M complex) = gx + i gy, the weighted means of the stitched phase differences, zero where the weight is
// below wmin or outside the object
__global__ void k_warm_pack(const float* __restrict__ acc, int X, int Y, int M, float wmin, float2* __restrict__ z) {
  const size_t n = size_t(M) * M, XY = size_t(X) * Y;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int i = int(q / M), j = int(q % M);
    float2 v = make_float2(0.f, 0.f);
    if (i < X && j < Y) {
      const size_t k = size_t(i) * Y + j;
      const float ws = acc[3 * XY + k];
      if (ws > wmin) v = make_float2(acc[XY + k] / ws, acc[2 * XY + k] / ws);
    }
    z[q] = v;
  }
}

// Least-squares phase from forward differences gx(i,j) ~ phi(i+1,j) - phi(i,j), gy(i,j) ~ phi(i,j+1) - phi(i,j) on
// the periodic M x M grid: in Fourier space (forward transform F(k) = sum f(n) e^{-2 pi i k n / M}, so a shift by
// +1 multiplies by D(k) = e^{2 pi i k / M} - 1), phi^ = (conj(Dx) Gx^ + conj(Dy) Gy^) / (|Dx|^2 + |Dy|^2), phi^(0) = 0.
// Z = F(gx + i gy) carries both real transforms: Gx^(k) = (Z(k) + conj Z(-k)) / 2, Gy^(k) = (Z(k) - conj Z(-k)) / 2i.
__global__ void k_warm_poisson(const float2* __restrict__ Z, int M, float2* __restrict__ out) {
  const size_t n = size_t(M) * M;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int u = int(q / M), v = int(q % M);
    const float2 zk = Z[q];
    const float2 zm = Z[size_t((M - u) % M) * M + (M - v) % M];
    const float2 gx = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 gy = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    float su, cu, sv, cv;
    sincospif(2.f * float(u) / float(M), &su, &cu);
    sincospif(2.f * float(v) / float(M), &sv, &cv);
    const float2 dx = make_float2(cu - 1.f, su), dy = make_float2(cv - 1.f, sv);
    const float den = dx.x * dx.x + dx.y * dx.y + dy.x * dy.x + dy.y * dy.y;
    float2 r = make_float2(0.f, 0.f);
    if (den > 0.f) {
      // conj(d) * g = (d.x g.x + d.y g.y) + i (d.x g.y - d.y g.x)
      r.x = (dx.x * gx.x + dx.y * gx.y + dy.x * gy.x + dy.y * gy.y) / den;
      r.y = (dx.x * gx.y - dx.y * gx.x + dy.x * gy.y - dy.y * gy.x) / den;
    }
    out[q] = r;
  }
}

// obj = A exp(i phi): A the weighted mean amplitude (amp_fill where the weight is below wmin), phi = Re(ifft) / M^2
__global__ void k_warm_compose(const float* __restrict__ acc, const float2* __restrict__ phi, int X, int Y, int M,
                               float wmin, float amp_fill, float2* __restrict__ obj) {
  const size_t XY = size_t(X) * Y;
  const float inv = 1.f / (float(M) * float(M));
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < XY; q += size_t(gridDim.x) * blockDim.x) {
    const int i = int(q / Y), j = int(q % Y);
    const float ws = acc[3 * XY + q];
    const float A = ws > wmin ? acc[q] / ws : amp_fill;
    float s, c;
    sincosf(phi[size_t(i) * M + j].x * inv, &s, &c);
    obj[q] = make_float2(A * c, A * s);
  }
}

// sums[0] += sum amp^2 over n values
__global__ void k_warm_data_energy(const float* __restrict__ amp, size_t n, double* __restrict__ sums) {
  double e = 0.0;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const double a = amp[q];
    e += a * a;
  }
  e = block_reduce_sum(e);
  if (threadIdx.x == 0) atomicAdd(&sums[0], e);
}

// sums[1] += sum_p sum_{i,j} |P(i,j)|^2 |O(round(pos_p) + (i,j))|^2 (window clamped to the object); one CTA per
// position, grid-strided
__global__ void k_warm_model_energy(const float2* __restrict__ obj, int X, int Y, const float2* __restrict__ probe,
                                    int N, const float* __restrict__ pos, int P, double* __restrict__ sums) {
  double e = 0.0;
  const size_t NN = size_t(N) * N;
  for (int p = blockIdx.x; p < P; p += gridDim.x) {
    const int r0 = int(rintf(pos[2 * size_t(p)])), c0 = int(rintf(pos[2 * size_t(p) + 1]));
    for (size_t q = threadIdx.x; q < NN; q += blockDim.x) {
      const int i = min(max(r0 + int(q / N), 0), X - 1), j = min(max(c0 + int(q % N), 0), Y - 1);
      const float2 pr = probe[q], o = obj[size_t(i) * Y + j];
      e += double(pr.x * pr.x + pr.y * pr.y) * double(o.x * o.x + o.y * o.y);
    }
  }
  e = block_reduce_sum(e);
  if (threadIdx.x == 0) atomicAdd(&sums[1], e);
}

// obj *= sqrt(sums[0] / (N^2 sums[1])): the unnormalised FFT multiplies the exit wave's energy by N^2
__global__ void k_warm_scale(float2* __restrict__ obj, size_t n, const double* __restrict__ sums, int N) {
  const double m = sums[1] * double(N) * double(N);
  const float k = m > 0.0 ? float(sqrt(sums[0] / m)) : 1.f;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const float2 v = obj[q];
    obj[q] = make_float2(v.x * k, v.y * k);
  }
}

int grid1(size_t n) {
  const size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

int fail(const std::string& msg, int code) {
  set_last_error(msg);
  return code;
}

int finish(cudaError_t e, const char* what) {
  if (e != cudaSuccess) return fail(std::string(what) + ": " + cudaGetErrorString(e), PTY_ERR_CUDA);
  return PTY_OK;
}

}  // namespace

int warm_grid_size(int X, int Y) {
  int M = 32;
  while (M < X || M < Y) M *= 2;
  return M;
}

// The twiddle table of the M x M Poisson-solve transforms, made once per device and size and kept until the process
// exits (at most 5 x 4 KB per device): making and freeing it per call cost a device synchronisation each time.
cudaError_t warm_twiddles(int M, const float2** out, cudaStream_t st) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static float2* table[kMaxDevices][10] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int lg = 0;
  while ((1 << lg) < M) ++lg;
  if (dev < 0 || dev >= kMaxDevices || (1 << lg) != M || lg >= 10) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  if (table[dev][lg]) {  // a table from before a device reset is gone: make it again
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, table[dev][lg]) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      table[dev][lg] = nullptr;
    }
  }
  if (!table[dev][lg]) {
    float2* tw = nullptr;
    e = make_twiddles(M, &tw, st);
    if (e != cudaSuccess) return e;
    table[dev][lg] = tw;
  }
  *out = table[dev][lg];
  return cudaSuccess;
}

}  // namespace pty

using namespace pty;

extern "C" {

int pty_warm_input(const float* amp, float* x, int B, int N, float scale, void* stream) {
  if (!amp || !x || B < 1 || N < 2 || (N & 1)) return fail("pty_warm_input: bad argument", PTY_ERR_INVALID);
  const size_t n = size_t(B) * N * N;
  k_warm_input<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(amp, x, size_t(B), N, scale);
  return finish(cudaGetLastError(), "pty_warm_input");
}

int pty_warm_stitch(const float* out, const float* pos_px, int P, const float* weight, int S, int N, float amp_mean,
                    float amp_scale, float grad_scale, float* acc, int X, int Y, void* stream) {
  if (!out || !pos_px || !weight || !acc || P < 1 || S < 1 || S > N || X < 1 || Y < 1)
    return fail("pty_warm_stitch: bad argument", PTY_ERR_INVALID);
  const int tiles = ((X + ST - 1) / ST) * ((Y + ST - 1) / ST);
  k_warm_stitch<<<tiles, ST * ST, 0, static_cast<cudaStream_t>(stream)>>>(
      out, pos_px, P, weight, S, (N - S) / 2, amp_mean, amp_scale, grad_scale, acc, X, Y);
  return finish(cudaGetLastError(), "pty_warm_stitch");
}

int pty_warm_object(const float* acc, int X, int Y, float wmin, float amp_fill, const float* probe_c64, int N,
                    const float* pos_px, int P, const float* amp, float* work, float* obj_c64, void* stream) {
  if (!acc || !probe_c64 || !pos_px || !amp || !work || !obj_c64 || X < 1 || Y < 1 || P < 1 || N < 1)
    return fail("pty_warm_object: bad argument", PTY_ERR_INVALID);
  const int M = warm_grid_size(X, Y);
  if (!fft_size_supported(M)) return fail("pty_warm_object: object larger than 512 x 512", PTY_ERR_INVALID);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t MM = size_t(M) * M;
  float2* z = reinterpret_cast<float2*>(work);
  float2* spec = z + MM;
  float2* fwork = spec + MM;
  double* sums = reinterpret_cast<double*>(fwork + MM);
  float2* obj = reinterpret_cast<float2*>(obj_c64);
  const float2* tw = nullptr;
  cudaError_t e = warm_twiddles(M, &tw, st);
  if (e != cudaSuccess) return finish(e, "pty_warm_object: twiddles");
  k_warm_pack<<<grid1(MM), 256, 0, st>>>(acc, X, Y, M, wmin, z);
  e = fft2(z, fwork, tw, 1, M, false, st);
  if (e == cudaSuccess) {
    k_warm_poisson<<<grid1(MM), 256, 0, st>>>(z, M, spec);
    e = fft2(spec, fwork, tw, 1, M, true, st);
  }
  if (e == cudaSuccess) {
    const size_t XY = size_t(X) * Y;
    k_warm_compose<<<grid1(XY), 256, 0, st>>>(acc, spec, X, Y, M, wmin, amp_fill, obj);
    e = cudaMemsetAsync(sums, 0, 2 * sizeof(double), st);
    if (e == cudaSuccess) {
      const size_t n = size_t(P) * N * N;
      k_warm_data_energy<<<grid1(n) < 1024 ? grid1(n) : 1024, 256, 0, st>>>(amp, n, sums);
      k_warm_model_energy<<<P < 1024 ? P : 1024, 256, 0, st>>>(obj, X, Y, reinterpret_cast<const float2*>(probe_c64),
                                                               N, pos_px, P, sums);
      k_warm_scale<<<grid1(XY), 256, 0, st>>>(obj, XY, sums, N);
      e = cudaGetLastError();
    }
  }
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = e2;
  return finish(e, "pty_warm_object");
}

}  // extern "C"
