// Kernels of the warm-start network (a small convolutional encoder-decoder mapping a diffraction pattern to the
// object patch under the probe): 3x3 convolutions (stride 1, zero padding 1) forward with an optional fused ReLU,
// backward-data and backward-weight, ReLU, 2x2 average pooling, 2x nearest upsampling, a weighted mean-squared-error
// loss and an Adam step.  Float32, NCHW, batch-major; every entry point takes device pointers and a stream and
// launches asynchronously.  No counterpart in the reference (it has no learned component); the C ABI is in
// include/ptychopy_b200.h.
#include <cuda_runtime.h>

#include <cstddef>
#include <string>

#include "../../include/ptychopy_b200.h"
#include "kernel_util.cuh"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

namespace {

constexpr int CONV_THREADS = 256;
constexpr int CONV_CIB = 8;  // input channels staged in shared memory per round

// y[b][co][i][j] = bias[co] + sum_ci sum_k w'[co][ci][k] x[b][ci][i+ky-1][j+kx-1]  (zero padding), then ReLU if
// `relu`.
// FLIP = false: w' = w[co][ci][ky][kx]                    (forward, weights Cout x Cin x 3 x 3)
// FLIP = true:  w' = w[ci][co][2-ky][2-kx]: backward data through the forward layer whose weights are w (that
//               layer's Cin is Cout here and its Cout is Cin here).
// A CTA computes a TH x TW pixel tile of one image for COB output channels; each thread owns 2 x 2 pixels x 8
// channels (32 accumulators), reading a 4 x 4 input window and two float4 of weights per input channel and tap.
template <int TH, int TW, bool FLIP>
__global__ void __launch_bounds__(CONV_THREADS) k_conv3x3(const float* __restrict__ x, const float* __restrict__ w,
                                                          const float* __restrict__ bias, float* __restrict__ y,
                                                          int Cin, int Cout, int H, int W, int relu) {
  constexpr int PGX = TW / 2, PG = (TH / 2) * PGX, CG = CONV_THREADS / PG, COB = CG * 8;
  constexpr int SH = TH + 2, SW = TW + 2;
  __shared__ float s_in[CONV_CIB][SH][SW];
  __shared__ __align__(16) float s_w[CONV_CIB][9][COB];
  const int tilesX = (W + TW - 1) / TW;
  const int ti = blockIdx.x / tilesX, tj = blockIdx.x % tilesX;
  const int co0 = blockIdx.y * COB, b = blockIdx.z;
  const int pg = threadIdx.x % PG, cg = threadIdx.x / PG;
  const int pr = 2 * (pg / PGX), pc = 2 * (pg % PGX);
  float acc[8][4];
#pragma unroll
  for (int o = 0; o < 8; ++o)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[o][q] = 0.f;
  const size_t HW = size_t(H) * W;
  for (int ci0 = 0; ci0 < Cin; ci0 += CONV_CIB) {
    for (int q = threadIdx.x; q < CONV_CIB * SH * SW; q += CONV_THREADS) {
      const int c = q / (SH * SW), r = (q / SW) % SH, cc = q % SW;
      const int ci = ci0 + c, gi = ti * TH + r - 1, gj = tj * TW + cc - 1;
      float v = 0.f;
      if (ci < Cin && gi >= 0 && gi < H && gj >= 0 && gj < W) v = x[(size_t(b) * Cin + ci) * HW + size_t(gi) * W + gj];
      s_in[c][r][cc] = v;
    }
    for (int q = threadIdx.x; q < CONV_CIB * 9 * COB; q += CONV_THREADS) {
      const int o = q % COB, k = (q / COB) % 9, c = q / (9 * COB);
      const int ci = ci0 + c, co = co0 + o;
      float v = 0.f;
      if (ci < Cin && co < Cout) v = FLIP ? w[(size_t(ci) * Cout + co) * 9 + (8 - k)] : w[(size_t(co) * Cin + ci) * 9 + k];
      s_w[c][k][o] = v;
    }
    __syncthreads();
    const int nc = min(CONV_CIB, Cin - ci0);
#pragma unroll 2
    for (int c = 0; c < nc; ++c) {
      float v[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int e = 0; e < 4; ++e) v[a][e] = s_in[c][pr + a][pc + e];
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const float4 w0 = *reinterpret_cast<const float4*>(&s_w[c][ky * 3 + kx][cg * 8]);
          const float4 w1 = *reinterpret_cast<const float4*>(&s_w[c][ky * 3 + kx][cg * 8 + 4]);
          const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
          for (int o = 0; o < 8; ++o) {
            acc[o][0] += wv[o] * v[ky][kx];
            acc[o][1] += wv[o] * v[ky][kx + 1];
            acc[o][2] += wv[o] * v[ky + 1][kx];
            acc[o][3] += wv[o] * v[ky + 1][kx + 1];
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    const int co = co0 + cg * 8 + o;
    if (co >= Cout) continue;
    const float bv = bias ? bias[co] : 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = ti * TH + pr + (q >> 1), j = tj * TW + pc + (q & 1);
      if (i < H && j < W) {
        float r = acc[o][q] + bv;
        if (relu) r = fmaxf(r, 0.f);
        y[(size_t(b) * Cout + co) * HW + size_t(i) * W + j] = r;
      }
    }
  }
}

// Weight gradient as a GEMM over pixels: dw[co][ci][k] += sum_{b,i,j} dy[b][co][i][j] x[b][ci][i+ky-1][j+kx-1].
// A CTA owns 32 output x 32 input channels (all 9 taps); each thread 4 output channels x 1 input channel x 9 taps.
// It walks the (image, 8 x 8 pixel tile) pairs blockIdx.z, blockIdx.z + gridDim.z, ..., staging dy (pixel-major,
// channel-minor, for float4 reads) and the 10 x 10 input halo, and adds its partial sums to dw atomically (dw zero
// on entry).
constexpr int DW_CO = 32, DW_CI = 32, DW_T = 8;
__global__ void __launch_bounds__(256) k_conv3x3_dw(const float* __restrict__ x, const float* __restrict__ dy,
                                                   float* __restrict__ dw, int B, int Cin, int Cout, int H, int W) {
  __shared__ __align__(16) float s_dy[DW_T * DW_T][DW_CO];
  __shared__ float s_x[DW_CI][DW_T + 2][DW_T + 2 + 1];
  const int co0 = blockIdx.x * DW_CO, ci0 = blockIdx.y * DW_CI;
  const int cg = threadIdx.x % 8, cl = threadIdx.x / 8;
  const int tilesX = (W + DW_T - 1) / DW_T, tilesY = (H + DW_T - 1) / DW_T, tiles = tilesX * tilesY;
  const size_t HW = size_t(H) * W;
  float acc[4][9];
#pragma unroll
  for (int o = 0; o < 4; ++o)
#pragma unroll
    for (int k = 0; k < 9; ++k) acc[o][k] = 0.f;
  for (int u = blockIdx.z; u < B * tiles; u += gridDim.z) {
    const int b = u / tiles, t = u % tiles, ti = t / tilesX, tj = t % tilesX;
    for (int q = threadIdx.x; q < DW_T * DW_T * DW_CO; q += 256) {
      const int o = q % DW_CO, p = q / DW_CO, i = ti * DW_T + p / DW_T, j = tj * DW_T + p % DW_T, co = co0 + o;
      s_dy[p][o] = (co < Cout && i < H && j < W) ? dy[(size_t(b) * Cout + co) * HW + size_t(i) * W + j] : 0.f;
    }
    for (int q = threadIdx.x; q < DW_CI * (DW_T + 2) * (DW_T + 2); q += 256) {
      const int c = q / ((DW_T + 2) * (DW_T + 2)), r = (q / (DW_T + 2)) % (DW_T + 2), cc = q % (DW_T + 2);
      const int ci = ci0 + c, gi = ti * DW_T + r - 1, gj = tj * DW_T + cc - 1;
      s_x[c][r][cc] = (ci < Cin && gi >= 0 && gi < H && gj >= 0 && gj < W)
                          ? x[(size_t(b) * Cin + ci) * HW + size_t(gi) * W + gj]
                          : 0.f;
    }
    __syncthreads();
#pragma unroll 4
    for (int p = 0; p < DW_T * DW_T; ++p) {
      const int pi = p / DW_T, pj = p % DW_T;
      const float4 g = *reinterpret_cast<const float4*>(&s_dy[p][cg * 4]);
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const float xv = s_x[cl][pi + ky][pj + kx];
          acc[0][ky * 3 + kx] += g.x * xv;
          acc[1][ky * 3 + kx] += g.y * xv;
          acc[2][ky * 3 + kx] += g.z * xv;
          acc[3][ky * 3 + kx] += g.w * xv;
        }
    }
    __syncthreads();
  }
  const int ci = ci0 + cl;
  if (ci >= Cin) return;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const int co = co0 + cg * 4 + o;
    if (co < Cout)
#pragma unroll
      for (int k = 0; k < 9; ++k) atomicAdd(&dw[(size_t(co) * Cin + ci) * 9 + k], acc[o][k]);
  }
}

// db[co] += sum over images and pixels of dy[b][co] (db zero on entry).  Grid (Cout, chunks).
__global__ void k_bias_grad(const float* __restrict__ dy, float* __restrict__ db, int B, int Cout, size_t HW) {
  const int co = blockIdx.x;
  const size_t total = size_t(B) * HW;
  double acc = 0.0;
  for (size_t q = blockIdx.y * size_t(blockDim.x) + threadIdx.x; q < total; q += size_t(gridDim.y) * blockDim.x) {
    const size_t b = q / HW, p = q % HW;
    acc += dy[(b * Cout + co) * HW + p];
  }
  acc = block_reduce_sum(acc);
  if (threadIdx.x == 0) atomicAdd(&db[co], float(acc));
}

__global__ void k_relu(float* __restrict__ a, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    a[i] = fmaxf(a[i], 0.f);
}
// g *= (y > 0), y the ReLU output
__global__ void k_relu_bwd(const float* __restrict__ y, float* __restrict__ g, size_t n) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    if (!(y[i] > 0.f)) g[i] = 0.f;
}
// y[bc][i][j] = mean of x[bc][2i..2i+1][2j..2j+1]; planes = B*C, H x W the output size
__global__ void k_pool2(const float* __restrict__ x, float* __restrict__ y, size_t planes, int H, int W) {
  const size_t n = planes * H * W;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t pl = q / (size_t(H) * W);
    const int p = int(q % (size_t(H) * W)), i = p / W, j = p % W;
    const float* xp = x + pl * 4 * H * W;
    const int W2 = 2 * W;
    y[q] = 0.25f * (xp[(2 * i) * W2 + 2 * j] + xp[(2 * i) * W2 + 2 * j + 1] + xp[(2 * i + 1) * W2 + 2 * j] +
                    xp[(2 * i + 1) * W2 + 2 * j + 1]);
  }
}
// gradient of k_pool2: dx (2H x 2W) = dy / 4 broadcast
__global__ void k_pool2_bwd(const float* __restrict__ dy, float* __restrict__ dx, size_t planes, int H, int W) {
  const size_t n = planes * 4 * H * W;
  const int W2 = 2 * W;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t pl = q / (4 * size_t(H) * W);
    const int p = int(q % (4 * size_t(H) * W)), i = p / W2, j = p % W2;
    dx[q] = 0.25f * dy[pl * H * W + size_t(i / 2) * W + j / 2];
  }
}
// y (2H x 2W) = nearest upsampling of x (H x W)
__global__ void k_up2(const float* __restrict__ x, float* __restrict__ y, size_t planes, int H, int W) {
  const size_t n = planes * 4 * H * W;
  const int W2 = 2 * W;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t pl = q / (4 * size_t(H) * W);
    const int p = int(q % (4 * size_t(H) * W)), i = p / W2, j = p % W2;
    y[q] = x[pl * H * W + size_t(i / 2) * W + j / 2];
  }
}
// gradient of k_up2: dx (H x W) = sum of the 2x2 block of dy
__global__ void k_up2_bwd(const float* __restrict__ dy, float* __restrict__ dx, size_t planes, int H, int W) {
  const size_t n = planes * H * W;
  const int W2 = 2 * W;
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t pl = q / (size_t(H) * W);
    const int p = int(q % (size_t(H) * W)), i = p / W, j = p % W;
    const float* d = dy + pl * 4 * H * W;
    dx[q] = d[(2 * i) * W2 + 2 * j] + d[(2 * i) * W2 + 2 * j + 1] + d[(2 * i + 1) * W2 + 2 * j] +
            d[(2 * i + 1) * W2 + 2 * j + 1];
  }
}
// Weighted MSE over n values, weight wp[i % plane] (1 when wp is null):
// loss[0] += sum w (p - t)^2 / n (loss zero on entry), g = 2 w (p - t) / n.
__global__ void k_mse(const float* __restrict__ p, const float* __restrict__ t, const float* __restrict__ wp,
                      size_t plane, float* __restrict__ g, size_t n, double* __restrict__ loss) {
  double acc = 0.0;
  const float inv = 1.f / float(n);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float d = p[i] - t[i], wv = wp ? wp[i % plane] : 1.f;
    g[i] = 2.f * wv * d * inv;
    acc += double(wv) * d * d;
  }
  acc = block_reduce_sum(acc);
  if (threadIdx.x == 0) atomicAdd(loss, acc / double(n));
}
// Adam (Kingma & Ba, 2015): m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2; p -= lr mhat / (sqrt(vhat) + eps)
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       size_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

int grid1(size_t n) {
  const size_t g = (n + 255) / 256;
  return int(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

int finish(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return PTY_ERR_CUDA;
  }
  return PTY_OK;
}

int bad(const char* what) {
  set_last_error(std::string(what) + ": bad argument (null pointer or empty size)");
  return PTY_ERR_INVALID;
}

template <int T, bool FLIP>
void launch_conv(const float* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H, int W,
                 int relu, cudaStream_t st) {
  constexpr int COB = (CONV_THREADS / ((T / 2) * (T / 2))) * 8;
  const dim3 grid(((H + T - 1) / T) * ((W + T - 1) / T), (Cout + COB - 1) / COB, B);
  k_conv3x3<T, T, FLIP><<<grid, CONV_THREADS, 0, st>>>(x, w, bias, y, Cin, Cout, H, W, relu);
}

// Tile choice: 8 x 8 pixels x 128 channels for images up to 8 x 8; 16 x 16 x 32 when Cout fills whole groups of 32;
// otherwise 32 x 32 x 8 on images of at least 32 x 32 (thin layers: the 1-channel input layer's 16 outputs, the
// 3-plane output layer), else 16 x 16 x 32.
template <bool FLIP>
void conv(const float* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H, int W,
          int relu, cudaStream_t st) {
  if (H <= 8 && W <= 8)
    launch_conv<8, FLIP>(x, w, bias, y, B, Cin, Cout, H, W, relu, st);
  else if (Cout % 32 != 0 && H >= 32 && W >= 32)
    launch_conv<32, FLIP>(x, w, bias, y, B, Cin, Cout, H, W, relu, st);
  else
    launch_conv<16, FLIP>(x, w, bias, y, B, Cin, Cout, H, W, relu, st);
}

}  // namespace
}  // namespace pty

using namespace pty;

extern "C" {

int pty_nn_conv3x3(const float* x, const float* w, const float* bias, float* y, int B, int Cin, int Cout, int H, int W,
                   int relu, void* stream) {
  if (!x || !w || !y || B < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1 || B > 65535) return bad("pty_nn_conv3x3");
  conv<false>(x, w, bias, y, B, Cin, Cout, H, W, relu, static_cast<cudaStream_t>(stream));
  return finish(cudaGetLastError(), "pty_nn_conv3x3");
}

int pty_nn_conv3x3_bwd(const float* x, const float* w, const float* dy, float* dx, float* dw, float* db, int B,
                       int Cin, int Cout, int H, int W, void* stream) {
  if (!x || !w || !dy || !dw || B < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1 || B > 65535)
    return bad("pty_nn_conv3x3_bwd");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(dw, 0, sizeof(float) * size_t(Cout) * Cin * 9, st);
  if (e == cudaSuccess && db) e = cudaMemsetAsync(db, 0, sizeof(float) * size_t(Cout), st);
  if (e != cudaSuccess) return finish(e, "pty_nn_conv3x3_bwd");
  if (dx) conv<true>(dy, w, nullptr, dx, B, Cout, Cin, H, W, 0, st);
  const int tiles = ((H + DW_T - 1) / DW_T) * ((W + DW_T - 1) / DW_T);
  const int gx = (Cout + DW_CO - 1) / DW_CO, gy = (Cin + DW_CI - 1) / DW_CI;
  // enough CTAs for about four waves over 148 SMs, each walking several (image, tile) pairs
  int gz = (4 * 148 + gx * gy - 1) / (gx * gy);
  if (gz > B * tiles) gz = B * tiles;
  if (gz > 65535) gz = 65535;
  k_conv3x3_dw<<<dim3(gx, gy, gz), 256, 0, st>>>(x, dy, dw, B, Cin, Cout, H, W);
  if (db) {
    const size_t HW = size_t(H) * W;
    int chunks = int((size_t(B) * HW + 256 * 8 - 1) / (256 * 8));
    if (chunks > 64) chunks = 64;
    k_bias_grad<<<dim3(Cout, chunks), 256, 0, st>>>(dy, db, B, Cout, HW);
  }
  return finish(cudaGetLastError(), "pty_nn_conv3x3_bwd");
}

int pty_nn_relu(float* a, size_t n, void* stream) {
  if (!a || n == 0) return bad("pty_nn_relu");
  k_relu<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(a, n);
  return finish(cudaGetLastError(), "pty_nn_relu");
}
int pty_nn_relu_bwd(const float* y, float* g, size_t n, void* stream) {
  if (!y || !g || n == 0) return bad("pty_nn_relu_bwd");
  k_relu_bwd<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(y, g, n);
  return finish(cudaGetLastError(), "pty_nn_relu_bwd");
}
int pty_nn_pool2(const float* x, float* y, size_t planes, int H, int W, void* stream) {
  if (!x || !y || planes == 0 || H < 1 || W < 1) return bad("pty_nn_pool2");
  k_pool2<<<grid1(planes * H * W), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, y, planes, H, W);
  return finish(cudaGetLastError(), "pty_nn_pool2");
}
int pty_nn_pool2_bwd(const float* dy, float* dx, size_t planes, int H, int W, void* stream) {
  if (!dy || !dx || planes == 0 || H < 1 || W < 1) return bad("pty_nn_pool2_bwd");
  k_pool2_bwd<<<grid1(planes * 4 * H * W), 256, 0, static_cast<cudaStream_t>(stream)>>>(dy, dx, planes, H, W);
  return finish(cudaGetLastError(), "pty_nn_pool2_bwd");
}
int pty_nn_up2(const float* x, float* y, size_t planes, int H, int W, void* stream) {
  if (!x || !y || planes == 0 || H < 1 || W < 1) return bad("pty_nn_up2");
  k_up2<<<grid1(planes * 4 * H * W), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, y, planes, H, W);
  return finish(cudaGetLastError(), "pty_nn_up2");
}
int pty_nn_up2_bwd(const float* dy, float* dx, size_t planes, int H, int W, void* stream) {
  if (!dy || !dx || planes == 0 || H < 1 || W < 1) return bad("pty_nn_up2_bwd");
  k_up2_bwd<<<grid1(planes * H * W), 256, 0, static_cast<cudaStream_t>(stream)>>>(dy, dx, planes, H, W);
  return finish(cudaGetLastError(), "pty_nn_up2_bwd");
}
int pty_nn_mse(const float* p, const float* t, const float* w, size_t plane, float* g, size_t n, double* loss,
               void* stream) {
  if (!p || !t || !g || !loss || n == 0 || (w && plane == 0)) return bad("pty_nn_mse");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(double), st);
  if (e != cudaSuccess) return finish(e, "pty_nn_mse");
  const int g1 = grid1(n);
  k_mse<<<g1 < 1024 ? g1 : 1024, 256, 0, st>>>(p, t, w, plane, g, n, loss);
  return finish(cudaGetLastError(), "pty_nn_mse");
}
int pty_nn_adam(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2, float eps,
                int step, void* stream) {
  if (!p || !g || !m || !v || n == 0 || step < 1) return bad("pty_nn_adam");
  const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  k_adam<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return finish(cudaGetLastError(), "pty_nn_adam");
}

}  // extern "C"
