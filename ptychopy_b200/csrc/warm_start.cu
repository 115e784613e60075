// Learned warm start inside pty_init: the trained encoder-decoder (parameters handed over with pty_set_warm_start)
// runs on the session's own patterns on the tensor-core inference path, and its per-position predictions are
// assembled into the session's starting object, which then takes the place of the reference's constant start
// (src/Sample.cpp:216-220) or objectNP.  The network layout, the output decoding and the input scale are those of
// ptychopy_b200/warmstart.py (layer_plan, AMP_MEAN, AMP_SCALE, GRAD_SCALE, INPUT_SCALE), which trains it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include "../../include/ptychopy_b200.h"
#include "session.h"

namespace pty {

int warm_grid_size(int X, int Y);  // kernels_warm.cu

namespace {

constexpr float WARM_AMP_MEAN = 0.9f, WARM_AMP_SCALE = 0.1f, WARM_GRAD_SCALE = 0.2f, WARM_INPUT_SCALE = 0.25f;
constexpr float WARM_WMIN = 1e-3f;

struct WarmLayer {
  int cin, cout, H;
  bool relu;
  int after;  // 0 none, 1 2x2 average pooling, 2 2x nearest upsampling
};

// The encoder-decoder for N x N patterns at width w (warmstart.layer_plan)
std::vector<WarmLayer> warm_plan(int N, int w) {
  return {{1, w, N, true, 1},           {w, 2 * w, N / 2, true, 1},          {2 * w, 4 * w, N / 4, true, 1},
          {4 * w, 8 * w, N / 8, true, 1}, {8 * w, 16 * w, N / 16, true, 0},  {16 * w, 16 * w, N / 16, true, 2},
          {16 * w, 4 * w, N / 8, true, 2}, {4 * w, 2 * w, N / 4, true, 0},   {2 * w, 3, N / 4, false, 0}};
}

void call(int rc, const char* what) {
  if (rc != PTY_OK) fail(rc, std::string(what) + ": " + pty_last_error());
}
void need(bool cond, const std::string& msg, int code = PTY_ERR_INVALID) {
  if (!cond) fail(code, msg);
}

}  // namespace

size_t warm_param_count(int N, int w) {
  size_t n = 0;
  for (const WarmLayer& l : warm_plan(N, w)) n += size_t(l.cout) * l.cin * 9 + l.cout;
  return n;
}

// Runs after the probe and the (zero) object exist and before the amplitudes change layout; writes s->obj.
void run_warm_start(pty_session* s) {
  const int N = s->N, w = s->warm_width, S = N / 4, P = s->P;
  const size_t NN = size_t(N) * N;
  cudaStream_t st = s->stream;
  const std::vector<WarmLayer> plan = warm_plan(N, w);
  const int last = int(plan.size()) - 1;
  // parameters and the packed BF16 weights of the tensor-core layers
  DeviceBuf prm;
  prm.alloc(sizeof(float) * s->warm_params.size(), "warm-start parameters");
  check_cuda(cudaMemcpyAsync(prm.p, s->warm_params.data(), prm.bytes, cudaMemcpyHostToDevice, st), "H2D parameters");
  std::vector<const float*> wl(plan.size()), bl(plan.size());
  std::vector<bool> cuda_core(plan.size(), false);
  std::vector<size_t> wpk_off(plan.size(), 0);
  size_t off = 0, ws = 0;
  for (size_t l = 0; l < plan.size(); ++l) {
    const WarmLayer& L = plan[l];
    wl[l] = prm.as<float>() + off;
    bl[l] = wl[l] + size_t(L.cout) * L.cin * 9;
    off += size_t(L.cout) * L.cin * 9 + L.cout;
    // first layer (K = 9) on CUDA cores; the output layer (N = 3) on the tensor cores in the shifted-GEMM form where
    // its size allows (H a multiple of 16), else on CUDA cores
    cuda_core[l] = (l == 0 && L.cout == 16) || (int(l) == last && L.cin == 32 && L.cout <= 4 && L.H % 16 != 0);
    if (!cuda_core[l]) {
      const int n = pty_tc_weights_size(L.cin, L.cout);
      need(n > 0, "warm-start layer " + std::to_string(l) + " is not supported by the tensor-core path");
      wpk_off[l] = ws;
      ws += (2 * size_t(n) + 255) / 256 * 256;
    }
  }
  // one workspace: the packed weights, the activations of one chunk of patterns (NHWC BF16, pooling fused into the
  // producing layer), the network outputs of all patterns and the error flag
  const int chunk = std::min(P, 1024);
  std::vector<size_t> act_off(plan.size(), 0);
  for (int l = 0; l < last; ++l) {
    const int side = plan[l].after == 1 ? plan[l].H / 2 : plan[l].H;
    act_off[l] = ws;
    ws += (2 * size_t(chunk) * side * side * plan[l].cout + 255) / 256 * 256;
  }
  const size_t out_off = ws;
  ws += (sizeof(float) * size_t(P) * 3 * S * S + 255) / 256 * 256;
  const size_t err_off = ws;
  ws += 256;
  DeviceBuf work_all;
  work_all.alloc(ws, "warm-start workspace");
  char* base = work_all.as<char>();
  std::vector<void*> wpk(plan.size(), nullptr);
  for (size_t l = 0; l < plan.size(); ++l)
    if (!cuda_core[l]) {
      wpk[l] = base + wpk_off[l];
      call(pty_tc_pack_weights(wl[l], plan[l].cin, plan[l].cout, wpk[l], st), "pack weights");
    }
  std::vector<void*> act(plan.size(), nullptr);
  for (int l = 0; l < last; ++l) act[l] = base + act_off[l];
  float* out = reinterpret_cast<float*>(base + out_off);
  int* err = reinterpret_cast<int*>(base + err_off);
  check_cuda(cudaMemsetAsync(err, 0, sizeof(int), st), "memset flag");
  for (int c0 = 0; c0 < P; c0 += chunk) {
    const int B = std::min(chunk, P - c0);
    const void* cur = s->amp.as<float>() + size_t(c0) * NN;
    int in_mode = 2;
    for (int l = 0; l <= last; ++l) {
      const WarmLayer& L = plan[l];
      void* y = l == last ? static_cast<void*>(out + size_t(c0) * 3 * S * S) : act[l];
      if (cuda_core[l] && l == 0) {
        call(pty_tc_first_layer(static_cast<const float*>(cur), wl[l], bl[l], y, B, L.cout, L.H, L.H,
                                WARM_INPUT_SCALE, st),
             "first layer");
      } else if (cuda_core[l]) {
        call(pty_tc_last_layer(cur, wl[l], bl[l], static_cast<float*>(y), B, L.cin, L.cout, L.H, L.H, st),
             "output layer");
      } else {
        const int out_mode = l == last ? 1 : (L.after == 1 ? 2 : 0);
        call(pty_tc_conv3x3(cur, wpk[l], bl[l], y, B, L.cin, L.cout, L.H, L.H, L.relu ? 1 : 0, in_mode, out_mode,
                            WARM_INPUT_SCALE, err, st),
             "convolution");
      }
      cur = y;
      in_mode = L.after == 2 ? 1 : 0;
    }
  }
  // stitching weights |P|^2 / max over the central S x S window of probe mode 0
  std::vector<float2> ph(NN);
  check_cuda(cudaMemcpyAsync(ph.data(), s->probe.p, sizeof(float2) * NN, cudaMemcpyDeviceToHost, st), "D2H probe");
  check_cuda(cudaStreamSynchronize(st), "warm-start network");
  int flag = 0;
  check_cuda(cudaMemcpy(&flag, err, sizeof(int), cudaMemcpyDeviceToHost), "D2H flag");
  need(flag == 0, "warm-start network: a tensor-core pipeline wait timed out", PTY_ERR_CUDA);
  const int o = (N - S) / 2;
  std::vector<float> wgt(size_t(S) * S);
  float wmax = 0.f;
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j) {
      const float2 v = ph[size_t(i + o) * N + j + o];
      wgt[size_t(i) * S + j] = v.x * v.x + v.y * v.y;
      wmax = std::max(wmax, wgt[size_t(i) * S + j]);
    }
  need(wmax > 0.f, "warm start: the probe is zero over the central window");
  for (float& v : wgt) v /= wmax;
  DeviceBuf wd, pos, acc, work;
  wd.alloc(sizeof(float) * wgt.size(), "stitching weights");
  pos.alloc(sizeof(float) * 2 * size_t(P), "positions");
  const int M = warm_grid_size(s->X, s->Y);
  acc.alloc(sizeof(float) * 4 * size_t(s->X) * s->Y, "stitching sums");
  work.alloc(sizeof(float) * (6 * size_t(M) * M + 4), "phase integration");
  check_cuda(cudaMemcpyAsync(wd.p, wgt.data(), wd.bytes, cudaMemcpyHostToDevice, st), "H2D weights");
  check_cuda(cudaMemcpyAsync(pos.p, s->geo.pos.data(), pos.bytes, cudaMemcpyHostToDevice, st), "H2D positions");
  call(pty_warm_stitch(out, pos.as<float>(), P, wd.as<float>(), S, N, WARM_AMP_MEAN, WARM_AMP_SCALE,
                       WARM_GRAD_SCALE, acc.as<float>(), s->X, s->Y, st),
       "stitching");
  call(pty_warm_object(acc.as<float>(), s->X, s->Y, WARM_WMIN, WARM_AMP_MEAN, static_cast<const float*>(s->probe.p), N,
                       pos.as<float>(), P, s->amp.as<float>(), work.as<float>(), static_cast<float*>(s->obj.p), st),
       "assembly");
}

}  // namespace pty
