// Simulation mode (simulate=1): the patterns of an ePIE / DM run come from the engine's forward model instead of
// data, as in the reference's IPhaser::init (src/IPhaser.cpp:93-117,181-192).
//
// Object (Sample::loadFromFile, src/Sample.cpp:109-162; h_applyHammingToSample, src/SampleKernels.cu:75-90,510-518):
// the 8-bit PGM images data/lena<N>.pgm (magnitude) and data/baboon<N>.pgm (phase), read relative to the working
// directory like the reference, give magnitude (v / max) * 0.9 + 0.1 and phase (v / max) * pi/3; the image times the
// 2-D Hamming window (0.53836 - 0.46164 cos(2 pi c / (w - 1))) (same over rows) sits centred in an object of the
// scan's size, zero elsewhere.
// Probe (Probe::simulate, src/Probe.cpp:184-207,332-340; d_initProbeSimulated, src/ProbeKernels.cu:192-205):
// amplitude |sinc(r dx_s / beamSize) exp(-r^2 / window^2)| with r the distance from (N/2, N/2) in pixels and
// window = N / 4.7, phase pi * f with f a random field smoothed by a Gaussian of FWHM 10 px (circular convolution
// with the kernel centred at (N/2, N/2)) and divided by its maximum.  The reference seeds that field from the clock;
// here it comes from the session's seed (SplitMix64 from seed ^ 0xA0761D6478BD642F, u = ((next >> 11) + 0.5) 2^-53).
// Patterns (Diffractions::simulate, src/Diffractions.cpp:80-117): |FFT2(O_bilinear(pos) * P)| at every scan
// position, no noise.  The reconstruction then starts as the reference's does, from a cleared object and the probe
// guess of these patterns (prePhase, src/IPhaser.cpp:296-304).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "kernels.h"
#include "session.h"

namespace pty {
namespace {

struct Pgm {
  int w = 0, h = 0;
  std::vector<unsigned char> px;  // row-major, h rows of w
};

// Binary (P5) or plain (P2) PGM with maxval <= 255 (sdkLoadPGM<unsigned char> reads 8-bit P5).
Pgm read_pgm(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) fail(PTY_ERR_IO, "simulate: cannot open " + path + " (read relative to the working directory)");
  auto token = [&]() {
    std::string t;
    int c;
    while ((c = f.get()) != EOF) {
      if (c == '#') {  // comment to the end of the line
        while ((c = f.get()) != EOF && c != '\n') {
        }
        continue;
      }
      if (std::isspace(c)) {
        if (!t.empty()) break;
        continue;
      }
      t.push_back(char(c));
    }
    return t;
  };
  const std::string magic = token();
  if (magic != "P5" && magic != "P2") fail(PTY_ERR_INVALID, "simulate: " + path + " is not a PGM image");
  Pgm g;
  g.w = std::atoi(token().c_str());
  g.h = std::atoi(token().c_str());
  const int maxval = std::atoi(token().c_str());
  if (g.w < 1 || g.h < 1 || maxval < 1 || maxval > 255)
    fail(PTY_ERR_INVALID, "simulate: " + path + " must be an 8-bit PGM image");
  g.px.resize(size_t(g.w) * g.h);
  if (magic == "P5") {
    f.read(reinterpret_cast<char*>(g.px.data()), std::streamsize(g.px.size()));
    if (size_t(f.gcount()) != g.px.size()) fail(PTY_ERR_INVALID, "simulate: " + path + " is truncated");
  } else {
    for (auto& v : g.px) {
      const std::string t = token();
      if (t.empty()) fail(PTY_ERR_INVALID, "simulate: " + path + " is truncated");
      v = static_cast<unsigned char>(std::atoi(t.c_str()));
    }
  }
  return g;
}

}  // namespace

// The object of simulation mode (X x Y complex64, interleaved) from the two images.
std::vector<float> sim_object_from_files(int N, int X, int Y) {
  char a[64], b[64];
  std::snprintf(a, sizeof(a), "data/lena%d.pgm", N);
  std::snprintf(b, sizeof(b), "data/baboon%d.pgm", N);
  const Pgm mag = read_pgm(a), arg = read_pgm(b);
  if (mag.w != arg.w || mag.h != arg.h) fail(PTY_ERR_INVALID, "simulate: the two images differ in size");
  if (mag.h > X || mag.w > Y)
    fail(PTY_ERR_INVALID, "simulate: the " + std::to_string(mag.h) + " x " + std::to_string(mag.w) +
                              " image does not fit the scan's " + std::to_string(X) + " x " + std::to_string(Y) +
                              " object");
  unsigned char mmax = 0, amax = 0;
  for (unsigned char v : mag.px) mmax = v > mmax ? v : mmax;
  for (unsigned char v : arg.px) amax = v > amax ? v : amax;
  if (!mmax || !amax) fail(PTY_ERR_INVALID, "simulate: an image is all zero");
  std::vector<float> obj(2 * size_t(X) * Y, 0.f);
  const int h = mag.h, w = mag.w, ox = X / 2 - h / 2, oy = Y / 2 - w / 2;
  const int aw = (w + 31) / 32 * 32;  // the window's period is the launch's block width (alignUp(w, 32)) - 1
  for (int r = 0; r < h; ++r)
    for (int c = 0; c < w; ++c) {
      const float m = float(double(float(mag.px[size_t(r) * w + c]) / float(mmax)) * double(0.9f) + (1.0 - double(0.9f)));
      const float ph = float(double(float(arg.px[size_t(r) * w + c]) / float(amax)) * 1.0471975512);
      const double hc = 0.53836 - 0.46164 * std::cos(M_PI * (2.0 * c / (aw - 1)));
      const double hr = 0.53836 - 0.46164 * std::cos(M_PI * (2.0 * r / (aw - 1)));
      const float ham = float(hc * hr);
      const size_t o = size_t(ox + r) * Y + (oy + c);
      obj[2 * o] = float(m * std::cos(double(ph))) * ham;
      obj[2 * o + 1] = float(m * std::sin(double(ph))) * ham;
    }
  return obj;
}

// The simulated probe (N x N complex64, interleaved).
std::vector<float> sim_probe(int N, double beamSize, double dx_s, uint64_t seed) {
  const size_t NN = size_t(N) * N;
  std::vector<double> u(NN), t(NN), f(NN);
  uint64_t st = seed ^ 0xA0761D6478BD642Full;
  for (auto& v : u) v = (double(splitmix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  // circular convolution with exp(-((a - N/2)^2 + (b - N/2)^2) / s^2), s = 10 / 2.3548, separable
  const double sg = 10.0 / 2.3548;
  const int R = 40;
  std::vector<double> g(2 * R + 1);
  for (int d = -R; d <= R; ++d) g[d + R] = std::exp(-double(d) * d / (sg * sg));
  const int h = N / 2;
  for (int i = 0; i < N; ++i)  // along columns: t[i][j] = sum_b u[i][(j - b) mod N] g(b - N/2)
    for (int j = 0; j < N; ++j) {
      double acc = 0;
      for (int d = -R; d <= R; ++d) acc += u[size_t(i) * N + ((j - h - d) % N + 2 * N) % N] * g[d + R];
      t[size_t(i) * N + j] = acc;
    }
  double mx = 0;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double acc = 0;
      for (int d = -R; d <= R; ++d) acc += t[size_t(((i - h - d) % N + 2 * N) % N) * N + j] * g[d + R];
      f[size_t(i) * N + j] = acc;
      mx = acc > mx ? acc : mx;
    }
  const double window = double(N) / (2 * 2.35), factor = double(float(dx_s / beamSize));
  std::vector<float> pr(2 * NN);
  for (int x = 0; x < N; ++x)
    for (int y = 0; y < N; ++y) {
      const double a = x - N * 0.5, b = y - N * 0.5, r = std::sqrt(a * a + b * b);
      const double q = r * factor;
      double p = q != 0 ? std::sin(M_PI * q) / (M_PI * q) : 1.0;
      p = std::fabs(p * std::exp(-r * r / (window * window)));
      const double ph = M_PI * f[size_t(x) * N + y] / mx;
      pr[2 * (size_t(x) * N + y)] = float(p * std::cos(ph));
      pr[2 * (size_t(x) * N + y) + 1] = float(p * std::sin(ph));
    }
  return pr;
}

// Fills the session's patterns (s->amp) from the forward model at the positions of the session's geometry (s->geo,
// s->X, s->Y, s->P already set).
void simulate_session_patterns(pty_session* s) {
  const pty_params& p = s->prm;
  const int N = s->N, X = s->X, Y = s->Y, P = s->P;
  const std::vector<float> obj = sim_object_from_files(N, X, Y);
  const std::vector<float> probe = sim_probe(N, p.beamSize, sample_pixel_size(p.lambd, p.z, p.dx_d, N), p.seed);
  const size_t NN = size_t(N) * N;
  const int chunk = int(std::max<size_t>(1, std::min<size_t>(size_t(P), (size_t(256) << 20) / (16 * NN))));
  DeviceBuf dobj, dprobe, dpos, psi, work, tw;
  dobj.alloc(sizeof(float) * obj.size(), "simulated object");
  dprobe.alloc(sizeof(float) * probe.size(), "simulated probe");
  dpos.alloc(sizeof(float) * s->geo.pos.size(), "positions");
  psi.alloc(sizeof(float2) * NN * chunk, "exit waves");
  work.alloc(sizeof(float2) * NN * chunk, "FFT work");
  s->amp.alloc(sizeof(float) * NN * P, "patterns");
  check_cuda(cudaMemcpyAsync(dobj.p, obj.data(), dobj.bytes, cudaMemcpyHostToDevice, s->stream), "H2D object");
  check_cuda(cudaMemcpyAsync(dprobe.p, probe.data(), dprobe.bytes, cudaMemcpyHostToDevice, s->stream), "H2D probe");
  check_cuda(cudaMemcpyAsync(dpos.p, s->geo.pos.data(), dpos.bytes, cudaMemcpyHostToDevice, s->stream), "H2D pos");
  float2* twp = nullptr;
  check_cuda(make_twiddles(N, &twp, s->stream), "twiddles");
  tw.p = twp;
  tw.bytes = tw.cap = sizeof(float2) * N;
  tw.dev = s->dev;
  for (int i0 = 0; i0 < P; i0 += chunk) {
    const int cnt = std::min(chunk, P - i0);
    check_cuda(simulate_patterns(dobj.as<float2>(), X, Y, dprobe.as<float2>(), N, dpos.as<float2>() + i0, cnt,
                                 psi.as<float2>(), work.as<float2>(), tw.as<float2>(), s->amp.as<float>() + NN * i0,
                                 s->stream),
               "simulate");
    s->launches += 2;
  }
  check_cuda(cudaStreamSynchronize(s->stream), "simulate");
  s->have_patterns = true;
}

}  // namespace pty
