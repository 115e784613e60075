// ============================================================================================================
// ORACLE — TEST INFRASTRUCTURE ONLY.  NOT PART OF THE PRODUCT.
//
// A plain C++ restatement of the reference's ptychography inner loop (ePIE and its "reference DM"), used by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.  The product (libptychopy_b200)
// never links, loads or calls anything in this directory.
//
// Parity status: pinned to the reference's own device code.  oracle/ref_build.py compiles the reference's
// hot-path device functions unchanged (DM callbacks, ePIE modulus / object / probe updates and error metric, the
// texture gather, the forward model, the MLs step-length terms and modulus factor, the raster mesh) and
// tests/test_gpu_refstages.py runs them on the GPU against this file's stages and whole iterations (DM and ePIE
// to FP32 round-off; the raster mesh and the texture filter weights bit for bit).  The reference ships no golden
// vectors; numpy.fft, hand-derived known answers (tests/test_oracle.py) and committed fixtures generated from this
// file (tests/golden/make_golden.py) pin the rest.
//
// Numerics: templated on the real type.  `double` is the FP64 oracle; `float` + std::thread is the multithreaded
// FP32 CPU baseline that bench.py times.  Scan geometry is computed in FP32 exactly as the reference does it
// (its positions are FP32 on the device), so both instantiations share it.
//
// Reference files restated (paths inside the ptychopy project):
//   geometry       src/Parameters.h:175-179, src/Parameters.cpp:650-652, src/ScanMeshKernels.cu:46-93,153-170,
//                  src/IPtychoScanMesh.cpp:86-109, src/CartesianScanMesh.cpp:57-92, src/ListScanMesh.cpp:55-129
//   probe guess    src/Probe.cpp:303-318,342-374, src/ProbeKernels.cu:52-63,207-218,388-407,582-590,
//                  src/utilities.cpp:138-154, src/utilitiesKernels.cu:619-682
//   ePIE           src/ePIE.cpp:65-129, src/SampleKernels.cu:167-178,209-215,244-294 (texture setup :493-502),
//                  src/ProbeKernels.cu:425-458, src/Sample.cpp:266-275,333-345, src/Probe.cpp:1750-1774,
//                  src/utilities.cpp:188-216, src/utilitiesKernels.cu:619-712,1866-1925
//   probe modes    src/Probe.cpp:229-242,320-330,1768-1781, src/ProbeKernels.cu:82-97,509-515,
//                  src/utilitiesKernels.cu:853-867,2051-2082
//   DM             src/DM.cu:46-128, src/SampleKernels.cu:416-490,686-719, src/Sample.cpp:333-345,
//                  src/Probe.cpp:296-301,1761-1766
//   error metric   src/utilities.cpp:188-195, src/utilitiesKernels.cu:684-712, src/Diffractions.cpp:234-242
// ============================================================================================================
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace {

template <typename R> using cx = std::complex<R>;

// ---------------------------------------------------------------- FFT (unnormalised, cuFFT sign convention)
// Forward: X[k] = sum_n x[n] exp(-2*pi*i*k*n/L); inverse: exp(+...), no 1/L scaling (CUFFT_FORWARD/INVERSE).
template <typename R> struct Fft1 {
  int L = 0, logL = 0;
  std::vector<cx<R>> tw;       // exp(-2*pi*i*m/L), m < L/2, computed in double
  std::vector<int> rev;
  explicit Fft1(int n) : L(n) {
    while ((1 << logL) < L) ++logL;
    tw.resize(L / 2);
    for (int m = 0; m < L / 2; ++m) {
      double a = -2.0 * M_PI * double(m) / double(L);
      tw[m] = cx<R>(R(std::cos(a)), R(std::sin(a)));
    }
    rev.resize(L);
    for (int i = 0; i < L; ++i) {
      int r = 0;
      for (int b = 0; b < logL; ++b) r |= ((i >> b) & 1) << (logL - 1 - b);
      rev[i] = r;
    }
  }
  // In-place transform of L points with element stride `stride`.
  void run(cx<R>* x, int stride, bool inverse, cx<R>* scratch) const {
    for (int i = 0; i < L; ++i) scratch[rev[i]] = x[i * stride];
    for (int len = 2; len <= L; len <<= 1) {
      int half = len >> 1, step = L / len;
      for (int s = 0; s < L; s += len)
        for (int j = 0; j < half; ++j) {
          cx<R> w = tw[j * step];
          if (inverse) w = std::conj(w);
          cx<R> a = scratch[s + j], b = scratch[s + j + half] * w;
          scratch[s + j] = a + b;
          scratch[s + j + half] = a - b;
        }
    }
    for (int i = 0; i < L; ++i) x[i * stride] = scratch[i];
  }
};

// 2-D transform of an N x N row-major array (rows = first index x, columns = second index y).
template <typename R> void fft2(const Fft1<R>& f, cx<R>* a, bool inverse, std::vector<cx<R>>& scratch) {
  const int N = f.L;
  scratch.resize(N);
  for (int r = 0; r < N; ++r) f.run(a + size_t(r) * N, 1, inverse, scratch.data());
  for (int c = 0; c < N; ++c) f.run(a + c, N, inverse, scratch.data());
}

// The same transform with the rows, then the columns, split over nthreads threads (same arithmetic per line, so
// the result is identical to fft2).
template <typename R> void fft2_mt(const Fft1<R>& f, cx<R>* a, bool inverse, int nthreads) {
  const int N = f.L;
  if (nthreads <= 1 || N < 256) {
    std::vector<cx<R>> scr;
    fft2(f, a, inverse, scr);
    return;
  }
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
      th.emplace_back([&, t, pass] {
        std::vector<cx<R>> scr(N);
        for (int l = t; l < N; l += nthreads) {
          if (pass == 0)
            f.run(a + size_t(l) * N, 1, inverse, scr.data());
          else
            f.run(a + l, N, inverse, scr.data());
        }
      });
    for (auto& x : th) x.join();
  }
}

// K stacked N x N transforms: one thread per mode when there are several, else the rows / columns of the one
// transform split over the threads.  Each line sees the same arithmetic as fft2.
template <typename R> void fft2_modes(const Fft1<R>& f, cx<R>* a, int K, bool inverse, int nthreads) {
  const size_t NN = size_t(f.L) * f.L;
  if (K == 1 || nthreads <= 1) {
    for (int k = 0; k < K; ++k) fft2_mt(f, a + k * NN, inverse, nthreads);
    return;
  }
  const int T = std::min(K, nthreads);
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&, t] {
      std::vector<cx<R>> scr;
      for (int k = t; k < K; k += T) fft2(f, a + k * NN, inverse, scr);
    });
  for (auto& x : th) x.join();
}

// fn(i) for i in [0, n), split into contiguous chunks over nthreads threads (serial when nthreads <= 1).
template <typename F> void parallel_rows(int n, int nthreads, F&& fn) {
  if (nthreads <= 1 || n < 2 * nthreads) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([&, t] {
      for (int i = int(int64_t(n) * t / nthreads); i < int(int64_t(n) * (t + 1) / nthreads); ++i) fn(i);
    });
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------- geometry (FP32 like the reference)
// src/Parameters.h:175-179 returns real_t (float): dx_s = (float)(lambda*z/(N*dx_d)).
double sample_pixel(double lambda, double z, double dx_d, int N) {
  return double(float((lambda * z) / (double(N) * dx_d)));
}

struct Mesh {
  std::vector<float> pos;  // 2*P, (x=row, y=column), shifted by -min
  int X = 0, Y = 0;
};

// Applies min/max, object size and -min shift: src/IPtychoScanMesh.cpp:86-109.
void finish_mesh(std::vector<float>& raw, int P, bool padZero, int N, bool flip, Mesh& m) {
  float mnx = std::numeric_limits<float>::max(), mny = mnx, mxx = -mnx, mxy = -mnx;
  for (int i = 0; i < P; ++i) {
    mnx = std::min(mnx, raw[2 * i]); mxx = std::max(mxx, raw[2 * i]);
    mny = std::min(mny, raw[2 * i + 1]); mxy = std::max(mxy, raw[2 * i + 1]);
  }
  if (padZero) {  // list meshes are padded to a multiple of 1024 with (0,0) entries that join the min/max
    mnx = std::min(mnx, 0.f); mxx = std::max(mxx, 0.f); mny = std::min(mny, 0.f); mxy = std::max(mxy, 0.f);
  }
  volatile float ex = (mxx - mnx) + float(N), ey = (mxy - mny) + float(N);
  m.X = int(std::ceil(ex));
  m.Y = int(std::ceil(ey));
  m.pos.resize(2 * size_t(P));
  for (int i = 0; i < P; ++i) {
    float tx = raw[2 * i], ty = raw[2 * i + 1];
    m.pos[2 * i] = flip ? ty - mny : tx - mnx;
    m.pos[2 * i + 1] = flip ? tx - mnx : ty - mny;
  }
}

// ---------------------------------------------------------------- bilinear patch fetch (texture emulation)
// tex2D(obj, col+qy+0.5f, row+qx+0.5f) with linear filtering, clamp addressing, unnormalised coordinates
// (src/SampleKernels.cu:167-178, :493-502).  Texture filtering weights are 1.8 fixed point; this restatement
// rounds the fractional part to the nearest 1/256.
inline void tex_coord(float base, int idx, int extent, int& i0, int& i1, double& a) {
  volatile float c = float(idx) + base;  // col + offsetY, rounded to float
  volatile float t = c + 0.5f;           // + 0.5f, rounded to float
  double xb = double(t) - 0.5;
  double fl = std::floor(xb);
  double fr = xb - fl;
  a = std::floor(fr * 256.0 + 0.5) / 256.0;
  long long i = (long long)fl;
  auto clampi = [&](long long v) { return int(v < 0 ? 0 : (v >= extent ? extent - 1 : v)); };
  i0 = clampi(i);
  i1 = clampi(i + 1);
}

template <typename R>
void extract_patch(const cx<R>* O, int X, int Y, float qx, float qy, int N, cx<R>* out) {
  std::vector<int> c0(N), c1(N);
  std::vector<double> ca(N);
  for (int c = 0; c < N; ++c) tex_coord(qy, c, Y, c0[c], c1[c], ca[c]);
  for (int r = 0; r < N; ++r) {
    int r0, r1;
    double b;
    tex_coord(qx, r, X, r0, r1, b);
    for (int c = 0; c < N; ++c) {
      double a = ca[c];
      cx<R> v00 = O[size_t(r0) * Y + c0[c]], v01 = O[size_t(r0) * Y + c1[c]];
      cx<R> v10 = O[size_t(r1) * Y + c0[c]], v11 = O[size_t(r1) * Y + c1[c]];
      out[size_t(r) * N + c] = v00 * R((1 - a) * (1 - b)) + v01 * R(a * (1 - b)) + v10 * R((1 - a) * b) +
                               v11 * R(a * b);
    }
  }
}

// ---------------------------------------------------------------- seeded visiting order (ePIE)
// The reference draws `rand() % remaining` from the list of not-yet-visited positions and erases the pick
// (src/ePIE.cpp:93-97) with a time seed.  The seeded generator here is SplitMix64; one stream per session,
// continued across iterations.  The product's host code implements the same generator.
inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void visiting_order(uint64_t& state, int P, int* order) {
  std::vector<int> rem(P);
  for (int i = 0; i < P; ++i) rem[i] = i;
  for (int s = 0; s < P; ++s) {
    int k = int(splitmix64(state) % uint64_t(rem.size()));
    order[s] = rem[k];
    rem.erase(rem.begin() + k);
  }
}

template <typename R> inline cx<R> constrain_phase(cx<R> v) {
  // src/SampleKernels.cu:209-215: arg clamped to <= 0, magnitude kept.
  R mag = std::abs(v), arg = std::atan2(v.imag(), v.real());
  arg = arg <= R(0) ? arg : R(0);
  return cx<R>(mag * std::cos(arg), mag * std::sin(arg));
}

// MLs modulus factor (d_modulus_amplitude with R_offset = 1, src/DiffractionsKernels.cu:127-137, called from
// Diffractions::modulus_constraint, src/Diffractions.cpp:281-310): A / (|Psi| + 1e-9) - 1.
template <typename R> inline R mls_modulus_factor(R A, R ap) { return A / (ap + R(1e-9)) - R(1); }

// Per-pixel terms of the MLs 2x2 step-length system (d_get_optimal_step_lsq, src/utilitiesKernels.cu:444-466):
// dOP = oup * probe; AA1 = |dOP|^2 + lambda, AA2 = dOP conj(dPO), AA4 = |dPO|^2 + lambda, Atb1 = Re(conj(dOP) chi),
// Atb2 = Re(conj(dPO) chi).
template <typename R>
inline void mls_lsq_terms(cx<R> chi, cx<R> oup, cx<R> dPO, cx<R> probe, R lam, R& a1, cx<R>& a2, R& a4, R& b1,
                          R& b2) {
  const cx<R> dOP = oup * probe;
  a1 = std::norm(dOP) + lam;
  a2 = dOP * std::conj(dPO);
  a4 = std::norm(dPO) + lam;
  b1 = (std::conj(dOP) * chi).real();
  b2 = (std::conj(dPO) * chi).real();
}

template <typename R> inline cx<R> modulus_phase(cx<R> psi, R amp) {
  // src/utilitiesKernels.cu:626-631 / src/SampleKernels.cu:443-447: amp * exp(i*atan2(im, re)).
  // psi == 0 (either zero sign) is pinned to phase 0: atan2 of signed zeros is implementation-defined there.
  if (psi.real() == R(0) && psi.imag() == R(0)) return cx<R>(amp, R(0));
  R ph = std::atan2(psi.imag(), psi.real());
  return cx<R>(amp * std::cos(ph), amp * std::sin(ph));
}

// ---------------------------------------------------------------- probe guess (Q10 in the build notes)
// src/Probe.cpp:360-372 with d_initProbe (src/ProbeKernels.cu:207-218), d_normalizeDiffractionIntensities
// (:388-407), the modulus projection onto the mean amplitude (src/utilities.cpp:138-154) and normalize()
// (src/Probe.cpp:303-318).  Mode 0 only; modes >= 1 are zero.
template <typename R>
void probe_guess(const R* amp, int P, int N, double beamSize, double dx_s, int K, cx<R>* probe) {
  const double window = double(N) / (2 * 2.35);
  const double factor = double(float(dx_s / beamSize));
  std::fill(probe, probe + size_t(K) * N * N, cx<R>(0, 0));
  for (int x = 0; x < N; ++x)
    for (int y = 0; y < N; ++y) {
      double a = double(x) - N * 0.5, b = double(y) - N * 0.5;
      double r = std::sqrt(a * a + b * b);
      double p = r * factor;
      p = (p != 0) ? std::sin(M_PI * p) / (M_PI * p) : 1.0;
      double g = std::exp(-std::pow(window, -2.0) * r * r);
      probe[size_t(x) * N + y] = cx<R>(R(std::fabs(p * g)), 0);
    }
  std::vector<R> avg(size_t(N) * N, R(0));
  for (int p = 0; p < P; ++p)
    for (size_t i = 0; i < size_t(N) * N; ++i) avg[i] += amp[size_t(p) * N * N + i];
  for (auto& v : avg) v *= R(1.0 / double(P));
  Fft1<R> f(N);
  std::vector<cx<R>> scr;
  fft2(f, probe, false, scr);
  const R nrm = R(1.0 / double(N * N));
  for (size_t i = 0; i < size_t(N) * N; ++i) probe[i] = modulus_phase(probe[i], avg[i]) * nrm;
  fft2(f, probe, true, scr);
  R mx = 0;
  for (size_t i = 0; i < size_t(K) * N * N; ++i) mx = std::max(mx, std::abs(probe[i]));
  for (size_t i = 0; i < size_t(K) * N * N; ++i) probe[i] *= R(1.0 / double(mx));
}

// ---------------------------------------------------------------- session state shared by ePIE and DM
struct Flags {
  int phaseConstraint = 1, updateProbe = 10, updateModes = 20;
  int calculateRMS = 0;
  // ePIE's saturation level (float, as the reference's saturationValue): a pixel whose amplitude A has
  // A - saturation >= 0 floats (letFloat, src/utilitiesKernels.cu:619-624); +inf: none floats
  float saturation = std::numeric_limits<float>::infinity();
};

template <typename R> struct State {
  int N = 0, K = 1, P = 0, X = 0, Y = 0;
  std::vector<cx<R>> O, Pr;     // object X*Y, probe K*N*N
  std::vector<R> Ocache, Pcache;  // |O|^2 (m_objectIntensities), |P_k|^2 (m_intensities)
  R objMax = 0;                   // Sample::m_maxObjectIntensity (starts 0, src/Sample.cpp:216-220)
  R probeMax = 1;                 // Probe::m_maxIntensity (constructor value 1, src/Probe.cpp:54-58)
  bool useAll = false, modesInitialized = false;
};

// Probe::getModalDoubleMax (src/utilities.cpp:204-216): with all modes active and K>1, the max over pixels of
// the per-pixel modal sum; otherwise the max over the whole stacked K*N*N intensity array.
template <typename R> R probe_modal_max(const State<R>& s) {
  const size_t NN = size_t(s.N) * s.N;
  R mx = 0;
  if (s.useAll && s.K > 1) {
    for (size_t i = 0; i < NN; ++i) {
      R t = 0;
      for (int k = 0; k < s.K; ++k) t += s.Pcache[k * NN + i];
      mx = std::max(mx, t);
    }
  } else {
    for (size_t i = 0; i < size_t(s.K) * NN; ++i) mx = std::max(mx, s.Pcache[i]);
  }
  return mx;
}

// Probe::orthogonalize (src/Probe.cpp:229-242) with h_projectUtoV (src/ProbeKernels.cu:509-515):
// classical Gram-Schmidt against the ORIGINAL copy of mode i; factor = <v,u>/<u,u> with <a,b> = sum conj(a)*b.
template <typename R> void orthogonalize(State<R>& s) {
  const size_t NN = size_t(s.N) * s.N;
  std::vector<cx<R>> copy(s.Pr);
  for (int i = 1; i < s.K; ++i)
    for (int j = i - 1; j >= 0; --j) {
      const cx<R>* u = &s.Pr[j * NN];
      const cx<R>* v = &copy[i * NN];
      cx<R> vu(0, 0), uu(0, 0);
      for (size_t p = 0; p < NN; ++p) {
        vu += std::conj(v[p]) * u[p];
        uu += std::conj(u[p]) * u[p];
      }
      cx<R> fac = vu / uu;
      for (size_t p = 0; p < NN; ++p) s.Pr[i * NN + p] -= fac * u[p];
    }
}

// Probe::beginModalReconstruction / initProbeModes (src/Probe.cpp:320-330,1768-1774).
template <typename R> void begin_modal(State<R>& s) {
  const size_t NN = size_t(s.N) * s.N;
  s.useAll = true;
  if (!s.modesInitialized) {
    if (s.K > 1) {
      for (int k = 1; k < s.K; ++k)
        for (size_t p = 0; p < NN; ++p) {
          cx<R> v = s.Pr[p] * R(0.05);
          s.Pr[k * NN + p] = v;
          R m = std::abs(v);
          s.Pcache[k * NN + p] = m * m;
        }
      orthogonalize(s);
      s.modesInitialized = true;
    }
    s.probeMax = probe_modal_max(s);
  }
}

// ---------------------------------------------------------------- ePIE iteration (src/ePIE.cpp:65-129)
template <typename R>
R epie_iteration(State<R>& s, const R* amp, const float* pos, const R* sqsum, const Flags& fl, int iter,
                 uint64_t& rng, int* status, int nthreads = 1) {
  const int N = s.N, K = s.K, P = s.P;
  const size_t NN = size_t(N) * N;
  const bool pc = iter <= fl.phaseConstraint, up = iter >= fl.updateProbe, um = iter >= fl.updateModes;
  if (um) begin_modal(s);
  const int Ka = s.useAll ? K : 1;
  std::vector<int> order(P);
  visiting_order(rng, P, order.data());
  Fft1<R> f(N);
  std::vector<cx<R>> patch(NN), psiOld(size_t(Ka) * NN), Psi(size_t(Ka) * NN), psi(size_t(Ka) * NN);
  const R nrm = R(1.0 / double(N * N));
  double err = 0;
  for (int step = 0; step < P; ++step) {
    const int i = order[step];
    const float qx = pos[2 * i], qy = pos[2 * i + 1];
    if (qx < 0 || qy < 0) { *status = -2; return R(0); }
    extract_patch(s.O.data(), s.X, s.Y, qx, qy, N, patch.data());
    for (int k = Ka - 1; k >= 0; --k)
      for (size_t p = 0; p < NN; ++p) psiOld[k * NN + p] = patch[p] * s.Pr[k * NN + p];
    for (int k = 0; k < Ka; ++k) std::copy(&psiOld[k * NN], &psiOld[k * NN] + NN, &Psi[k * NN]);
    fft2_modes(f, Psi.data(), Ka, false, nthreads);
    const R* A = amp + size_t(i) * NN;
    // a floating pixel (d_adjustFFT / d_adjustModalFFT, src/utilitiesKernels.cu:634-682) keeps Psi with one mode
    // and takes the modal factor with 1 in place of A with several
    auto floats = [&](size_t p) { return float(A[p]) - fl.saturation >= 0.f; };
    if (Ka == 1) {
      for (size_t p = 0; p < NN; ++p) psi[p] = (floats(p) ? Psi[p] : modulus_phase(Psi[p], A[p])) * nrm;
    } else {
      for (size_t p = 0; p < NN; ++p) {
        R m2 = 0;
        for (int k = 0; k < Ka; ++k) m2 += std::norm(Psi[k * NN + p]);
        // rsqrt(0) gives inf and 0*inf = NaN in the reference; a pixel with no modal power is pinned to 0 here.
        R sc = m2 > R(0) ? R(1) / std::sqrt(m2) : R(0);
        const R a = floats(p) ? R(1) : A[p];
        for (int k = 0; k < Ka; ++k) psi[k * NN + p] = Psi[k * NN + p] * (a * sc * nrm);
      }
    }
    if (fl.calculateRMS) {  // error on FFT(psi_old), src/utilities.cpp:188-195, src/utilitiesKernels.cu:684-712
      double e = 0;
      for (size_t p = 0; p < NN; ++p) {
        cx<R> t(0, 0);
        for (int k = 0; k < Ka; ++k) t += Psi[k * NN + p];
        e += std::fabs(double(A[p]) - double(std::abs(t)));
      }
      err += (e / Ka) / double(sqsum[i]);
    }
    fft2_modes(f, psi.data(), Ka, true, nthreads);
    const int ox = int(std::round(qx)), oy = int(std::round(qy));
    // Object update (d_updateObjectArray[M], src/SampleKernels.cu:244-294), c = 1/probeMax.
    const R cO = R(1.0 / double(s.probeMax));
    parallel_rows(N, nthreads, [&](int r) {
      for (int c = 0; c < N; ++c) {
        size_t p = size_t(r) * N + c, o = size_t(r + ox) * s.Y + (c + oy);
        cx<R> inc(0, 0);
        for (int k = 0; k < Ka; ++k) inc += std::conj(s.Pr[k * NN + p]) * (psi[k * NN + p] - psiOld[k * NN + p]);
        cx<R> v = s.O[o] + inc * cO;
        R mag = std::abs(v);
        if (pc) v = constrain_phase(v);
        s.O[o] = v;
        s.Ocache[o] = mag * mag;
      }
    });
    s.objMax = *std::max_element(s.Ocache.begin(), s.Ocache.end());
    if (up) {  // d_updateProbe[M] (src/ProbeKernels.cu:425-458), c = 1/objMax, uses the updated object
      const R cP = R(1.0 / double(s.objMax));
      parallel_rows(N, nthreads, [&](int r) {
        for (int c = 0; c < N; ++c) {
          size_t p = size_t(r) * N + c, o = size_t(r + ox) * s.Y + (c + oy);
          cx<R> oc = std::conj(s.O[o]);
          for (int k = 0; k < Ka; ++k) {
            cx<R> v = oc * (psi[k * NN + p] - psiOld[k * NN + p]) * cP + s.Pr[k * NN + p];
            R m = std::abs(v);
            s.Pr[k * NN + p] = v;
            s.Pcache[k * NN + p] = m * m;
          }
        }
      });
      s.probeMax = probe_modal_max(s);
    }
  }
  return R(err / P);
}

// ---------------------------------------------------------------- reference DM iteration (src/DM.cu:80-128)
template <typename R> struct DMState {
  std::vector<cx<R>> psi;        // P*N*N, zero at start (Cuda3DArray zeroed on allocation)
  double fac[2] = {0, 0};        // {1/objMax, 1/probeMax}, cached with hysteresis EPS
  bool started = false;
};

template <typename R> double sum_sq(const cx<R>* a, size_t n) {
  double t = 0;
  for (size_t i = 0; i < n; ++i) t += double(std::norm(a[i]));
  return t;
}

// Sum of the iteration's object / probe increments over position shards (interleaved re, im doubles), in place;
// identity when the whole scan is in one session.
typedef void (*DmReduceFn)(double* dO, size_t n_obj, double* dP, size_t n_probe, void* user);

template <typename R>
void dm_iteration(State<R>& s, DMState<R>& d, const R* amp, const float* pos, const Flags& fl, int iter,
                  int nthreads, DmReduceFn reduce = nullptr, void* reduce_user = nullptr) {
  const int N = s.N, P = s.P;
  const size_t NN = size_t(N) * N, XY = size_t(s.X) * s.Y;
  const bool pc = iter <= fl.phaseConstraint, up = iter >= fl.updateProbe;
  if (!d.started) {
    d.started = true;
    d.psi.assign(size_t(P) * NN, cx<R>(0, 0));
    d.fac[0] = 1.0 / double(s.objMax);
    d.fac[1] = 1.0 / double(s.probeMax);
  }
  // checkCache (src/DM.cu:54-73): a factor moves only when it changed by more than EPS = 1e-3.
  const double passed[2] = {1.0 / double(s.objMax), 1.0 / double(s.probeMax)};
  for (int j = 0; j < 2; ++j)
    if (std::fabs(d.fac[j] - passed[j]) > 1e-3) d.fac[j] = passed[j];
  const R f0 = R(d.fac[0]), f1 = R(d.fac[1]);
  const R nrm = R(1.0 / double(N * N));
  if (nthreads < 1) nthreads = 1;
  std::vector<std::vector<cx<R>>> dO(nthreads, std::vector<cx<R>>(XY)), dP(nthreads, std::vector<cx<R>>(NN));
  auto work = [&](int t) {
    Fft1<R> f(N);
    std::vector<cx<R>> scr, u(NN);
    for (int j = t; j < P; j += nthreads) {
      const int ox = int(std::round(pos[2 * j])), oy = int(std::round(pos[2 * j + 1]));
      cx<R>* pj = &d.psi[size_t(j) * NN];
      const R* A = amp + size_t(j) * NN;
      // forward: load callback 2*P*O - psi, store callback A*exp(i*arg)/N^2 (src/SampleKernels.cu:418-450)
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) {
          size_t p = size_t(r) * N + c;
          cx<R> ph = s.Pr[p] * s.O[size_t(r + ox) * s.Y + (c + oy)];
          u[p] = ph * R(2) - pj[p];
        }
      fft2(f, u.data(), false, scr);
      for (size_t p = 0; p < NN; ++p) u[p] = modulus_phase(u[p], A[p]) * nrm;
      fft2(f, u.data(), true, scr);
      // inverse store callback (src/SampleKernels.cu:452-490) with snapshot O and P
      for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) {
          size_t p = size_t(r) * N + c, o = size_t(r + ox) * s.Y + (c + oy);
          cx<R> ov = s.O[o], pv = s.Pr[p];
          cx<R> v = pj[p] + u[p] - (ov * pv) * R(2);
          cx<R> inc = std::conj(pv) * v * f1;
          if (pc) inc = constrain_phase(inc);
          dO[t][o] += inc;
          if (up) dP[t][p] += std::conj(ov) * v * f0;
          pj[p] = v;
        }
    }
  };
  if (nthreads == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  for (int t = 1; t < nthreads; ++t) {
    for (size_t i = 0; i < XY; ++i) dO[0][i] += dO[t][i];
    for (size_t i = 0; i < NN; ++i) dP[0][i] += dP[t][i];
  }
  if (reduce) {  // position shards: every shard adds the others' increments before applying them
    std::vector<double> bo(2 * XY), bp(2 * NN);
    for (size_t i = 0; i < XY; ++i) { bo[2 * i] = double(dO[0][i].real()); bo[2 * i + 1] = double(dO[0][i].imag()); }
    for (size_t i = 0; i < NN; ++i) { bp[2 * i] = double(dP[0][i].real()); bp[2 * i + 1] = double(dP[0][i].imag()); }
    reduce(bo.data(), XY, bp.data(), NN, reduce_user);
    for (size_t i = 0; i < XY; ++i) dO[0][i] = cx<R>(R(bo[2 * i]), R(bo[2 * i + 1]));
    for (size_t i = 0; i < NN; ++i) dP[0][i] = cx<R>(R(bp[2 * i]), R(bp[2 * i + 1]));
  }
  for (size_t i = 0; i < XY; ++i) s.O[i] += dO[0][i];
  if (up)
    for (size_t i = 0; i < NN; ++i) s.Pr[i] += dP[0][i];
  // updateIntensities(true) on object and probe: sums of |.|^2 (all stacked modes for the probe)
  s.objMax = R(sum_sq(s.O.data(), XY));
  s.probeMax = R(sum_sq(s.Pr.data(), size_t(s.K) * NN));
}

template <typename R> void load_state(State<R>& s, int N, int K, int P, int X, int Y, const double* obj,
                                      const double* probe, int probeCacheValid) {
  s.N = N; s.K = K; s.P = P; s.X = X; s.Y = Y;
  const size_t NN = size_t(N) * N, XY = size_t(X) * Y;
  s.O.resize(XY); s.Ocache.assign(XY, R(0));
  s.Pr.resize(size_t(K) * NN); s.Pcache.assign(size_t(K) * NN, R(0));
  for (size_t i = 0; i < XY; ++i) s.O[i] = cx<R>(R(obj[2 * i]), R(obj[2 * i + 1]));
  for (size_t i = 0; i < size_t(K) * NN; ++i) s.Pr[i] = cx<R>(R(probe[2 * i]), R(probe[2 * i + 1]));
  if (probeCacheValid) {  // Probe::init's guess path ends in updateIntensities(); a given probe does not
    for (size_t i = 0; i < size_t(K) * NN; ++i) s.Pcache[i] = std::norm(s.Pr[i]);
    s.probeMax = probe_modal_max(s);
  }
}

template <typename R> void store_state(const State<R>& s, double* obj, double* probe) {
  for (size_t i = 0; i < s.O.size(); ++i) { obj[2 * i] = double(s.O[i].real()); obj[2 * i + 1] = double(s.O[i].imag()); }
  for (size_t i = 0; i < s.Pr.size(); ++i) {
    probe[2 * i] = double(s.Pr[i].real());
    probe[2 * i + 1] = double(s.Pr[i].imag());
  }
}

// ---------------------------------------------------------------- MLs (src/MLS.cpp:74-490)
// LSQ-ML with random groups for one probe mode and one object.  Two paths: the reference's defaults
// (src/Parameters.h:162-163: variable probe with one extra mode, variable intensity, sub-pixel probe shift,
// position search from iteration PPS), and the fixed-probe core (none of these).  Geometry (ML mesh, src/CartesianScanMesh.cpp:94-177, src/IPtychoScanMesh.cpp:123-184):
// raw centred positions, object Np_o_new = ceil(extent * 1.2), window starts round(pos + ceilvar) - 1.
struct MlsGeometry {
  int X = 0, Y = 0;
  std::vector<int> r0, c0;   // window starts (0-based)
  int roix0 = 0, roiy0 = 0, roinx = 0, roiny = 0;  // object ROI of calc_object_norm (0-based start, size)
};

// The ROI is kept inside the object (the reference indexes it unchecked); an empty range stays empty.
void clamp_roi(int& a, int& n, int len) {
  const int b = std::min(len, a + std::max(n, 0));
  a = std::max(0, std::min(a, len));
  n = std::max(0, b - a);
}

MlsGeometry mls_geometry(const std::vector<float>& raw, int P, int N) {
  // raw: 2*P positions (x, y) in pixels, centred, as the ML mesh keeps them (no -min shift)
  float mnx = std::numeric_limits<float>::max(), mny = mnx, mxx = -mnx, mxy = -mnx;
  for (int i = 0; i < P; ++i) {
    mnx = std::min(mnx, raw[2 * i]); mxx = std::max(mxx, raw[2 * i]);
    mny = std::min(mny, raw[2 * i + 1]); mxy = std::max(mxy, raw[2 * i + 1]);
  }
  const float Np0 = 1e5f;
  const float cv0x = std::ceil(Np0 * 1.0f / 2 - float(N) * 1.0f / 2), cv0y = cv0x;
  const float rpx = (mxx + mnx) / 2, rpy = (mxy + mny) / 2;
  long long minx = 1LL << 40, maxx = -1, miny = 1LL << 40, maxy = -1;
  for (int i = 0; i < P; ++i) {  // tmpx from .y and tmpy from .x, as the reference's loop has them
    long long tx = (long long)std::round(raw[2 * i + 1] - rpy + cv0x);
    minx = std::min(minx, tx - 1); maxx = std::max(maxx, tx + N - 2);
    long long ty = (long long)std::round(raw[2 * i] - rpx + cv0y);
    miny = std::min(miny, ty - 1); maxy = std::max(maxy, ty + N - 2);
  }
  MlsGeometry g;
  g.X = int(std::ceil(double(float(maxx - minx) * (1 + 0.2f))));
  g.Y = int(std::ceil(double(float(maxy - miny) * (1 + 0.2f))));
  const float cvx = std::ceil(float(g.X) * 1.0f / 2 - float(N) * 1.0f / 2);
  const float cvy = std::ceil(float(g.Y) * 1.0f / 2 - float(N) * 1.0f / 2);
  g.r0.resize(P); g.c0.resize(P);
  for (int i = 0; i < P; ++i) {
    g.r0[i] = int(std::round(raw[2 * i] + cvx)) - 1;
    g.c0[i] = int(std::round(raw[2 * i + 1] + cvy)) - 1;
  }
  // precalculate_ROI: round(Np_o*0.5 + min) .. round(Np_o*0.5 + max) - 1, 1-based inclusive
  const long long ax = (long long)std::round(g.X * 0.5 + mnx), bx = (long long)std::round(g.X * 0.5 + mxx) - 1;
  const long long ay = (long long)std::round(g.Y * 0.5 + mny), by = (long long)std::round(g.Y * 0.5 + mxy) - 1;
  g.roix0 = int(ax - 1); g.roinx = int(bx - ax + 1);
  g.roiy0 = int(ay - 1); g.roiny = int(by - ay + 1);
  clamp_roi(g.roix0, g.roinx, g.X);
  clamp_roi(g.roiy0, g.roiny, g.Y);
  return g;
}

// Group partition of one iteration: a SplitMix64 Fisher-Yates permutation cut into groups of G = max(1, P/100)
// (src/IPtychoScanMesh.cpp:826-913), visited in a second shuffled order (src/MLS.cpp:106-113).
void mls_groups(uint64_t& rng, int P, std::vector<std::vector<int>>& groups) {
  std::vector<int> perm(P);
  for (int i = 0; i < P; ++i) perm[i] = i;
  for (int i = P - 1; i > 0; --i) std::swap(perm[i], perm[splitmix64(rng) % uint64_t(i + 1)]);
  const int G = std::max(1, P / 100);
  const int ng = (P + G - 1) / G;
  std::vector<std::vector<int>> g(ng);
  for (int k = 0; k < ng; ++k)
    for (int m = k * G; m < std::min(P, (k + 1) * G); ++m) g[k].push_back(perm[m]);
  std::vector<int> order(ng);
  for (int i = 0; i < ng; ++i) order[i] = i;
  for (int i = ng - 1; i > 0; --i) std::swap(order[i], order[splitmix64(rng) % uint64_t(i + 1)]);
  groups.clear();
  for (int i = 0; i < ng; ++i) groups.push_back(g[order[i]]);
}

template <typename R> struct MlsState {
  int N = 0, P = 0;
  MlsGeometry geo;
  std::vector<cx<R>> O, Pr;
  std::vector<R> A;           // sqrt(I), P*N*N
  std::vector<R> pobj;        // illumination weights (p_object), X*Y
  R maxIllum = 0;             // Probe::MAX_ILLUM from the set-up (src/Probe.cpp:507-613)
  double delta_p = 0.1, beta_LSQ = 0.9, beta_object = 1, beta_probe = 1;
  // the reference-default path
  bool variable = false;
  int PPS = 1 << 30;          // first iteration of the position search (probe_pos_search)
  int iter = 0;               // iterations done
  int K = 1;                  // probe modes (default path only)
  std::vector<cx<R>> Pk;      // modes 1..K-1, (K-1)*N*N (mode 0 is Pr)
  std::vector<cx<R>> E;       // extra probe mode (m_extramodes)
  std::vector<double> evo0, evo1;       // probe evolution: intensity and variable-mode weights per position
  std::vector<float> pos, pos_o, sub;   // 2*P: positions (x = rows), the originals, sub-pixel shifts (x = columns)
};

// Window starts and sub-pixel shifts from the positions (find_reconstruction_ROI, src/IPtychoScanMesh.cpp:122-171):
// position + ceil(Np_o/2 - N/2) in FP32, rounded; the start is one below; the shift's x is the column remainder.
// A start that would leave the object is clamped into it (the reference reads outside the array there).
template <typename R> void mls_windows(MlsState<R>& s) {
  const int N = s.N;
  const float cvx = std::ceil(float(s.geo.X) * 1.0f / 2 - float(N) * 1.0f / 2);
  const float cvy = std::ceil(float(s.geo.Y) * 1.0f / 2 - float(N) * 1.0f / 2);
  for (int i = 0; i < s.P; ++i) {
    const float p1 = s.pos[2 * i] + cvx, p2 = s.pos[2 * i + 1] + cvy;
    const float t1 = std::round(p1), t2 = std::round(p2);
    s.sub[2 * i] = p2 - t2;
    s.sub[2 * i + 1] = p1 - t1;
    s.geo.r0[i] = std::min(std::max(int(t1) - 1, 0), s.geo.X - N);
    s.geo.c0[i] = std::min(std::max(int(t2) - 1, 0), s.geo.Y - N);
  }
}

// Seeded stand-ins for the reference's time-seeded draws: curand uniforms for the extra mode (initVarModes,
// src/Probe.cpp:497-505 with d_initVarMOdes, src/ProbeKernels.cu:99-110: r1 e^{2 pi i r2}, all r1 drawn before all
// r2) and normalRandom for the variable-mode weights (1e-6 N(0,1), src/Probe.cpp:520-525).  SplitMix64 from
// seed ^ 0x3C6EF372FE94F82B, u = (bits >> 11 + 0.5) 2^-53, Box-Muller cos branch, one normal per pair.
// With K > 1 probe modes, 2 (K - 1) normals for the modes' phase tilts (initMLH, src/Probe.cpp:422-431) are drawn
// after the extra mode and before the weights.
void mls_variable_draws(uint64_t seed, int N, int P, int K, std::vector<cx<double>>& E, std::vector<double>& tilts,
                        std::vector<double>& evo1) {
  uint64_t st = seed ^ 0x3C6EF372FE94F82Bull;
  auto u = [&] { return (double(splitmix64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
  const size_t NN = size_t(N) * N;
  std::vector<double> r1(NN), r2(NN);
  for (auto& v : r1) v = u();
  for (auto& v : r2) v = u();
  E.resize(NN);
  for (size_t i = 0; i < NN; ++i) E[i] = cx<double>(r1[i] * std::cos(2 * M_PI * r2[i]), r1[i] * std::sin(2 * M_PI * r2[i]));
  auto normal = [&] {
    const double a = u(), b = u();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(2 * M_PI * b);
  };
  tilts.resize(2 * size_t(K > 1 ? K - 1 : 0));
  for (auto& v : tilts) v = normal();
  evo1.resize(P);
  for (auto& v : evo1) v = 1e-6 * normal();
}

// Eigen-decomposition of a Hermitian K x K matrix (row-major) by cyclic complex Jacobi rotations, FP64.  Eigenpairs
// in descending |eigenvalue|; each eigenvector (a column of V, unit norm) is turned so that its first component of at
// least half the largest magnitude is real and positive (robust to the equal-magnitude components that equal-power
// modes give).
void hermitian_eigen(int K, std::vector<cx<double>> A, std::vector<double>& lam, std::vector<cx<double>>& V) {
  V.assign(size_t(K) * K, cx<double>(0, 0));
  for (int i = 0; i < K; ++i) V[size_t(i) * K + i] = 1;
  double scale = 0;
  for (const auto& v : A) scale += std::norm(v);
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0;
    for (int p = 0; p < K; ++p)
      for (int q = p + 1; q < K; ++q) off += std::norm(A[size_t(p) * K + q]);
    if (off <= 1e-30 * scale) break;
    for (int p = 0; p < K; ++p)
      for (int q = p + 1; q < K; ++q) {
        const cx<double> apq = A[size_t(p) * K + q];
        const double m = std::abs(apq);
        if (m == 0.0) continue;
        const double app = A[size_t(p) * K + p].real(), aqq = A[size_t(q) * K + q].real();
        const double th = 0.5 * std::atan2(2 * m, aqq - app);
        const double c = std::cos(th), s = std::sin(th);
        const cx<double> em = std::conj(apq) / m;  // e^{-i phi}
        // A <- A G, G = [[c, s], [-s e^{-i phi}, c e^{-i phi}]] on columns p, q; then A <- G^H A; V <- V G
        for (int k = 0; k < K; ++k) {
          const cx<double> x = A[size_t(k) * K + p], y = A[size_t(k) * K + q];
          A[size_t(k) * K + p] = c * x - s * em * y;
          A[size_t(k) * K + q] = s * x + c * em * y;
          const cx<double> vx = V[size_t(k) * K + p], vy = V[size_t(k) * K + q];
          V[size_t(k) * K + p] = c * vx - s * em * vy;
          V[size_t(k) * K + q] = s * vx + c * em * vy;
        }
        for (int k = 0; k < K; ++k) {
          const cx<double> x = A[size_t(p) * K + k], y = A[size_t(q) * K + k];
          A[size_t(p) * K + k] = c * x - s * std::conj(em) * y;
          A[size_t(q) * K + k] = s * x + c * std::conj(em) * y;
        }
      }
  }
  std::vector<int> idx(K);
  for (int i = 0; i < K; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
    return std::abs(A[size_t(x) * K + x].real()) > std::abs(A[size_t(y) * K + y].real());
  });
  std::vector<cx<double>> W(size_t(K) * K);
  lam.resize(K);
  for (int j = 0; j < K; ++j) {
    const int c = idx[j];
    lam[j] = A[size_t(c) * K + c].real();
    double mx = 0;
    for (int k = 0; k < K; ++k) mx = std::max(mx, std::abs(V[size_t(k) * K + c]));
    int best = 0;
    while (best < K - 1 && std::abs(V[size_t(best) * K + c]) < 0.5 * mx) ++best;
    const cx<double> v = V[size_t(best) * K + c];
    const cx<double> ph = std::abs(v) > 0 ? std::conj(v) / std::abs(v) : cx<double>(1, 0);
    for (int k = 0; k < K; ++k) W[size_t(k) * K + j] = V[size_t(k) * K + c] * ph;
  }
  V = W;
}

// The MLs probe modes 1..K-1 (initMLH, src/Probe.cpp:422-490): mode 0 times the phase tilt
// e^{-2 pi i (t1 (c/N - 0.5) + t2 (r/N - 0.5))} (h_initVarProbe: fftshift, d_imshift_fft, fftshift back), then the
// modes are recombined by the eigenvectors of their Gram matrix G_ij = sum conj(m_i) m_j, in descending eigenvalue
// order (the reference's assignment m[sigma(i)] = combination i equals this when its eigen solver returns descending
// order; eigenvector phases are pinned by hermitian_eigen's convention).
template <typename R> void mls_init_modes(MlsState<R>& s, const std::vector<double>& tilts) {
  const int N = s.N, K = s.K;
  const size_t NN = size_t(N) * N;
  std::vector<std::vector<cx<R>>> m(K, std::vector<cx<R>>(NN));
  m[0] = s.Pr;
  for (int k = 1; k < K; ++k) {
    const double t1 = double(float(tilts[2 * (k - 1)])), t2 = double(float(tilts[2 * (k - 1) + 1]));
    for (int r = 0; r < N; ++r)
      for (int c = 0; c < N; ++c) {
        const double ph = -2 * M_PI * (t1 * (double(c) / N - 0.5) + t2 * (double(r) / N - 0.5));
        m[k][size_t(r) * N + c] = s.Pr[size_t(r) * N + c] * cx<R>(R(std::cos(ph)), R(std::sin(ph)));
      }
  }
  std::vector<cx<double>> G(size_t(K) * K);
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < K; ++j) {
      cx<double> acc(0, 0);
      for (size_t p = 0; p < NN; ++p) acc += std::conj(cx<double>(m[i][p])) * cx<double>(m[j][p]);
      G[size_t(i) * K + j] = acc;
    }
  std::vector<double> lam;
  std::vector<cx<double>> V;
  hermitian_eigen(K, G, lam, V);
  std::vector<std::vector<cx<R>>> out(K, std::vector<cx<R>>(NN, cx<R>(0, 0)));
  for (int i = 0; i < K; ++i)
    for (int q = 0; q < K; ++q) {
      const cx<R> v(R(V[size_t(q) * K + i].real()), R(V[size_t(q) * K + i].imag()));
      for (size_t p = 0; p < NN; ++p) out[i][p] += m[q][p] * v;
    }
  s.Pr = out[0];
  s.Pk.resize(size_t(K - 1) * NN);
  for (int k = 1; k < K; ++k) std::copy(out[k].begin(), out[k].end(), s.Pk.begin() + size_t(k - 1) * NN);
}

// ortho_modes (src/Probe.cpp:244-294), run after each iteration when K > 1: Gram-Schmidt in mode order (each mode
// minus its projections on the already orthogonalised earlier ones), then modes 1..K-1 are replaced by the modes
// ranked 1..K-1 by their power before the Gram-Schmidt; mode 0 is never replaced, as written.
template <typename R> void mls_ortho_modes(MlsState<R>& s) {
  const int K = s.K;
  const size_t NN = size_t(s.N) * s.N;
  auto mode = [&](int k) { return k == 0 ? s.Pr.data() : s.Pk.data() + size_t(k - 1) * NN; };
  std::vector<std::pair<double, int>> rank;
  for (int i = 0; i < K; ++i) {
    double pw = 0;
    for (size_t p = 0; p < NN; ++p) pw += std::norm(mode(i)[p]);
    rank.push_back({-pw, i});
    for (int j = 0; j < i; ++j) {
      double nj = 0;
      cx<double> sl(0, 0);
      for (size_t p = 0; p < NN; ++p) {
        nj += std::norm(mode(j)[p]);
        sl += cx<double>(mode(i)[p] * std::conj(mode(j)[p]));
      }
      const cx<R> pr(R(sl.real() / nj), R(sl.imag() / nj));
      for (size_t p = 0; p < NN; ++p) mode(i)[p] -= pr * mode(j)[p];
    }
  }
  std::sort(rank.begin(), rank.end());
  std::vector<cx<R>> all(s.Pr);
  all.insert(all.end(), s.Pk.begin(), s.Pk.end());
  for (int i = 1; i < K; ++i)
    std::copy(all.begin() + size_t(rank[i].second) * NN, all.begin() + size_t(rank[i].second + 1) * NN,
              s.Pk.begin() + size_t(i - 1) * NN);
}

// FFT frequency grid of the sub-pixel shift and the position gradient: fftshift(k/N - 0.5) (src/Probe.cpp:92-121),
// i.e. k/N for k < N/2 and k/N - 1 above.
inline double fft_freq(int k, int N) { return k < N / 2 ? double(k) / N : double(k) / N - 1.0; }

// a <- IFFT2(FFT2(a) e^{-2 pi i (sx f[c] + sy f[r])}) / N^2 (shift_probe, src/Probe.cpp:1261-1337)
template <typename R>
void mls_shift(const Fft1<R>& f, cx<R>* a, double sx, double sy, std::vector<cx<R>>& scr) {
  const int N = f.L;
  fft2(f, a, false, scr);
  for (int r = 0; r < N; ++r)
    for (int c = 0; c < N; ++c) {
      const double ph = -2.0 * M_PI * (sx * fft_freq(c, N) + sy * fft_freq(r, N));
      a[size_t(r) * N + c] *= cx<R>(R(std::cos(ph) / (double(N) * N)), R(std::sin(ph) / (double(N) * N)));
    }
  fft2(f, a, true, scr);
}

// p_object = sum_j |P|^2 placed at the windows (set_projections of aprobe2, src/Probe.cpp:701-729)
template <typename R> void mls_illumination(MlsState<R>& s, std::vector<R>& out) {
  const int N = s.N;
  out.assign(size_t(s.geo.X) * s.geo.Y, R(0));
  for (int j = 0; j < s.P; ++j)
    for (int x = 0; x < N; ++x)
      for (int y = 0; y < N; ++y)
        out[size_t(s.geo.r0[j] + x) * s.geo.Y + (s.geo.c0[j] + y)] += std::norm(s.Pr[size_t(x) * N + y]);
}

// initEvo normalisations (src/Probe.cpp:563-608 with h_preCalillum, src/ProbeKernels.cu:697-741), no variable modes.
template <typename R> void mls_setup(MlsState<R>& s, const std::vector<double>& intensitySums) {
  const int N = s.N;
  const size_t NN = size_t(N) * N;
  if (s.variable) {  // evolution weights; extra mode to unit RMS, its weights carry the norm (src/Probe.cpp:511-560)
    s.evo0.assign(s.P, 1.0);
    double se = 0;
    for (const auto& v : s.E) se += double(std::norm(v));
    const double rE = std::sqrt(se / double(NN));
    for (auto& v : s.E) v *= R(1.0 / rE);
    for (auto& v : s.evo1) v *= rE;
  }
  std::vector<R> illum;
  mls_illumination(s, illum);
  double si = 0, soi = 0;
  for (size_t i = 0; i < illum.size(); ++i) {
    si += illum[i];
    soi += double(std::norm(s.O[i])) * illum[i];
  }
  const R onorm = R(std::sqrt(soi / si));
  for (auto& v : s.O) v *= R(1) / onorm;
  double sp = 0;
  for (size_t i = 0; i < NN; ++i) sp += std::norm(s.Pr[i]);
  for (const auto& v : s.Pk) sp += std::norm(v);  // the mean illumination counts every mode
  const double meanillum = sp / double(NN);
  std::vector<double> corrv;
  for (int i = 0; i < s.P; ++i) corrv.push_back(meanillum / (intensitySums[i] / double(NN)));
  std::sort(corrv.begin(), corrv.end());
  const size_t n = corrv.size();
  double corr = (n % 2) ? corrv[n / 2] : 0.5 * (corrv[n / 2 - 1] + corrv[n / 2]);
  corr = std::sqrt(corr * double(NN));
  for (auto& v : s.Pr) v *= R(1.0 / corr);
  for (auto& v : s.Pk) v *= R(1.0 / corr);
  for (auto& v : s.E) v *= R(1.0 / corr);
  s.pobj = illum;
  for (auto& v : s.pobj) v /= R(corr * corr);
  s.maxIllum = *std::max_element(s.pobj.begin(), s.pobj.end());
}

template <typename R>
void mls_mode_updates(MlsState<R>& s, const std::vector<int>& g, const std::vector<std::vector<cx<R>>>& op,
                      const std::vector<std::vector<std::vector<cx<R>>>>& chm, cx<R> bpr);

template <typename R> double mls_iteration(MlsState<R>& s, uint64_t& rng, bool want_err) {
  const int N = s.N, X = s.geo.X, Y = s.geo.Y;
  const size_t NN = size_t(N) * N, XY = size_t(X) * Y;
  const int iter = ++s.iter;  // 1-based, as MLS::iteration's iter
  const bool var = s.variable;
  if (var && (iter == 1 || iter >= s.PPS)) mls_windows(s);  // find_reconstruction_ROI_O (src/MLS.cpp:86-89)
  // calc_object_norm (src/Probe.cpp:671-699): ||W o O|| / ||W|| over the object ROI, W = p_object
  {
    double sw = 0, swo = 0;
    for (int x = 0; x < s.geo.roinx; ++x)
      for (int y = 0; y < s.geo.roiny; ++y) {
        size_t i = size_t(s.geo.roix0 + x) * Y + (s.geo.roiy0 + y);
        double w = s.pobj[i];
        sw += w * w;
        swo += w * w * double(std::norm(s.O[i]));
      }
    const R on = sw > 0 ? R(std::sqrt(swo) / std::sqrt(sw)) : R(1);  // empty / unlit ROI: no rescale
    for (auto& v : s.Pr) v *= on;
    for (auto& v : s.Pk) v *= on;
    for (auto& v : s.E) v *= on;
    for (auto& v : s.O) v *= R(1) / on;
  }
  if (var) {
    // updateScanPositionsDiff (src/IPtychoScanMesh.cpp:340-368): remove the mean drift from the originals
    double s1x = 0, s1y = 0, s2x = 0, s2y = 0;
    for (int i = 0; i < s.P; ++i) {
      s1x += s.pos[2 * i]; s1y += s.pos[2 * i + 1];
      s2x += s.pos_o[2 * i]; s2y += s.pos_o[2 * i + 1];
    }
    const float dx = float(s1x / s.P) - float(s2x / s.P), dy = float(s1y / s.P) - float(s2y / s.P);
    for (int i = 0; i < s.P; ++i) { s.pos[2 * i] -= dx; s.pos[2 * i + 1] -= dy; }
  }
  if (var && iter > 1) {
    // remove_extra_degree (src/Probe.cpp:615-669).  Its mean and norm loops run over m_probe_evolution.size() = 2
    // entries (the number of evolution vectors), so only positions 0 and 1 are re-centred; kept as written.
    double se = 0;
    for (const auto& v : s.E) se += double(std::norm(v));
    const double vn = std::sqrt(se / double(NN));
    for (auto& v : s.E) v *= R(1.0 / vn);
    for (auto& v : s.evo1) v *= vn;
    const int len = std::min(2, s.P);
    double a0 = 0, a1 = 0;
    for (int i = 0; i < len; ++i) { a0 += s.evo0[i]; a1 += s.evo1[i]; }
    const float m0 = float(a0 / len), m1 = float(a1 / len);
    double sq = 0;
    for (int i = 0; i < len; ++i) {
      s.evo0[i] = (s.evo0[i] - m0) * 0.99 + 1;
      s.evo1[i] = s.evo1[i] - m1;
      sq += s.evo0[i] * s.evo0[i];
    }
    const double cn = std::sqrt(sq / len);
    for (int i = 0; i < len; ++i) s.evo0[i] /= cn;
    for (auto& v : s.Pr) v *= R(cn);
  }
  // updated_cached_illumination: h_set_projections adds sum |P|^2 at the windows to p_object without clearing it,
  // then /2, so p_object is a running average (MAX_ILLUM keeps its set-up value)
  {
    std::vector<R> il;
    mls_illumination(s, il);
    for (size_t i = 0; i < XY; ++i) s.pobj[i] = (s.pobj[i] + il[i]) / R(2);
  }
  const R pmax = *std::max_element(s.pobj.begin(), s.pobj.end());  // update_variable_probe's weight scale
  std::vector<std::vector<int>> groups;
  mls_groups(rng, s.P, groups);
  Fft1<R> f(N);
  std::vector<cx<R>> scr;
  const R nrm = R(1.0 / double(NN));
  const R lam = R(std::numeric_limits<float>::epsilon() / double(NN));
  double errsum = 0;
  std::vector<cx<R>> S(XY), pum(NN);
  for (const auto& g : groups) {
    const int G = int(g.size());
    std::vector<std::vector<cx<R>>> op(G, std::vector<cx<R>>(NN)), chi(G, std::vector<cx<R>>(NN)),
        vp(G, std::vector<cx<R>>(NN)), pu(G, std::vector<cx<R>>(NN));
    std::vector<std::vector<std::vector<cx<R>>>> chm(s.K - 1, std::vector<std::vector<cx<R>>>(G, std::vector<cx<R>>(NN)));
    for (int k = 0; k < G; ++k) {
      const int j = g[k];
      // get_illumination_probe (src/Probe.cpp:887-954): the position's probe P evo0 + E evo1, sub-pixel shifted
      for (size_t p = 0; p < NN; ++p)
        vp[k][p] = var ? s.Pr[p] * R(s.evo0[j]) + s.E[p] * R(s.evo1[j]) : s.Pr[p];
      if (var) mls_shift(f, vp[k].data(), s.sub[2 * j], s.sub[2 * j + 1], scr);
      for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
          const size_t p = size_t(x) * N + y;
          op[k][p] = s.O[size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y)];
          chi[k][p] = vp[k][p] * op[k][p];
        }
      fft2(f, chi[k].data(), false, scr);
      for (int m = 1; m < s.K; ++m) {  // the other modes' exit waves, unshifted (get_illumination_probe)
        auto& c = chm[m - 1][k];
        const cx<R>* Pm = s.Pk.data() + size_t(m - 1) * NN;
        for (size_t p = 0; p < NN; ++p) c[p] = Pm[p] * op[k][p];
        fft2(f, c.data(), false, scr);
      }
      const R* A = &s.A[size_t(j) * NN];
      double e = 0;
      for (size_t p = 0; p < NN; ++p) {  // modulus_constraint, R = A/(|Psi|+1e-9) - 1 (src/Diffractions.cpp:281-310)
        R a2 = std::norm(chi[k][p]);
        for (int m = 1; m < s.K; ++m) a2 += std::norm(chm[m - 1][k][p]);
        const R ap = s.K > 1 ? std::sqrt(a2) : std::abs(chi[k][p]);
        e += double(A[p] - ap) * double(A[p] - ap) * 0.25;
        const R rr = mls_modulus_factor(A[p], ap);
        chi[k][p] *= rr;
        for (int m = 1; m < s.K; ++m) chm[m - 1][k][p] *= rr;
      }
      errsum += std::sqrt(e / double(NN));
      fft2(f, chi[k].data(), true, scr);
      for (auto& v : chi[k]) v *= nrm;
      for (int m = 1; m < s.K; ++m) {
        fft2(f, chm[m - 1][k].data(), true, scr);
        for (auto& v : chm[m - 1][k]) v *= nrm;
      }
      // probe direction of this window, shifted back by the sub-pixel remainder (src/MLS.cpp:232-240)
      for (size_t p = 0; p < NN; ++p) pu[k][p] = chi[k][p] * std::conj(op[k][p]);
      if (var) mls_shift(f, pu[k].data(), -double(s.sub[2 * j]), -double(s.sub[2 * j + 1]), scr);
    }
    // probe direction: mean_j W[window] * pu_j, W = p/(p + 0.01 MAX_ILLUM) (src/MLS.cpp:249-285)
    std::fill(pum.begin(), pum.end(), cx<R>(0, 0));
    for (int k = 0; k < G; ++k) {
      const int j = g[k];
      for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
          const size_t p = size_t(x) * N + y;
          const R w0 = s.pobj[size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y)];
          pum[p] += pu[k][p] * (w0 / (w0 + s.maxIllum * R(0.01)));
        }
    }
    for (auto& v : pum) v *= R(1.0 / G);
    // object direction: set_projections of chi conj(vp), preconditioned by p + delta_p MAX_ILLUM (src/MLS.cpp:287-347)
    std::fill(S.begin(), S.end(), cx<R>(0, 0));
    for (int k = 0; k < G; ++k) {
      const int j = g[k];
      for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
          const size_t p = size_t(x) * N + y;
          S[size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y)] += chi[k][p] * std::conj(vp[k][p]);
        }
    }
    const R dmax = R(s.maxIllum * s.delta_p);
    // LSQ step sizes (d_get_optimal_step_lsq, src/utilitiesKernels.cu:444-466, and the 2x2 solve, src/MLS.cpp:349-417)
    std::vector<double> a1(G), a4(G), b1(G), b2(G);
    std::vector<cx<double>> a2(G);
    for (int k = 0; k < G; ++k) {
      const int j = g[k];
      double s1 = 0, s4 = 0, t1 = 0, t2 = 0;
      cx<double> s2(0, 0);
      for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
          const size_t p = size_t(x) * N + y, o = size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y);
          const cx<R> oup = S[o] / (s.pobj[o] + dmax);
          R a1p, a4p, b1p, b2p;
          cx<R> a2p;
          mls_lsq_terms(chi[k][p], oup, pum[p] * op[k][p], vp[k][p], lam, a1p, a2p, a4p, b1p, b2p);
          s1 += double(a1p);
          s4 += double(a4p);
          s2 += cx<double>(a2p);
          t1 += double(b1p);
          t2 += double(b2p);
        }
      a1[k] = s1; a4[k] = s4; a2[k] = s2; b1[k] = t1; b2[k] = t2;
    }
    double m1 = 0, m4 = 0;
    for (int k = 0; k < G; ++k) { m1 += a1[k]; m4 += a4[k]; }
    m1 = 0.1 * m1 / G; m4 = 0.1 * m4 / G;
    cx<double> bo(0, 0), bp(0, 0);
    for (int k = 0; k < G; ++k) {
      const double A11 = a1[k] + m1, A22 = a4[k] + m4;
      const cx<double> A12 = a2[k], A21 = std::conj(a2[k]);
      const cx<double> det = A11 * A22 - A12 * A21;
      const cx<double> x0 = (b1[k] * A22 - A12 * b2[k]) / det;
      const cx<double> x1 = (A11 * b2[k] - A21 * b1[k]) / det;
      bo += x0 * (s.beta_object * s.beta_LSQ);
      bp += x1 * (s.beta_probe * s.beta_LSQ);
    }
    bo /= double(G); bp /= double(G);
    // update_object / update_probe with the group-mean steps (src/Sample.cpp:277-331, src/Probe.cpp:1339-1364)
    const cx<R> bor(R(bo.real()), R(bo.imag())), bpr(R(bp.real()), R(bp.imag()));
    for (size_t i = 0; i < XY; ++i)
      if (S[i] != cx<R>(0, 0)) s.O[i] += bor * (S[i] / (s.pobj[i] + dmax));
    for (size_t p = 0; p < NN; ++p) s.Pr[p] += bpr * pum[p];
    if (var && iter >= s.PPS) {
      // gradient_position_solver (src/Probe.cpp:956-1118): object gradients by the Fourier derivative, a least-
      // squares shift per window clamped to 0.2 px.  The column-direction gradient (dX, the column frequency grid)
      // moves the position's x (the row coordinate) and the row-direction one its y, as the reference pairs them.
      for (int k = 0; k < G; ++k) {
        const int j = g[k];
        std::vector<cx<R>> img(op[k]), dX(NN), dY(NN);
        fft2(f, img.data(), false, scr);
        for (int r = 0; r < N; ++r)
          for (int c = 0; c < N; ++c) {
            const size_t p = size_t(r) * N + c;
            const cx<R> d = img[p] * cx<R>(0, R(2.0 * M_PI));
            dX[p] = d * R(fft_freq(c, N));
            dY[p] = d * R(fft_freq(r, N));
          }
        fft2(f, dX.data(), true, scr);
        fft2(f, dY.data(), true, scr);
        double nx = 0, dnx = 0, ny = 0, dny = 0;
        for (size_t p = 0; p < NN; ++p) {
          const cx<R> gx = dX[p] * nrm * vp[k][p], gy = dY[p] * nrm * vp[k][p];
          dnx += double(std::norm(gx));
          nx += double((chi[k][p] * std::conj(gx)).real());
          dny += double(std::norm(gy));
          ny += double((chi[k][p] * std::conj(gy)).real());
        }
        const double ddx = nx / dnx, ddy = ny / dny;
        const double shx = std::min(std::abs(ddx), 0.2) * double((0.0 < ddx) - (ddx < 0.0));
        const double shy = std::min(std::abs(ddy), 0.2) * double((0.0 < ddy) - (ddy < 0.0));
        s.pos[2 * j] = float(s.pos[2 * j] + shx);
        s.pos[2 * j + 1] = float(s.pos[2 * j + 1] + shy);
      }
    }
    if (var && iter > 2) {
      // update_variable_probe (src/Probe.cpp:1366-1516): one SVD-like step of the extra mode on the weighted
      // residual of the probe directions, then the variable-mode and intensity weights of the group's positions
      const double relaxU = double(G) / s.P;
      std::vector<double> ev(G);
      double evn = 0;
      for (int k = 0; k < G; ++k) { ev[k] = s.evo1[g[k]]; evn += ev[k] * ev[k]; }
      std::vector<cx<R>> upd(NN, cx<R>(0, 0));
      for (int k = 0; k < G; ++k) {
        const int j = g[k];
        std::vector<cx<R>> res(NN);
        double pr = 0;
        for (int x = 0; x < N; ++x)
          for (int y = 0; y < N; ++y) {
            const size_t p = size_t(x) * N + y;
            const R w = s.pobj[size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y)] / pmax;
            res[p] = (pu[k][p] - pum[p]) * w;
            pr += (double((s.E[p] * std::conj(res[p])).real()) + ev[k]) / evn;
          }
        pr /= double(NN);
        for (size_t p = 0; p < NN; ++p) upd[p] += res[p] * R(pr);
      }
      double su = 0;
      for (auto& v : upd) { v *= nrm; su += double(std::norm(v)); }
      const double un = std::sqrt(su / double(NN));
      const R us = R(relaxU / std::max(1.0, un));
      double se = 0;
      for (size_t p = 0; p < NN; ++p) { s.E[p] += upd[p] * us; se += double(std::norm(s.E[p])); }
      const R en = R(1.0 / std::sqrt(se / double(NN)));
      for (auto& v : s.E) v *= en;
      std::vector<double> den(G), num(G), dI(G), nI(G);
      double dsum = 0;
      for (int k = 0; k < G; ++k) {
        double a = 0, b = 0, c = 0, d = 0;
        for (size_t p = 0; p < NN; ++p) {
          const cx<R> v = op[k][p] * s.E[p], w = op[k][p] * s.Pr[p];
          a += double(std::norm(v));
          b += double((chi[k][p] * std::conj(v)).real());
          c += double(std::norm(w));
          d += double((chi[k][p] * std::conj(w)).real());
        }
        den[k] = a / double(NN); num[k] = b / double(NN); dI[k] = c; nI[k] = d;
        dsum += den[k];
      }
      const double dmean = dsum / G;
      for (int k = 0; k < G; ++k) {
        s.evo1[g[k]] += num[k] / (den[k] + 0.1 * dmean);
        s.evo0[g[k]] += 0.1 * nI[k] / dI[k];
      }
    }
    if (s.K > 1) mls_mode_updates(s, g, op, chm, bpr);
  }
  if (s.K > 1) mls_ortho_modes(s);
  return want_err ? errsum / s.P : 0.0;
}

// ll = 2..K of MLS::iteration's mode loop for one group (src/MLS.cpp:241-285,465-469): mode m's direction
// mean_j W chi_m conj(obj_proj) (no sub-pixel shift, no object step) with the group's LSQ probe step.
template <typename R>
void mls_mode_updates(MlsState<R>& s, const std::vector<int>& g, const std::vector<std::vector<cx<R>>>& op,
                      const std::vector<std::vector<std::vector<cx<R>>>>& chm, cx<R> bpr) {
  const int N = s.N, Y = s.geo.Y, G = int(g.size());
  const size_t NN = size_t(N) * N;
  for (int m = 1; m < s.K; ++m) {
    std::vector<cx<R>> pm(NN, cx<R>(0, 0));
    for (int k = 0; k < G; ++k) {
      const int j = g[k];
      for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
          const size_t p = size_t(x) * N + y;
          const R w0 = s.pobj[size_t(s.geo.r0[j] + x) * Y + (s.geo.c0[j] + y)];
          pm[p] += chm[m - 1][k][p] * std::conj(op[k][p]) * (w0 / (w0 + s.maxIllum * R(0.01)));
        }
    }
    cx<R>* Pm = s.Pk.data() + size_t(m - 1) * NN;
    for (size_t p = 0; p < NN; ++p) Pm[p] += bpr * (pm[p] * R(1.0 / G));
  }
}

// Position jitter (d_generateMesh, src/ScanMeshKernels.cu:53-60: jitter = r - u*2r per axis, u uniform in (0,1]
// from curand with a time seed).  Restated with a seeded stream: SplitMix64 from seed ^ 0x6A09E667F3BCC909,
// u = ((next >> 40) + 1) * 2^-24, x drawn before y, positions in generation order (padding included).
void mesh_jitter(uint64_t seed, size_t n, unsigned radius, std::vector<float>& out) {
  out.assign(2 * n, 0.f);
  if (!radius) return;
  uint64_t st = seed ^ 0x6A09E667F3BCC909ull;
  const float r = float(radius);
  for (size_t i = 0; i < 2 * n; ++i) {
    const float u = float((splitmix64(st) >> 40) + 1) * (1.0f / 16777216.0f);
    volatile float t = u * 2.0f;
    volatile float t2 = t * r;
    out[i] = r - t2;
  }
}

}  // namespace

// ============================================================================================================
// C ABI of the oracle (ctypes from tests/ and bench.py).  Complex arrays are interleaved (re, im) doubles.
// ============================================================================================================
// The scan drift of d_generateMesh (src/ScanMeshKernels.cu:86-87): `initialValues += index * driftCoeff` in float,
// metres per row (x) or column (y) of the mesh array.  The reference's compiled kernel fuses the add with the
// product that formed the value where there is one, fma(a, step, index * drift) for the Cartesian and spiral
// meshes (checked against it on the GPU), and with index * drift for a loaded value, fma(index, drift, v) (list).
static float drift_add(float v, int index, float drift) {
  return drift != 0.f ? std::fma(float(index), drift, v) : v;
}
static float drift_mul_add(float a, float step, int index, float drift) {
  if (drift == 0.f) return a * step;
  volatile float d = float(index) * drift;
  return std::fma(a, step, float(d));
}

// Raw pixel positions of an nx x ny raster before the -min shift (d_generateMesh<1>, src/ScanMeshKernels.cu:46-93,
// launched at :153-160 with one_over_dxs = (float)(1.0/dx_s)): ((i - (nx-1)/2) * stepx + i * driftx) *
// one_over_dxs in float, index i*ny + j.
static void cartesian_raw(int nx, int ny, double stepx, double stepy, double dx_s, int mirrorX, int mirrorY,
                          float dfx, float dfy, float* raw) {
  const float inv = float(1.0 / dx_s), sx = float(stepx), sy = float(stepy);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      volatile float mi = float(i), md = float(nx - 1) * 0.5f;
      volatile float dxv = mirrorX ? (md - mi) : (mi - md);
      volatile float vx = drift_mul_add(dxv, sx, i, dfx);
      volatile float mj = float(j), mdy = float(ny - 1) * 0.5f;
      volatile float dyv = mirrorY ? (mdy - mj) : (mj - mdy);
      volatile float vy = drift_mul_add(dyv, sy, j, dfy);
      volatile float px = vx * inv, py = vy * inv;
      raw[2 * (size_t(i) * ny + j)] = px;
      raw[2 * (size_t(i) * ny + j) + 1] = py;
    }
}

// The list mesh array (d_generateMesh<2>): M = ceil(P/1024)*1024 entries of 1024-wide rows, the positions in metres
// (zero past P) plus the drift of their row index / 1024 and column index % 1024, times one_over_dxs.
static void list_raw(const double* xy_m, int P, double dx_s, float dfx, float dfy, size_t M, float* raw) {
  const float inv = float(1.0 / dx_s);
  for (size_t i = 0; i < M; ++i) {
    volatile float x = i < size_t(P) ? float(xy_m[2 * i]) : 0.f, y = i < size_t(P) ? float(xy_m[2 * i + 1]) : 0.f;
    volatile float xd = drift_add(x, int(i / 1024), dfx), yd = drift_add(y, int(i % 1024), dfy);
    volatile float px = xd * inv, py = yd * inv;
    raw[2 * i] = px; raw[2 * i + 1] = py;
  }
}

// The spiral mesh array (d_generateMesh<3>): every one of the M entries is a spiral point; drift as the list's.
static void spiral_raw(double stepx, double stepy, double dx_s, float dfx, float dfy, size_t M, float* raw) {
  const float inv = float(1.0 / dx_s), sx = float(stepx), sy = float(stepy);
  for (size_t i = 0; i < M; ++i) {
    const float s = std::sqrt(float(i));
    const float a = 4.0f * s;
    const float c = float(std::cos(double(a))), sn = float(std::sin(double(a)));
    volatile float vx = s * c;
    volatile float vy = s * sn;
    volatile float wx = drift_mul_add(vx, sx, int(i / 1024), dfx), wy = drift_mul_add(vy, sy, int(i % 1024), dfy);
    volatile float px = wx * inv, py = wy * inv;
    raw[2 * i] = px; raw[2 * i + 1] = py;
  }
}

extern "C" {

int orc_version() { return 1; }

// 2-D FFT of an N x N complex array in place (unnormalised, cuFFT sign convention).
int orc_fft2(double* data, int N, int inverse) {
  if (N < 2 || (N & (N - 1))) return -1;
  Fft1<double> f(N);
  std::vector<cx<double>> a(size_t(N) * N), scr;
  for (size_t i = 0; i < a.size(); ++i) a[i] = cx<double>(data[2 * i], data[2 * i + 1]);
  fft2(f, a.data(), inverse != 0, scr);
  for (size_t i = 0; i < a.size(); ++i) { data[2 * i] = a[i].real(); data[2 * i + 1] = a[i].imag(); }
  return 0;
}

double orc_sample_pixel(double lambda, double z, double dx_d, int N) { return sample_pixel(lambda, z, dx_d, N); }

int orc_cartesian_mesh_j(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                         int mirrorX, int mirrorY, int flip, unsigned jitter, uint64_t seed, float* pos, int* objXY);
int orc_list_mesh_j(const double* xy_m, int P, double lambda, double z, double dx_d, int N, int flip, unsigned jitter,
                    uint64_t seed, float* pos, int* objXY);

// Cartesian raster mesh (d_generateMesh<1>, src/ScanMeshKernels.cu:46-93, launched at :153-160).
// pos receives 2*nx*ny floats (raster order i*ny+j), objXY the object size.
int orc_cartesian_mesh(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                       int mirrorX, int mirrorY, int flip, float* pos, int* objXY) {
  return orc_cartesian_mesh_j(nx, ny, stepx, stepy, lambda, z, dx_d, N, mirrorX, mirrorY, flip, 0, 0, pos, objXY);
}

int orc_cartesian_mesh_jd(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                          int mirrorX, int mirrorY, int flip, unsigned jitter, uint64_t seed, double driftx,
                          double drifty, float* pos, int* objXY);

int orc_cartesian_mesh_j(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                         int mirrorX, int mirrorY, int flip, unsigned jitter, uint64_t seed, float* pos,
                         int* objXY) {
  return orc_cartesian_mesh_jd(nx, ny, stepx, stepy, lambda, z, dx_d, N, mirrorX, mirrorY, flip, jitter, seed, 0.0,
                               0.0, pos, objXY);
}

// ... with the scan drift (metres per raster row / column).
int orc_cartesian_mesh_jd(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                          int mirrorX, int mirrorY, int flip, unsigned jitter, uint64_t seed, double driftx,
                          double drifty, float* pos, int* objXY) {
  if (nx < 1 || ny < 1 || N < 1) return -1;
  std::vector<float> raw(2 * size_t(nx) * ny);
  cartesian_raw(nx, ny, stepx, stepy, sample_pixel(lambda, z, dx_d, N), mirrorX, mirrorY, float(driftx),
                float(drifty), raw.data());
  std::vector<float> jit;
  mesh_jitter(seed, size_t(nx) * ny, jitter, jit);
  for (size_t k = 0; k < raw.size(); ++k) {
    volatile float v = raw[k] + jit[k];
    raw[k] = v;
  }
  Mesh m;
  finish_mesh(raw, nx * ny, false, N, flip != 0, m);
  std::memcpy(pos, m.pos.data(), m.pos.size() * sizeof(float));
  objXY[0] = m.X; objXY[1] = m.Y;
  return 0;
}

// The raw raster before the -min shift (2*nx*ny floats, raw[2*(i*ny+j)] = x, +1 = y).
int orc_cartesian_mesh_raw(int nx, int ny, double stepx, double stepy, double lambda, double z, double dx_d, int N,
                           int mirrorX, int mirrorY, float* raw) {
  if (nx < 1 || ny < 1 || N < 1) return -1;
  cartesian_raw(nx, ny, stepx, stepy, sample_pixel(lambda, z, dx_d, N), mirrorX, mirrorY, 0.f, 0.f, raw);
  return 0;
}

// Raw mesh arrays with the scan drift, before jitter and the -min shift: type 1 Cartesian (2*nx*ny floats,
// nx = a, ny = b), 2 list (xy_m in metres, P = a; 2*ceil(P/1024)*1024 floats), 3 spiral (P = a; same size).
int orc_mesh_raw_drift(int type, int a, int b, const double* xy_m, double stepx, double stepy, double lambda,
                       double z, double dx_d, int N, int mirrorX, int mirrorY, double driftx, double drifty,
                       float* raw) {
  if (a < 1 || N < 1) return -1;
  const double dx_s = sample_pixel(lambda, z, dx_d, N);
  const size_t M = (size_t(a) + 1023) / 1024 * 1024;
  if (type == 1) {
    if (b < 1) return -1;
    cartesian_raw(a, b, stepx, stepy, dx_s, mirrorX, mirrorY, float(driftx), float(drifty), raw);
  } else if (type == 2) {
    if (!xy_m) return -1;
    list_raw(xy_m, a, dx_s, float(driftx), float(drifty), M, raw);
  } else if (type == 3) {
    spiral_raw(stepx, stepy, dx_s, float(driftx), float(drifty), M, raw);
  } else {
    return -1;
  }
  return 0;
}

// List mesh from positions in metres (ListScanMesh::loadarr + d_generateMesh<2>, src/ListScanMesh.cpp:55-129).
int orc_list_mesh(const double* xy_m, int P, double lambda, double z, double dx_d, int N, int flip, float* pos,
                  int* objXY) {
  return orc_list_mesh_j(xy_m, P, lambda, z, dx_d, N, flip, 0, 0, pos, objXY);
}

// The mesh array holds whole 1024-wide rows: entries past P are (0, 0) plus their jitter and take part in the
// min/max (calculateMeshDimensions reduces over the whole array).
int orc_list_mesh_jd(const double* xy_m, int P, double lambda, double z, double dx_d, int N, int flip,
                     unsigned jitter, uint64_t seed, double driftx, double drifty, float* pos, int* objXY);

int orc_list_mesh_j(const double* xy_m, int P, double lambda, double z, double dx_d, int N, int flip, unsigned jitter,
                    uint64_t seed, float* pos, int* objXY) {
  return orc_list_mesh_jd(xy_m, P, lambda, z, dx_d, N, flip, jitter, seed, 0.0, 0.0, pos, objXY);
}

// ... with the scan drift (metres per mesh-array row / column).
int orc_list_mesh_jd(const double* xy_m, int P, double lambda, double z, double dx_d, int N, int flip,
                     unsigned jitter, uint64_t seed, double driftx, double drifty, float* pos, int* objXY) {
  if (P < 1) return -1;
  const double dx_s = sample_pixel(lambda, z, dx_d, N);
  const size_t M = (size_t(P) + 1023) / 1024 * 1024;
  std::vector<float> raw(2 * M, 0.f), jit;
  list_raw(xy_m, P, dx_s, float(driftx), float(drifty), M, raw.data());
  mesh_jitter(seed, M, jitter, jit);
  for (size_t k = 0; k < raw.size(); ++k) {
    volatile float v = raw[k] + jit[k];
    raw[k] = v;
  }
  Mesh m;
  finish_mesh(raw, int(M), false, N, flip != 0, m);
  m.pos.resize(2 * size_t(P));
  std::memcpy(pos, m.pos.data(), m.pos.size() * sizeof(float));
  objXY[0] = m.X; objXY[1] = m.Y;
  return 0;
}

// Spiral mesh (d_generateMesh<3>, src/ScanMeshKernels.cu:77-82, SpiralScanMesh::generateMesh,
// src/SpiralScanMesh.cpp:57-84): point i at sqrt(i) * (cos, sin)(4 sqrt(i)) * step / dx_s.  The mesh array holds
// whole 1024-wide rows and every entry is a spiral point, so the min/max (object size, shift) cover
// ceil(P/1024)*1024 points while only the first P are scan positions.  cos/sin of the float argument in double,
// rounded to float.
int orc_spiral_mesh_d(int P, double stepx, double stepy, double lambda, double z, double dx_d, int N, int flip,
                      unsigned jitter, uint64_t seed, double driftx, double drifty, float* pos, int* objXY);

int orc_spiral_mesh(int P, double stepx, double stepy, double lambda, double z, double dx_d, int N, int flip,
                    unsigned jitter, uint64_t seed, float* pos, int* objXY) {
  return orc_spiral_mesh_d(P, stepx, stepy, lambda, z, dx_d, N, flip, jitter, seed, 0.0, 0.0, pos, objXY);
}

// ... with the scan drift (metres per mesh-array row / column).
int orc_spiral_mesh_d(int P, double stepx, double stepy, double lambda, double z, double dx_d, int N, int flip,
                      unsigned jitter, uint64_t seed, double driftx, double drifty, float* pos, int* objXY) {
  if (P < 1 || N < 1) return -1;
  const double dx_s = sample_pixel(lambda, z, dx_d, N);
  const size_t M = (size_t(P) + 1023) / 1024 * 1024;
  std::vector<float> raw(2 * M), jit;
  mesh_jitter(seed, M, jitter, jit);
  spiral_raw(stepx, stepy, dx_s, float(driftx), float(drifty), M, raw.data());
  for (size_t k = 0; k < raw.size(); ++k) {
    volatile float v = raw[k] + jit[k];
    raw[k] = v;
  }
  Mesh m;
  finish_mesh(raw, int(M), false, N, flip != 0, m);
  m.pos.resize(2 * size_t(P));
  std::memcpy(pos, m.pos.data(), m.pos.size() * sizeof(float));
  objXY[0] = m.X; objXY[1] = m.Y;
  return 0;
}

// The jitter stream itself (2*n floats: x, y per position).
int orc_mesh_jitter(uint64_t seed, int n, unsigned radius, float* out) {
  std::vector<float> j;
  mesh_jitter(seed, size_t(n), radius, j);
  std::memcpy(out, j.data(), j.size() * sizeof(float));
  return 0;
}

// Probe guess from the mean diffraction amplitude; probe_out has K*N*N complex (modes >= 1 zero).
int orc_probe_guess(const double* amp, int P, int N, double beamSize, double dx_s, int K, double* probe_out) {
  if (P < 1 || N < 2 || (N & (N - 1)) || K < 1) return -1;
  std::vector<cx<double>> pr(size_t(K) * N * N);
  probe_guess<double>(amp, P, N, beamSize, dx_s, K, pr.data());
  for (size_t i = 0; i < pr.size(); ++i) { probe_out[2 * i] = pr[i].real(); probe_out[2 * i + 1] = pr[i].imag(); }
  return 0;
}

// The seeded visiting order: `state` is advanced in place (one stream per session).
void orc_visiting_order(uint64_t* state, int P, int* order) { visiting_order(*state, P, order); }

// Bilinear patch fetch at fractional (qx, qy) (texture emulation); obj X*Y complex, out N*N complex.
int orc_extract_patch(const double* obj, int X, int Y, float qx, float qy, int N, double* out) {
  std::vector<cx<double>> O(size_t(X) * Y), o(size_t(N) * N);
  for (size_t i = 0; i < O.size(); ++i) O[i] = cx<double>(obj[2 * i], obj[2 * i + 1]);
  extract_patch(O.data(), X, Y, qx, qy, N, o.data());
  for (size_t i = 0; i < o.size(); ++i) { out[2 * i] = o[i].real(); out[2 * i + 1] = o[i].imag(); }
  return 0;
}

// Oracle session: one reconstruction (algo 0 = ePIE, 1 = reference DM) driven one iteration at a time, so the
// flag schedule (i <= phaseConstraint, i >= updateProbe, i >= updateModes) and all cached state (|O|^2 cache,
// probe intensity cache, running maxima, DM factors, visiting-order stream) persist exactly as in a session.
// precision 0 = FP64 (the oracle proper); 1 = the same code in FP32 (used to tell FP32 rounding from logic).
}  // extern "C"

namespace {
struct OrcBase {
  virtual ~OrcBase() {}
  virtual void set_reduce(DmReduceFn fn, void* user) = 0;
  virtual void set_saturation(float level) = 0;
  virtual int step(double* err) = 0;
  virtual void get(double* obj, double* probe, double* scalars) = 0;
  virtual void psi(double* out) = 0;
};

template <typename R> struct OrcSessionT : OrcBase {
  int algo = 0, iter = 0, nthreads = 1;
  DmReduceFn reduce = nullptr;
  void* reduce_user = nullptr;
  State<R> s;
  DMState<R> d;
  Flags fl;
  uint64_t rng = 0;
  std::vector<R> amp, sq;
  std::vector<float> pos;

  int step(double* err) override {
    int status = 0;
    const int it = ++iter;
    double e = 0;
    if (algo == 0)
      e = double(epie_iteration<R>(s, amp.data(), pos.data(), sq.data(), fl, it, rng, &status, nthreads));
    else
      dm_iteration<R>(s, d, amp.data(), pos.data(), fl, it, nthreads, reduce, reduce_user);
    if (err) *err = e;
    return status;
  }
  void set_reduce(DmReduceFn fn, void* user) override {
    reduce = fn;
    reduce_user = user;
  }
  void set_saturation(float level) override { fl.saturation = level; }
  void get(double* obj, double* probe, double* scalars) override {
    store_state(s, obj, probe);
    if (scalars) {
      scalars[0] = double(s.objMax); scalars[1] = double(s.probeMax);
      scalars[2] = d.fac[0]; scalars[3] = d.fac[1];
    }
  }
  void psi(double* out) override {
    const size_t n = size_t(s.P) * s.N * s.N;
    for (size_t i = 0; i < n; ++i) {
      cx<R> v = d.psi.empty() ? cx<R>(0, 0) : d.psi[i];
      out[2 * i] = double(v.real()); out[2 * i + 1] = double(v.imag());
    }
  }
};

template <typename R>
OrcBase* make_session(int algo, int N, int K, int P, int X, int Y, const double* amp, const float* pos,
                      const double* obj, const double* probe, int probeGuessPath, int modesGiven, uint64_t seed,
                      int phaseConstraint, int updateProbe, int updateModes, int calculateRMS, int nthreads) {
  auto* h = new OrcSessionT<R>;
  h->algo = algo;
  h->nthreads = nthreads < 1 ? 1 : nthreads;
  load_state(h->s, N, K, P, X, Y, obj, probe, probeGuessPath);
  h->s.modesInitialized = modesGiven != 0;
  h->fl.phaseConstraint = phaseConstraint; h->fl.updateProbe = updateProbe; h->fl.updateModes = updateModes;
  h->fl.calculateRMS = calculateRMS;
  h->rng = seed;
  const size_t NN = size_t(N) * N;
  h->amp.resize(size_t(P) * NN);
  for (size_t i = 0; i < h->amp.size(); ++i) h->amp[i] = R(amp[i]);
  h->pos.assign(pos, pos + 2 * size_t(P));
  h->sq.assign(P, R(1));
  if (calculateRMS)  // Diffractions::fillSquaredSums: the sum of each amplitude pattern
    for (int i = 0; i < P; ++i) {
      double t = 0;
      for (size_t p = 0; p < NN; ++p) t += amp[size_t(i) * NN + p];
      h->sq[i] = R(t);
    }
  return h;
}

}  // namespace

extern "C" {

// probeGuessPath != 0: the probe came from the guess (its intensity cache and max are valid, as after
// Probe::init's normalize()); otherwise it was supplied and the cache is zero with max 1 (src/Probe.cpp:354-358).
// modesGiven != 0: modes >= 1 were supplied, so the modal switch does not re-initialise them.
void* orc_create2(int precision, int algo, int N, int K, int P, int X, int Y, const double* amp, const float* pos,
                  const double* obj, const double* probe, int probeGuessPath, int modesGiven, uint64_t seed,
                  int phaseConstraint, int updateProbe, int updateModes, int calculateRMS, int nthreads) {
  if (N < 2 || (N & (N - 1)) || K < 1 || P < 1 || X < N || Y < N) return nullptr;
  if (precision == 1)
    return make_session<float>(algo, N, K, P, X, Y, amp, pos, obj, probe, probeGuessPath, modesGiven, seed,
                               phaseConstraint, updateProbe, updateModes, calculateRMS, nthreads);
  return make_session<double>(algo, N, K, P, X, Y, amp, pos, obj, probe, probeGuessPath, modesGiven, seed,
                              phaseConstraint, updateProbe, updateModes, calculateRMS, nthreads);
}

// DM position shards: fn sums the increments over all shards in place (a host-side all-reduce); the session then
// holds its shard's patterns and positions and the whole scan's object size.
int orc_set_dm_reduce(void* h, DmReduceFn fn, void* user) {
  static_cast<OrcBase*>(h)->set_reduce(fn, user);
  return 0;
}

void* orc_create(int algo, int N, int K, int P, int X, int Y, const double* amp, const float* pos,
                 const double* obj, const double* probe, int probeGuessPath, int modesGiven, uint64_t seed,
                 int phaseConstraint, int updateProbe, int updateModes, int calculateRMS, int nthreads) {
  return orc_create2(0, algo, N, K, P, X, Y, amp, pos, obj, probe, probeGuessPath, modesGiven, seed,
                     phaseConstraint, updateProbe, updateModes, calculateRMS, nthreads);
}

// ePIE's saturation level (pixels with amplitude >= level float); +inf (the default) floats none.
int orc_set_saturation(void* h, double level) {
  static_cast<OrcBase*>(h)->set_saturation(float(level));
  return 0;
}

// Runs the next iteration; err receives the iteration's error metric (ePIE with calculateRMS; 0 for DM).
int orc_step(void* hp, double* err) { return static_cast<OrcBase*>(hp)->step(err); }

// Copies out object (X*Y complex), probe (K*N*N complex) and {objMax, probeMax, fac0, fac1}.
int orc_get(void* hp, double* obj, double* probe, double* scalars) {
  static_cast<OrcBase*>(hp)->get(obj, probe, scalars);
  return 0;
}

// DM exit-wave state (P*N*N complex); zeros before the first DM iteration.
int orc_get_psi(void* hp, double* psi) {
  static_cast<OrcBase*>(hp)->psi(psi);
  return 0;
}

void orc_destroy(void* hp) { delete static_cast<OrcBase*>(hp); }

// FP32 multithreaded DM over float inputs: the CPU baseline.  Same equations as orc_dm_run; runs `iters`
// iterations from a zero object with the given probe and returns the wall time in seconds of those iterations.
double orc_dm_baseline_f32(int N, int P, int X, int Y, const float* amp, const float* pos, const float* probe,
                           int iters, int nthreads, float* obj_out) {
  State<float> s;
  const size_t NN = size_t(N) * N, XY = size_t(X) * Y;
  s.N = N; s.K = 1; s.P = P; s.X = X; s.Y = Y;
  s.O.assign(XY, cx<float>(0, 0)); s.Ocache.assign(XY, 0.f);
  s.Pr.resize(NN); s.Pcache.assign(NN, 0.f);
  for (size_t i = 0; i < NN; ++i) s.Pr[i] = cx<float>(probe[2 * i], probe[2 * i + 1]);
  s.objMax = 0; s.probeMax = 1;
  DMState<float> d;
  Flags fl;
  auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < iters; ++it) dm_iteration<float>(s, d, amp, pos, fl, it + 1, nthreads);
  auto t1 = std::chrono::steady_clock::now();
  if (obj_out)
    for (size_t i = 0; i < XY; ++i) { obj_out[2 * i] = s.O[i].real(); obj_out[2 * i + 1] = s.O[i].imag(); }
  return std::chrono::duration<double>(t1 - t0).count();
}

// ---- MLs core oracle ----------------------------------------------------------------------------------------
// raw_pos: 2*P centred pixel positions (x, y) of the ML mesh; intens: P*N*N intensities; probe N*N complex;
// obj: object (X*Y complex, X/Y from orc_mls_geometry) or NULL for a flat start (ones).
int orc_mls_geometry(const float* raw_pos, int P, int N, int* XY, int* starts, int* roi) {
  std::vector<float> raw(raw_pos, raw_pos + 2 * size_t(P));
  MlsGeometry g = mls_geometry(raw, P, N);
  XY[0] = g.X; XY[1] = g.Y;
  for (int i = 0; i < P; ++i) { starts[2 * i] = g.r0[i]; starts[2 * i + 1] = g.c0[i]; }
  roi[0] = g.roix0; roi[1] = g.roiy0; roi[2] = g.roinx; roi[3] = g.roiny;
  return 0;
}

struct OrcMls {
  MlsState<double> s;
  uint64_t rng = 0;
};

// variable: the reference-default path (variable probe and intensity, sub-pixel shift, position search from
// iteration pps); 0 = the fixed-probe core.  The variable path's draws come from `seed` (mls_variable_draws).
// probe: K modes of N*N complex (K > 1 only on the variable path; modes 1..K-1 are initialised from mode 0).
void* orc_mls_create(const float* raw_pos, int P, int N, const double* intens, const double* probe, const double* obj,
                     uint64_t seed, double delta_p, int variable, int pps, int K) {
  auto* h = new OrcMls;
  std::vector<float> raw(raw_pos, raw_pos + 2 * size_t(P));
  h->s.geo = mls_geometry(raw, P, N);
  h->s.N = N; h->s.P = P; h->s.delta_p = delta_p;
  h->s.variable = variable != 0;
  h->s.PPS = pps;
  std::vector<double> tilts;
  h->s.K = h->s.variable ? std::max(1, K) : 1;
  if (h->s.variable) {
    mls_variable_draws(seed, N, P, h->s.K, h->s.E, tilts, h->s.evo1);
    h->s.pos = raw;
    h->s.pos_o = raw;
    h->s.sub.assign(2 * size_t(P), 0.f);
  }
  const size_t NN = size_t(N) * N, XY = size_t(h->s.geo.X) * h->s.geo.Y;
  h->s.A.resize(size_t(P) * NN);
  std::vector<double> sums(P, 0.0);
  for (int i = 0; i < P; ++i)
    for (size_t p = 0; p < NN; ++p) {
      const double v = intens[size_t(i) * NN + p];
      sums[i] += v;
      h->s.A[size_t(i) * NN + p] = std::sqrt(v);
    }
  h->s.Pr.resize(NN);
  for (size_t p = 0; p < NN; ++p) h->s.Pr[p] = cx<double>(probe[2 * p], probe[2 * p + 1]);
  if (h->s.K > 1) mls_init_modes(h->s, tilts);
  h->s.O.assign(XY, cx<double>(1, 0));
  if (obj)
    for (size_t i = 0; i < XY; ++i) h->s.O[i] = cx<double>(obj[2 * i], obj[2 * i + 1]);
  mls_setup(h->s, sums);
  h->rng = seed;
  return h;
}

int orc_mls_step(void* hp, double* err) {
  auto* h = static_cast<OrcMls*>(hp);
  const double e = mls_iteration(h->s, h->rng, err != nullptr);
  if (err) *err = e;
  return 0;
}

int orc_mls_get(void* hp, double* obj, double* probe, double* scalars) {
  auto* h = static_cast<OrcMls*>(hp);
  for (size_t i = 0; i < h->s.O.size(); ++i) { obj[2 * i] = h->s.O[i].real(); obj[2 * i + 1] = h->s.O[i].imag(); }
  for (size_t i = 0; i < h->s.Pr.size(); ++i) {
    probe[2 * i] = h->s.Pr[i].real();
    probe[2 * i + 1] = h->s.Pr[i].imag();
  }
  for (size_t i = 0; i < h->s.Pk.size(); ++i) {  // modes 1..K-1 follow mode 0
    probe[2 * (h->s.Pr.size() + i)] = h->s.Pk[i].real();
    probe[2 * (h->s.Pr.size() + i) + 1] = h->s.Pk[i].imag();
  }
  if (scalars) scalars[0] = h->s.maxIllum;
  return 0;
}

// The variable path's state: extra mode E (N*N complex), evo0 / evo1 (P each), positions (2*P, x = rows).
int orc_mls_get_var(void* hp, double* E, double* evo0, double* evo1, float* pos) {
  auto* h = static_cast<OrcMls*>(hp);
  if (!h->s.variable) return -1;
  for (size_t i = 0; i < h->s.E.size(); ++i) { E[2 * i] = h->s.E[i].real(); E[2 * i + 1] = h->s.E[i].imag(); }
  for (int i = 0; i < h->s.P; ++i) { evo0[i] = h->s.evo0[i]; evo1[i] = h->s.evo1[i]; }
  for (size_t i = 0; i < h->s.pos.size(); ++i) pos[i] = h->s.pos[i];
  return 0;
}

void orc_mls_destroy(void* hp) { delete static_cast<OrcMls*>(hp); }

// Stage entry points of the MLs helpers (n pixels; complex arrays interleaved re, im doubles).
int orc_mls_modulus_factor(const double* A, const double* ap, int n, double* out) {
  for (int i = 0; i < n; ++i) out[i] = mls_modulus_factor(A[i], ap[i]);
  return 0;
}

int orc_mls_lsq_terms(const double* chi, const double* oup, const double* dPO, const double* probe, double lam, int n,
                      double* a1, double* a2, double* a4, double* b1, double* b2) {
  auto c = [](const double* v, int i) { return cx<double>(v[2 * i], v[2 * i + 1]); };
  for (int i = 0; i < n; ++i) {
    cx<double> t;
    mls_lsq_terms(c(chi, i), c(oup, i), c(dPO, i), c(probe, i), lam, a1[i], t, a4[i], b1[i], b2[i]);
    a2[2 * i] = t.real();
    a2[2 * i + 1] = t.imag();
  }
  return 0;
}

}  // extern "C"

