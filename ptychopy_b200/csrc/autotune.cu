// Autotuner: before a session's pty_init, times the launch variants of its algorithm on temporary sessions with the
// same parameters, positions, probe, object and patterns (the patterns are shared through their device copy) and
// keeps the fastest for the session: the DM wave size (patterns per pass of the three DM kernels, i.e. how much of the
// W1 / W2 hand-off stays in L2 against how often the kernels drain) and the number of waves in flight (one lane, or
// two alternating streams), and the ePIE kernel (shared-memory cluster, cluster of global-memory phases, the
// whole-GPU cooperative kernel, or the per-position kernel chain, whose transform passes also come with 2, 4 or 8
// rows per CTA).  No counterpart in the reference, which has
// one fixed launch configuration per kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ptychopy_b200.h"
#include "kernels.h"
#include "kernels_epie.h"
#include "session.h"

namespace pty {
void set_last_error(const std::string& msg);  // session.cu

namespace {

struct Candidate {
  int wave = 0;      // DM
  int variant = -1;  // ePIE
  std::string name;
  int lanes = 0;     // DM: 0 automatic, 1 one lane
  int rows = 0;      // ePIE kernel chain: rows per CTA of its transform passes (0 automatic)
};

// GPU time per iteration (ms) of one candidate: a temporary session, `iters` warm-up iterations, `iters` timed
double time_candidate(const pty_session* s, const Candidate& c, int iters) {
  pty_params p = s->prm;
  p.wave = c.wave;
  // time the steady state: the probe (and, with several modes, the modes) update from the first iteration, as they
  // do for most of a run (from updateProbe = 10 and updateModes = 20 of 100 by default)
  p.updateProbe = std::min(p.updateProbe, 1);
  p.updateModes = std::min(p.updateModes, 1);
  p.phaseConstraint = 0;  // one schedule regime throughout: graphs captured in the warm-up replay in the timed part
  pty_session* t = nullptr;
  if (pty_session_create(&p, &t) != PTY_OK) return -1.0;
  double ms = -1.0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  do {
    t->epie_variant = c.variant;
    t->dm_lanes_req = c.lanes;
    t->fft_rows = c.rows;
    if (pty_set_patterns(t, s->amp.p, PTY_F32, s->P, s->N) != PTY_OK) break;
    if (!s->pos_m.empty() && pty_set_positions(t, s->pos_m.data(), int(s->pos_m.size() / 2)) != PTY_OK) break;
    if (!s->probe_h.empty() &&
        pty_set_probe(t, s->probe_h.data(), s->probe_given_modes, s->N) != PTY_OK)
      break;
    if (!s->obj_h.empty() && pty_set_object(t, s->obj_h.data(), s->X, s->Y) != PTY_OK) break;
    if (pty_init(t) != PTY_OK) break;
    bool ok = true;
    for (int i = 0; i < iters && ok; ++i) ok = pty_step(t, nullptr) == PTY_OK;
    if (!ok || cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) break;
    cudaEventRecord(e0, t->stream);
    for (int i = 0; i < iters && ok; ++i) ok = pty_step(t, nullptr) == PTY_OK;
    cudaEventRecord(e1, t->stream);
    if (!ok || cudaEventSynchronize(e1) != cudaSuccess) break;
    float f = 0.f;
    cudaEventElapsedTime(&f, e0, e1);
    ms = double(f) / iters;
  } while (false);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  pty_session_destroy(t);
  return ms;
}

}  // namespace
}  // namespace pty

using namespace pty;

extern "C" int pty_autotune(pty_session* s, int iters, char* report, int report_len) {
  if (!s || iters < 1) {
    set_last_error("pty_autotune: bad argument");
    return PTY_ERR_INVALID;
  }
  if (s->initialized) {
    set_last_error("pty_autotune runs before pty_init");
    return PTY_ERR_STATE;
  }
  if (!s->have_patterns) {
    set_last_error("pty_autotune: set the patterns first");
    return PTY_ERR_STATE;
  }
  std::vector<Candidate> cands;
  const int P = s->P, N = s->N;
  if (s->algo == ALGO_DM) {
    std::vector<int> waves = {0};
    const size_t limit = size_t(2) << 30;  // W1 + W2 of a wave at most 2 GiB
    const int automatic = dm_wave_size(N, P);
    for (int d : {1, 2, 3, 4, 6, 8, 12}) {
      const int w = (P + d - 1) / d;
      if (w >= 1 && w != automatic && 2 * size_t(w) * N * N * 8 <= limit) waves.push_back(w);
    }
    std::sort(waves.begin() + 1, waves.end());
    waves.erase(std::unique(waves.begin() + 1, waves.end()), waves.end());
    for (int lanes : {0, 1})
      for (int w : waves) {
        const int wv = w ? w : automatic;
        if (lanes == 1 && (P + wv - 1) / wv < 2) continue;  // a single wave runs on one lane anyway
        Candidate c;
        c.wave = w;
        c.lanes = lanes;
        c.name = (w ? "wave " + std::to_string(w) : "wave " + std::to_string(automatic) + " (automatic)") +
                 (lanes == 1 ? " one lane" : "");
        cands.push_back(c);
      }
  } else if (s->algo == ALGO_EPIE) {
    if (epie_uses_smem(N, s->K)) cands.push_back({0, 0, "shared-memory cluster"});
    cands.push_back({0, 1, "cluster"});
    if (N == 256 || N == 512) cands.push_back({0, 2, "whole-GPU"});
    cands.push_back({0, 3, "kernel chain"});
    // the chain's transform passes with other row tiles (rows per CTA; 4 is the automatic tile at 512^2)
    for (int r : {2, 4, 8}) {
      if (N == 512 && r == 4) continue;
      Candidate c{0, 3, "kernel chain, " + std::to_string(r) + "-row FFT tiles"};
      c.rows = r;
      cands.push_back(c);
    }
  }
  std::string rep = s->algo == ALGO_DM ? "DM" : (s->algo == ALGO_EPIE ? "ePIE" : "MLs");
  int best = -1;
  double best_ms = 0.0;
  // two interleaved rounds, the faster of each candidate's two timings: the first candidate timed otherwise carries
  // the process's first-use costs
  std::vector<double> times(cands.size(), -1.0);
  for (int round = 0; round < 2; ++round)
    for (size_t i = 0; i < cands.size(); ++i) {
      const double t = time_candidate(s, cands[i], iters);
      if (t > 0.0 && (times[i] < 0.0 || t < times[i])) times[i] = t;
    }
  for (size_t i = 0; i < cands.size(); ++i)
    if (times[i] > 0.0 && (best < 0 || times[i] < best_ms)) {
      best = int(i);
      best_ms = times[i];
    }
  if (cands.empty()) {
    rep += ": no launch variants to tune";
  } else if (best < 0) {
    set_last_error("pty_autotune: no candidate ran");
    return PTY_ERR_CUDA;
  } else {
    if (s->algo == ALGO_DM) {
      s->prm.wave = cands[best].wave;
      s->dm_lanes_req = cands[best].lanes;
    } else {
      s->epie_variant = cands[best].variant;
      s->fft_rows = cands[best].rows;
    }
    char buf[96];
    std::snprintf(buf, sizeof(buf), ": %s (%.3f ms/iteration);", cands[best].name.c_str(), best_ms);
    rep += buf;
    for (size_t i = 0; i < cands.size(); ++i) {
      std::snprintf(buf, sizeof(buf), " %s %.3f", cands[i].name.c_str(), times[i]);
      rep += buf;
    }
  }
  cudaGetLastError();
  if (report && report_len > 0) {
    std::strncpy(report, rep.c_str(), size_t(report_len) - 1);
    report[report_len - 1] = 0;
  }
  return PTY_OK;
}
