// Command-line strings of the reference's `ptycho` program, as its CPython module hands them over
// (epiecmdstr / dmcmdstr / mlscmdstr / epieinit / mlsinit, src/ptychopy.c:578-689,902-1024), turned into a
// pty_params.  Host code only.
//
// What the reference does (src/ptychopy.c:543-576, src/Parameters.cpp:66-375, defaults src/Parameters.h:67-170):
//   * the string is split at white space; the first token is the program name and is skipped;
//   * a token "-name=value" (any number of leading dashes) sets `name`; a bare "-name" is a flag;
//   * integer values go through atoi, real values through atof, and each option keeps its own range check
//     (size >= 32, i >= 0, dpf >= 1, ...): a value out of range leaves the default;
//   * options absent from the string keep the command line's defaults, which differ from the Python keywords'
//     (beamSize 1e-7, lambda 2.48e-10, z 1, scanDims 12 x 12, size 256, PPS 5, ...).
// Deliberate differences (bugs or process-wide state there):
//   * names match exactly (case-insensitive); the reference's value lookup matches by prefix, so "-threshold=5"
//     after "-T=60" would reset T;
//   * "-step=v" with one value reads it as a real number (the reference truncates it with atoi);
//   * "-T=t" (the wall-time limit) keeps whole seconds, the limit pty_params holds;
//   * each call starts from the defaults (the reference's parameter singleton keeps what earlier calls set);
//   * a `bitDepth` above 32 is refused (the reference's 64-bit saturation level would overflow past 63).  Options
//     with no effect on a reconstruction here are accepted and ignored, as the reference ignores
//     names it does not know: blind (unused there), threads (file-reading threads), angles, overlap,
//     shareFrequency (multi-GPU stitching), updateVis, wsServerUrl (rendering).
#include <cctype>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <strings.h>
#include <vector>

#include "../../include/ptychopy_b200.h"

namespace pty {
void set_last_error(const std::string& msg);
}

namespace {

struct Option {
  std::string name, value;  // a bare "-name" has an empty value
};

// Whitespace-separated tokens after the program name.
std::vector<Option> split_options(const char* s) {
  std::vector<std::string> tokens;
  std::string cur;
  for (const char* c = s; *c; ++c) {
    if (std::isspace(static_cast<unsigned char>(*c))) {
      if (!cur.empty()) tokens.push_back(cur);
      cur.clear();
    } else {
      cur += *c;
    }
  }
  if (!cur.empty()) tokens.push_back(cur);
  std::vector<Option> out;
  for (size_t i = 1; i < tokens.size(); ++i) {
    const std::string& t = tokens[i];
    size_t start = 0;
    while (start < t.size() && t[start] == '-') ++start;
    Option o;
    const size_t eq = t.find('=', start);
    if (eq == std::string::npos) {
      o.name = t.substr(start);
    } else {
      o.name = t.substr(start, eq - start);
      o.value = t.substr(eq + 1);
    }
    out.push_back(o);
  }
  return out;
}

// atoi's reading (leading blanks, a sign, the digits up to the first other character; 0 when there are none),
// clamped to the int range where atoi's result would be undefined.
int to_int(const char* s) {
  const long long v = std::strtoll(s, nullptr, 10);
  if (v > INT_MAX) return INT_MAX;
  if (v < INT_MIN) return INT_MIN;
  return int(v);
}

struct Options {
  std::vector<Option> all;
  // The last occurrence of `name`, or nullptr.
  const Option* find(const char* name) const {
    const Option* hit = nullptr;
    for (const Option& o : all)
      if (strcasecmp(o.name.c_str(), name) == 0) hit = &o;
    return hit;
  }
  bool integer(const char* name, int* v) const {
    const Option* o = find(name);
    if (!o) return false;
    *v = to_int(o->value.c_str());  // a bare flag reads as 0, like the reference's integer lookup
    return true;
  }
  bool real(const char* name, double* v) const {
    const Option* o = find(name);
    if (!o) return false;
    *v = std::atof(o->value.c_str());
    return true;
  }
  // "a,b" into two values (a single value fills the first, and the second too or `second_default`).
  template <typename T, typename Conv>
  bool pair(const char* name, T* a, T* b, bool single_fills_both, T second_default, Conv conv) const {
    const Option* o = find(name);
    if (!o) return false;
    const std::string& v = o->value;
    const size_t comma = v.find(',');
    if (comma == std::string::npos) {
      *a = conv(v.c_str());
      *b = single_fills_both ? *a : second_default;
    } else {
      *a = conv(v.substr(0, comma).c_str());
      *b = conv(v.substr(comma + 1).c_str());
    }
    return true;
  }
};

struct Refusal {
  int code;
  std::string msg;
};

void text(const Options& opt, const char* name, char* dst, size_t cap) {
  const Option* o = opt.find(name);
  if (!o) return;
  if (o->value.size() >= cap)
    throw Refusal{PTY_ERR_INVALID, std::string(name) + " is longer than " + std::to_string(cap - 1) + " characters"};
  std::memcpy(dst, o->value.c_str(), o->value.size() + 1);
}

// The command line's defaults (src/Parameters.h:67-170); what the two front ends share comes from pty_params_init.
void command_line_defaults(pty_params* p) {
  pty_params_init(p);
  std::strcpy(p->hdf5path, "/entry/data/data");
  p->beamSize = 1e-7;
  p->lambd = 2.48e-10;
  p->dx_d = 172e-6;
  p->z = 1.0;
  p->scanDimsx = 12;
  p->scanDimsy = 12;
  p->stepx = 40e-9;
  p->stepy = 40e-9;
  p->size = 256;
  p->qx = 128;
  p->qy = 128;
  p->nx = 256;
  p->ny = 256;
  p->iter = 100;
  p->PPS = 5;
  p->delta_p = 0.1;
  p->save = 0;  // the reference's 999999: never within a run
  p->T = 0;     // the reference's -1: no time limit
}

void apply(const Options& opt, pty_params* p) {
  int v = 0;
  double d = 0;
  if (opt.find("sqrtData")) p->sqrtData = 1;
  if (opt.find("fftShiftData")) p->fftShiftData = 1;
  if (opt.integer("beamstopMask", &v)) p->beamstopMask = v > 0;
  if (opt.integer("simulate", &v)) p->simulate = v > 0;
  if (opt.integer("spiralScan", &v)) p->spiralScan = v > 0;
  if (opt.integer("bitDepth", &v) && v >= 1) {
    if (v > 32) throw Refusal{PTY_ERR_INVALID, "bitDepth " + std::to_string(v) + " is above 32"};
    p->bitDepth = v;
  }
  if (opt.integer("flipScanAxis", &v)) p->flipScanAxis = v > 0;
  if (opt.integer("mirror1stScanAxis", &v)) p->mirror1stScanAxis = v > 0;
  if (opt.integer("mirror2ndScanAxis", &v)) p->mirror2ndScanAxis = v > 0;
  if (opt.integer("RMS", &v)) p->calculateRMS = v > 0;
  if (opt.integer("binaryOutput", &v)) p->binaryOutput = v > 0;
  if (opt.integer("i", &v) && v >= 0) p->iter = v;
  if (opt.integer("save", &v) && v > 0) p->save = v;
  if (opt.real("T", &d)) p->T = d >= double(INT_MAX) ? INT_MAX : d > 0 ? int(d) : 0;
  if (opt.integer("size", &v) && v >= 32) p->size = v;
  if (opt.integer("PPS", &v) && v >= 1) p->PPS = v;
  if (opt.integer("probeModes", &v) && v >= 1) p->probeModes = v;
  if (opt.integer("fs", &v) && v >= 0) p->fs = v;
  if (opt.integer("dpf", &v) && v >= 1) p->dpf = v;
  if (opt.integer("threshold", &v) && v >= 0) p->threshold = v;
  if (opt.integer("jitterRadius", &v) && v >= 0) p->jitterRadius = v;
  if (opt.integer("rotate90", &v) && v >= 0) p->rotate90 = v;
  if (opt.integer("updateProbe", &v) && v >= 0) p->updateProbe = v;
  if (opt.integer("updateModes", &v) && v >= 0) p->updateModes = v;
  if (opt.integer("phaseConstraint", &v) && v >= 0) p->phaseConstraint = v;
  text(opt, "fp", p->fp, sizeof(p->fp));
  text(opt, "hdf5path", p->hdf5path, sizeof(p->hdf5path));
  auto to_real = [](const char* s) { return std::atof(s); };
  opt.pair("scanDims", &p->scanDimsx, &p->scanDimsy, false, 1, to_int);
  // one value without a comma fills both components: the reference reads the second from substr(npos + 1), i.e. from
  // the start of the value again (src/Parameters.cpp:279-304)
  opt.pair("drift", &p->driftx, &p->drifty, true, 0.0, to_real);
  opt.pair("qxy", &p->qx, &p->qy, true, 0, to_int);
  opt.pair("nxy", &p->nx, &p->ny, true, 0, to_int);
  opt.pair("step", &p->stepx, &p->stepy, true, 0.0, to_real);
  opt.real("beamSize", &p->beamSize);
  opt.real("lambda", &p->lambd);
  opt.real("dx_d", &p->dx_d);
  opt.real("z", &p->z);
  text(opt, "jobID", p->jobID, sizeof(p->jobID));
  text(opt, "algorithm", p->algorithm, sizeof(p->algorithm));
  text(opt, "lf", p->lf, sizeof(p->lf));
  text(opt, "probeGuess", p->probeGuess, sizeof(p->probeGuess));
  text(opt, "objectGuess", p->objectGuess, sizeof(p->objectGuess));
}

}  // namespace

extern "C" int pty_params_from_cmdline(const char* cmdstr, pty_params* p) {
  if (!p || !cmdstr) {
    pty::set_last_error("pty_params_from_cmdline: null argument");
    return PTY_ERR_INVALID;
  }
  pty_params q;
  command_line_defaults(&q);
  try {
    apply(Options{split_options(cmdstr)}, &q);
  } catch (const Refusal& r) {
    pty::set_last_error(r.msg);
    return r.code;
  } catch (const std::bad_alloc&) {
    pty::set_last_error("host allocation failed");
    return PTY_ERR_OOM;
  }
  *p = q;
  pty::set_last_error("");
  return PTY_OK;
}
