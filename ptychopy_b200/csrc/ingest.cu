// Whole-mode pattern ingest (`fp` runs): the reference's file readers and per-pattern preprocessing.
//
// Files (src/FileManager.cpp:145-260, chosen by extension): `.bin` is a raw float32 stack mapped with mmap, section
// i at i*rows*cols values; `.csv` holds float values separated by commas and line breaks, read into one array,
// section i likewise.  `.h5` needs the HDF5 library, which this build does not link: refused.  The file of pattern
// i is the pattern with its '#' turned into a printf conversion, formatted with i/dpf + fs, and the section is
// i % dpf (Diffractions::load, src/Diffractions.cpp:188-209; IPhaser::initDiffractions, src/IPhaser.cpp:203-205).
// Pattern i is scan position i in raster order (the mesh's file index i*scanDimsy + j,
// src/CartesianScanMesh.cpp:83-87).
//
// Preprocessing (DiffractionLoader::run, src/DiffractionLoader.cpp:55-131), on the device, one gather kernel per
// chunk of patterns: (1) a raw rows x cols (nx x ny) pattern that is not already size x size is cropped / zero-padded
// to size x size around the centre (qx, qy) (h_symmetrizeDiffraction, src/DiffractionsKernels.cu:100-107,171-178);
// (2) rotate90 with rotate90 % 4 == 1 turns it a quarter (out[i][j] = in[j][size-1-i], d_rot90,
// src/utilitiesKernels.cu:840-851; other values leave it as it is, src/utilitiesKernels.cu:2031-2049);
// (3) fftShiftData swaps the quadrants (d_shiftX / d_shiftY, src/utilitiesKernels.cu:737-781,1945-1964).
// The kernel computes each output pixel's source through the three steps in reverse, so the chain costs one read
// and one write per pixel.  threshold and sqrtData do not transform the data on the reference's path (its
// h_preprocessDiffractions call is commented out, src/Diffractions.cpp:226-229): they set the saturation level of
// the modulus step only (updatePixelSaturation, src/Parameters.cpp:54-62), as sessions fed from numpy do.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "session.h"

namespace pty {
namespace {

// Crop / pad window of step (1): source block [dox, dox + numX) x [doy, doy + numY) lands at [oox, ...) x [ooy, ...).
struct Window {
  int direct = 0;  // the raw pattern is already size x size: copied as it is
  int dox = 0, doy = 0, oox = 0, ooy = 0, numX = 0, numY = 0;
};

// The reference's offsets (src/DiffractionLoader.cpp:86-101).  Where the centre sits less than size/2 from the top
// (left) edge the block is shifted down (right) and the reference still copies `size` rows (columns), whose tail
// falls beyond the output pattern into the next one; here those rows stay outside the pattern.
Window make_window(int rows, int cols, int S, int qx, int qy) {
  Window w;
  if (rows == S && cols == S) {
    w.direct = 1;
    return w;
  }
  int dx = qx - S / 2, dy = qy - S / 2;
  w.oox = dx < 0 ? -dx : 0;
  w.dox = dx < 0 ? 0 : dx;
  w.ooy = dy < 0 ? -dy : 0;
  w.doy = dy < 0 ? 0 : dy;
  w.numX = (qx + S / 2 < rows) ? S : rows - w.dox;
  w.numY = (qy + S / 2 < cols) ? S : cols - w.doy;
  return w;
}

// out[p][i][j] for a chunk of patterns: undo the quadrant swap, then the quarter turn, then the crop.
__global__ void k_ingest(const float* __restrict__ raw, int rows, int cols, int S, Window w, int rot, int shift,
                         float* __restrict__ out, int count) {
  const size_t SS = size_t(S) * S, n = SS * size_t(count);
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const int p = int(q / SS), k = int(q % SS);
    int i = k / S, j = k % S;
    if (shift) {  // out3[i][j] = out2[(i + S/2) % S][(j + S/2) % S]
      i = (i + S / 2) % S;
      j = (j + S / 2) % S;
    }
    if (rot) {  // out2[i][j] = out1[j][S - 1 - i]
      const int r = j, c = S - 1 - i;
      i = r;
      j = c;
    }
    float v = 0.f;
    const float* src = raw + size_t(p) * rows * cols;
    if (w.direct) {
      v = src[size_t(i) * cols + j];
    } else {
      const int r = i - w.oox, c = j - w.ooy;
      if (r >= 0 && r < w.numX && c >= 0 && c < w.numY) v = src[size_t(r + w.dox) * cols + (c + w.doy)];
    }
    out[q] = v;
  }
}

// One open data file and the sections read from it.
struct DataFile {
  virtual ~DataFile() {}
  virtual const float* section(size_t i, size_t per) = 0;
};

struct BinFile : DataFile {
  int fd = -1;
  size_t bytes = 0;
  void* map = MAP_FAILED;
  std::string path;
  explicit BinFile(const std::string& p) : path(p) {
    fd = open(p.c_str(), O_RDONLY);
    if (fd < 0) fail(PTY_ERR_IO, "cannot open the pattern file " + p);
    struct stat st;
    if (fstat(fd, &st) != 0) fail(PTY_ERR_IO, "cannot stat the pattern file " + p);
    bytes = size_t(st.st_size);
    if (bytes) map = mmap(nullptr, bytes, PROT_READ, MAP_SHARED, fd, 0);
    if (bytes && map == MAP_FAILED) fail(PTY_ERR_IO, "cannot map the pattern file " + p);
  }
  ~BinFile() override {
    if (map != MAP_FAILED) munmap(map, bytes);
    if (fd >= 0) close(fd);
  }
  const float* section(size_t i, size_t per) override {
    if ((i + 1) * per * sizeof(float) > bytes)
      fail(PTY_ERR_INVALID, path + " holds " + std::to_string(bytes / sizeof(float)) + " values, too few for section " +
                                std::to_string(i) + " of " + std::to_string(per));
    return static_cast<const float*>(map) + i * per;
  }
};

struct CsvFile : DataFile {
  std::vector<float> values;
  std::string path;
  explicit CsvFile(const std::string& p) : path(p) {
    std::ifstream f(p, std::ios::binary);
    if (!f.is_open()) fail(PTY_ERR_IO, "cannot open the pattern file " + p);
    std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    const char* c = text.c_str();
    const char* end = c + text.size();
    while (c < end) {  // numbers separated by commas, blanks and line breaks
      while (c < end && (*c == ',' || std::isspace(static_cast<unsigned char>(*c)))) ++c;
      if (c >= end) break;
      char* stop = nullptr;
      const float v = std::strtof(c, &stop);
      if (stop == c) fail(PTY_ERR_INVALID, p + ": not a number at byte " + std::to_string(c - text.c_str()));
      values.push_back(v);
      c = stop;
    }
  }
  const float* section(size_t i, size_t per) override {
    if ((i + 1) * per > values.size())
      fail(PTY_ERR_INVALID, path + " holds " + std::to_string(values.size()) + " values, too few for section " +
                                std::to_string(i) + " of " + std::to_string(per));
    return values.data() + i * per;
  }
};

std::string lower_ext(const std::string& path) {
  const size_t dot = path.find_last_of('.');
  if (dot == std::string::npos || dot == 0) fail(PTY_ERR_INVALID, "fp: no file extension in " + path);
  std::string e = path.substr(dot + 1);
  std::transform(e.begin(), e.end(), e.begin(), [](unsigned char ch) { return char(std::tolower(ch)); });
  return e;
}

// The file pattern with its '#' made a printf conversion (src/IPhaser.cpp:203-205), formatted with `index`.
std::string file_name(const std::string& pattern, unsigned index) {
  const size_t hash = pattern.find('#');
  if (hash == std::string::npos) return pattern;
  std::string fmt = pattern;
  fmt[hash] = '%';
  // the conversion after '%': flags / width digits then one integer conversion letter
  size_t k = hash + 1;
  while (k < fmt.size() && (std::isdigit(static_cast<unsigned char>(fmt[k])) || fmt[k] == '-' || fmt[k] == '0'))
    ++k;
  if (k >= fmt.size() || std::strchr("diuxX", fmt[k]) == nullptr)
    fail(PTY_ERR_INVALID, "fp: '#' must start an integer conversion such as #06d (" + pattern + ")");
  if (fmt.find('%', k + 1) != std::string::npos) fail(PTY_ERR_INVALID, "fp: '%' outside the '#' conversion");
  char buf[1024];
  const int n = std::snprintf(buf, sizeof(buf), fmt.c_str(), index);
  if (n < 0 || n >= int(sizeof(buf))) fail(PTY_ERR_INVALID, "fp: file name too long");
  return std::string(buf);
}

}  // namespace

// Reads the session's P patterns from the files of p.fp, preprocesses them on the device into s->amp.
void ingest_patterns(pty_session* s, int P) {
  const pty_params& p = s->prm;
  const int S = s->N, rows = p.nx, cols = p.ny;
  if (lower_ext(p.fp) == "h5")
    fail(PTY_ERR_UNSUPPORTED, "HDF5 pattern files need the HDF5 library, which this build does not link; "
                              "convert them to .bin (raw float32) or .csv");
  if (rows < 1 || cols < 1) fail(PTY_ERR_INVALID, "nx and ny (the raw pattern size) must be positive");
  if (p.dpf < 1) fail(PTY_ERR_INVALID, "dpf must be >= 1");
  if (p.fs < 0) fail(PTY_ERR_INVALID, "fs must be >= 0");
  const Window w = make_window(rows, cols, S, p.qx, p.qy);
  const size_t per = size_t(rows) * cols, SS = size_t(S) * S;
  s->P = P;
  s->amp.alloc(SS * P * sizeof(float), "patterns");
  // chunks of raw patterns staged in pinned memory (two buffers: the host fills one while the other uploads)
  const int chunk = int(std::max<size_t>(1, std::min<size_t>(P, (size_t(64) << 20) / (per * sizeof(float)))));
  float* stage[2] = {nullptr, nullptr};
  DeviceBuf raw;
  raw.alloc(2 * size_t(chunk) * per * sizeof(float), "raw patterns");
  cudaEvent_t done[2] = {nullptr, nullptr};
  auto cleanup = [&] {
    for (int b = 0; b < 2; ++b) {
      if (done[b]) cudaEventDestroy(done[b]);
      if (stage[b]) cudaFreeHost(stage[b]);
    }
  };
  try {
    for (int b = 0; b < 2; ++b) {
      check_cuda(cudaMallocHost(&stage[b], size_t(chunk) * per * sizeof(float)), "pinned staging");
      check_cuda(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "event");
    }
    const std::string ext = lower_ext(file_name(p.fp, unsigned(p.fs)));
    if (ext != "bin" && ext != "csv")
      fail(PTY_ERR_INVALID, "fp: valid pattern file formats are .bin, .csv (and .h5, unsupported here)");
    std::map<std::string, std::unique_ptr<DataFile>> files;
    for (int c0 = 0, b = 0; c0 < P; c0 += chunk, b ^= 1) {
      const int cnt = std::min(chunk, P - c0);
      check_cuda(cudaEventSynchronize(done[b]), "staging");
      for (int i = 0; i < cnt; ++i) {
        const int idx = c0 + i;
        const std::string name = file_name(p.fp, unsigned(idx / p.dpf + p.fs));
        auto it = files.find(name);
        if (it == files.end()) {
          files.clear();  // patterns come in file order: one file open at a time
          std::unique_ptr<DataFile> f;
          if (lower_ext(name) == "bin")
            f.reset(new BinFile(name));
          else
            f.reset(new CsvFile(name));
          it = files.emplace(name, std::move(f)).first;
        }
        std::memcpy(stage[b] + size_t(i) * per, it->second->section(size_t(idx % p.dpf), per), per * sizeof(float));
      }
      float* rd = raw.as<float>() + size_t(b) * chunk * per;
      check_cuda(cudaMemcpyAsync(rd, stage[b], size_t(cnt) * per * sizeof(float), cudaMemcpyHostToDevice, s->stream),
                 "H2D raw patterns");
      check_cuda(cudaEventRecord(done[b], s->stream), "event");
      const size_t n = SS * cnt;
      const int grid = int(std::min<size_t>((n + 255) / 256, 148 * 8));
      k_ingest<<<grid, 256, 0, s->stream>>>(rd, rows, cols, S, w, (p.rotate90 % 4) == 1 ? 1 : 0, p.fftShiftData ? 1 : 0,
                                             s->amp.as<float>() + size_t(c0) * SS, cnt);
      check_cuda(cudaGetLastError(), "ingest kernel");
      s->launches += 1;
    }
    check_cuda(cudaStreamSynchronize(s->stream), "ingest");
  } catch (...) {
    cudaStreamSynchronize(s->stream);
    cleanup();
    throw;
  }
  cleanup();
  s->have_patterns = true;
}

}  // namespace pty

// Preprocessing of patterns already in device memory, for the parity tests: `count` raw rows x cols float32 patterns
// (raw_dev) into size x size patterns (out_dev) with the crop centre (qx, qy), rotate90 and fftShiftData as above.
extern "C" int pty_preprocess_patterns(const float* raw_dev, int count, int rows, int cols, int size, int qx, int qy,
                                       int rotate90, int fftShift, float* out_dev, void* stream) {
  using namespace pty;
  if (!raw_dev || !out_dev || count < 1 || rows < 1 || cols < 1 || size < 1) return PTY_ERR_INVALID;
  const Window w = make_window(rows, cols, size, qx, qy);
  const size_t n = size_t(size) * size * count;
  const int grid = int(std::min<size_t>((n + 255) / 256, 148 * 8));
  k_ingest<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(raw_dev, rows, cols, size, w, (rotate90 % 4) == 1 ? 1 : 0,
                                                                 fftShift ? 1 : 0, out_dev, count);
  return cudaGetLastError() == cudaSuccess ? PTY_OK : PTY_ERR_CUDA;
}
