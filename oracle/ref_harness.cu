// Launch wrappers around the reference's own device functions (extracted unchanged by oracle/ref_build.py).
// TEST INFRASTRUCTURE ONLY: the GPU stage tests call these through ctypes with device pointers and compare the
// results with the matching stages of the FP64 oracle.  Nothing in the product loads this library.
//
// Every wrapper launches the reference code the way the reference's host code does (same grid and block shape,
// same arguments; the launcher is cited beside each), synchronises and returns the CUDA error code (0 = success).
// Layouts follow the reference: row-major, pitched rows (alignedY = alignUp(Y, 32) complex or real elements).
// Several of the reference's kernels bound-check only one index or hold a __syncthreads() inside a condition, so
// each wrapper first refuses shapes for which the reference launch would index outside its buffers or diverge at
// a barrier (returns cudaErrorInvalidValue without launching): square power-of-two sizes from 32 to 1024.
#include "ref_shim.cuh"

#include REF_EXTRACT

#include <cstdio>
#include <cstring>

namespace {

constexpr unsigned kMaxThreads = 1024;  // GPUQuery::getGPUMaxThreads() on sm_100

bool pow2_window(int n) { return n >= 32 && n <= 1024 && (n & (n - 1)) == 0; }
unsigned align32(unsigned n) { return (n + 31u) / 32u * 32u; }
unsigned div_up(unsigned a, unsigned b) { return (a + b - 1) / b; }

int finish() {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return int(e);
}

// calcGrids (src/utilities.h:515-532) for alignedY <= 1024: block (alignedY, 1024/alignedY), grid rows/slice.
void calc_grids(unsigned x, unsigned alignedY, dim3& grid, dim3& block) {
  const unsigned slice = kMaxThreads / alignedY;
  grid = dim3(div_up(x, slice), 1, 1);
  block = dim3(alignedY, slice, 1);
}

// One texture object over the pitched object array, as h_bindObjArrayToTex (src/SampleKernels.cu:493-502) binds
// its texture reference: clamp addressing on both axes, linear filtering, unnormalised coordinates,
// width = Y (columns), height = X (rows), pitch alignedY complex.
int bind_object(const float2* obj, unsigned X, unsigned Y, unsigned alignedY, cudaTextureObject_t* out) {
  cudaResourceDesc rd;
  std::memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypePitch2D;
  rd.res.pitch2D.devPtr = const_cast<float2*>(obj);
  rd.res.pitch2D.desc = cudaCreateChannelDesc<float2>();
  rd.res.pitch2D.width = Y;
  rd.res.pitch2D.height = X;
  rd.res.pitch2D.pitchInBytes = size_t(alignedY) * sizeof(float2);
  cudaTextureDesc td;
  std::memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeClamp;
  td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaError_t e = cudaCreateTextureObject(out, &rd, &td, nullptr);
  if (e != cudaSuccess) return int(e);
  return int(cudaMemcpyToSymbol(g_objArrayTex, out, sizeof(*out)));
}

// ---- DM callbacks, called per element the way cuFFT calls them (callerInfo = the DM_info, offset = the
// element's index in the batched buffer).
__global__ void k_call_calc_psi(const DM_info info, float2* psi, float2* out, size_t n) {
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    DM_info a = info;
    out[q] = d_calculatePsi(psi, q, &a, nullptr);
  }
}

__global__ void k_call_modulus(const DM_info info, const float2* Psi, float2* out, size_t n) {
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    DM_info a = info;
    d_modulusConstraint(out, q, Psi[q], &a, nullptr);
  }
}

// The store callback adds each position's object and probe increments with atomics while other positions still
// read O and P, so its combined result depends on timing.  Here every position p gets its own copy of the
// iteration's starting object and probe (objCopies + p*objStride, probeCopies + p*N*N): the unchanged callback
// then runs exactly as for a single position, and the caller sums the copies' changes.
__global__ void k_call_update(const DM_info info, const float2* Pf, float2* out, float2* objCopies, size_t objStride,
                              float2* probeCopies, size_t NN, size_t n) {
  for (size_t q = blockIdx.x * size_t(blockDim.x) + threadIdx.x; q < n; q += size_t(gridDim.x) * blockDim.x) {
    const size_t p = q / NN;
    DM_info a = info;
    a.d_objectArray = objCopies + p * objStride;
    a.d_probe = probeCopies + p * NN;
    d_updateObject(out, q, Pf[q], &a, nullptr);
  }
}

DM_info dm_info(float2* obj, float2* probe, float2* psi, const float* A, const float2* pos, const bool* flags,
                const float* factors, unsigned P, unsigned N, unsigned X, unsigned Y, unsigned alignedY) {
  return DM_info(obj, probe, psi, A, pos, flags, factors, P, 1, N, N, N, X, Y, alignedY);
}

int grid_for(size_t n) { return int(n / 256 + 1 < 4096 ? n / 256 + 1 : 4096); }

}  // namespace

extern "C" {

int ref_version() { return 1; }

// d_calculatePsi (src/SampleKernels.cu:418-433) over P patterns: out = 2 P O - psi at rounded positions.
int ref_dm_calc_psi(float2* psi, float2* obj, float2* probe, const float2* pos, int P, int N, int X, int Y,
                    int alignedY, float2* out) {
  if (!pow2_window(N) || P < 1) return int(cudaErrorInvalidValue);
  const DM_info info = dm_info(obj, probe, psi, nullptr, pos, nullptr, nullptr, P, N, X, Y, alignedY);
  const size_t n = size_t(P) * N * N;
  k_call_calc_psi<<<grid_for(n), 256>>>(info, psi, out, n);
  return finish();
}

// d_modulusConstraint (src/SampleKernels.cu:436-448): out = A exp(i arg Psi) / N^2.
int ref_dm_modulus(const float2* Psi, const float* A, int P, int N, float2* out) {
  if (!pow2_window(N) || P < 1) return int(cudaErrorInvalidValue);
  const DM_info info = dm_info(nullptr, nullptr, nullptr, A, nullptr, nullptr, nullptr, P, N, N, N, N);
  const size_t n = size_t(P) * N * N;
  k_call_modulus<<<grid_for(n), 256>>>(info, Psi, out, n);
  return finish();
}

// d_updateObject (src/SampleKernels.cu:452-488) with per-position object / probe copies (see k_call_update).
// psi (P*N*N) is the persistent exit-wave state, updated in place; out receives the same values (dataOut).
// flags[2] = {phase constraint, probe update}; factors[2] = {1/objMax, 1/probeMax} (m_factors, src/DM.cu:95-98).
int ref_dm_update(const float2* Pf, float2* psi, float2* objCopies, float2* probeCopies, const float2* pos,
                  const bool* flags, const float* factors, int P, int N, int X, int Y, int alignedY, float2* out) {
  if (!pow2_window(N) || P < 1 || alignedY < Y) return int(cudaErrorInvalidValue);
  const DM_info info = dm_info(objCopies, probeCopies, psi, nullptr, pos, flags, factors, P, N, X, Y, alignedY);
  const size_t n = size_t(P) * N * N, NN = size_t(N) * N;
  k_call_update<<<grid_for(n), 256>>>(info, Pf, out, objCopies, size_t(X) * alignedY, probeCopies, NN, n);
  return finish();
}

// h_extractObjectArray (src/SampleKernels.cu:563-571): the bilinear texture gather of an N x N patch at (qx, qy).
int ref_extract_patch(const float2* obj, int X, int Y, int alignedY, float qx, float qy, int N, float2* out) {
  if (!pow2_window(N) || alignedY < Y) return int(cudaErrorInvalidValue);
  cudaTextureObject_t tex = 0;
  int rc = bind_object(obj, X, Y, alignedY, &tex);
  if (rc) return rc;
  dim3 grid, block;
  calc_grids(N, N, grid, block);
  d_extractObjectArray<true><<<grid, block>>>(obj, out, N, N, qx, qy, N, alignedY);
  rc = finish();
  cudaDestroyTextureObject(tex);
  return rc;
}

// h_simulatePSI (src/SampleKernels.cu:530-540): psi = texture(O)(patch at (qx, qy)) * probe.
int ref_simulate_psi(const float2* obj, int X, int Y, int alignedY, const float2* probe, float qx, float qy, int N,
                     float2* out) {
  if (!pow2_window(N) || alignedY < Y || X < N || Y < N) return int(cudaErrorInvalidValue);
  cudaTextureObject_t tex = 0;
  int rc = bind_object(obj, X, Y, alignedY, &tex);
  if (rc) return rc;
  const unsigned slice = kMaxThreads / N;
  // d_simulatePSI bounds its rows by the object's height, so rows beyond N would write past `out`: the grid
  // covers exactly N rows (N is a multiple of the slice for power-of-two N).
  d_simulatePSI<<<dim3(N / slice), dim3(N, slice)>>>(obj, probe, out, qx, qy, N, X, Y, alignedY);
  rc = finish();
  cudaDestroyTextureObject(tex);
  return rc;
}

// h_adjustFFT (src/utilitiesKernels.cu:1866-1877): modulus projection of K stacked modes against one amplitude
// pattern (d_adjustFFT for K = 1, d_adjustModalFFT otherwise), normalised by 1/N^2.  mask may be null.
int ref_adjust_fft(const float2* psi, float2* out, const float* detmod, const float* mask, float saturation, int K,
                   int N) {
  if (!pow2_window(N) || K < 1) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  const dim3 grid(div_up(N, slice)), block(N, slice);
  const float nrm = 1.0f / float(N * N);
  if (K > 1)
    d_adjustModalFFT<<<grid, block>>>(psi, out, detmod, mask, saturation, K, N, N, nrm);
  else
    d_adjustFFT<<<grid, block>>>(psi, out, detmod, mask, saturation, N, nrm);
  return finish();
}

// h_updateObjectArray (src/SampleKernels.cu:591-617): object update under the patch at integer (offX, offY) with
// factor c = 1/probeMax, |O|^2 cache written under the patch.
int ref_update_object(float2* obj, const float2* probe, const float2* psi, const float2* psi_old, float* intens,
                      int offX, int offY, float c, int K, int N, int X, int Y, int alignedY, int phaseConstraint) {
  if (!pow2_window(N) || K < 1 || offX < 0 || offY < 0 || offX + N > X || offY + N > Y || alignedY < Y)
    return int(cudaErrorInvalidValue);
  const unsigned rx = X / 2 - N / 2, ry = Y / 2 - N / 2;
  if (phaseConstraint) {
    if (K > 1)
      d_updateObjectArrayM<true><<<N, N>>>(obj, probe, psi, psi_old, intens, offX, offY, rx, ry, c, K, N, alignedY);
    else
      d_updateObjectArray<true><<<N, N>>>(obj, probe, psi, psi_old, intens, offX, offY, rx, ry, c, N, alignedY);
  } else {
    if (K > 1)
      d_updateObjectArrayM<false><<<N, N>>>(obj, probe, psi, psi_old, intens, offX, offY, rx, ry, c, K, N, alignedY);
    else
      d_updateObjectArray<false><<<N, N>>>(obj, probe, psi, psi_old, intens, offX, offY, rx, ry, c, N, alignedY);
  }
  return finish();
}

// h_updateProbe (src/ProbeKernels.cu:742-754): probe update from the updated object, c = 1/objMax, |P_k|^2 cache.
int ref_update_probe(float2* probe, const float2* obj, const float2* psi, const float2* psi_old, float* intens,
                     int offX, int offY, float c, int K, int N, int X, int Y, int alignedY) {
  if (!pow2_window(N) || K < 1 || offX < 0 || offY < 0 || offX + N > X || offY + N > Y || alignedY < Y)
    return int(cudaErrorInvalidValue);
  if (K > 1)
    d_updateProbeM<<<N, N>>>(probe, obj, psi, psi_old, intens, offX, offY, c, K, N, alignedY);
  else
    d_updateProbe<<<N, N>>>(probe, obj, psi, psi_old, intens, offX, offY, c, N, alignedY);
  return finish();
}

// h_calculateER (src/utilitiesKernels.cu:1879-1925) without its final thrust::reduce: partial[row] receives the
// block sum sum_col |A - |sum_k Psi_k|| of each row (the caller sums the N partials and divides by K).
int ref_calculate_er(const float2* Psi, const float* detmod, int K, int N, float* partial) {
  if (!pow2_window(N) || K < 1) return int(cudaErrorInvalidValue);
  const unsigned threads = N;  // getReductionThreadNum(N) for power-of-two N, <= 1024
  const size_t shm = threads <= 32 ? 2 * threads * sizeof(real_t) : threads * sizeof(real_t);
  switch (threads) {
    case 32: d_calculateER<32><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    case 64: d_calculateER<64><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    case 128: d_calculateER<128><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    case 256: d_calculateER<256><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    case 512: d_calculateER<512><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    case 1024: d_calculateER<1024><<<N, threads, shm>>>(Psi, detmod, partial, N, N, N, K, true); break;
    default: return int(cudaErrorInvalidValue);
  }
  return finish();
}

// h_get_optimal_step_lsq (src/utilitiesKernels.cu:1610-1621): the per-pixel terms of the MLs 2x2 step system.
int ref_lsq_terms(float2* chi, float2* oup, float2* dPO, float2* probe, float lambda, int N, float* AA1, float2* AA2,
                  float* AA4, float* Atb1, float* Atb2) {
  if (!pow2_window(N)) return int(cudaErrorInvalidValue);
  dim3 grid, block;
  calc_grids(N, N, grid, block);
  d_get_optimal_step_lsq<true><<<grid, block>>>(chi, oup, dPO, probe, lambda, AA1, AA2, AA4, Atb1, Atb2, N, N, N);
  return finish();
}

// h_modulus_amplitude (src/DiffractionsKernels.cu:200-208): result = modF / (aPsi + 1e-9) - R_offset.
int ref_modulus_amplitude(float* modF, float* aPsi, float* result, float R_offset, int N) {
  if (!pow2_window(N)) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  d_modulus_amplitude<<<dim3(div_up(N, slice)), dim3(N, slice)>>>(modF, aPsi, result, R_offset, N, N, N);
  return finish();
}

// h_generateCartesianMesh (src/ScanMeshKernels.cu:153-160) without jitter or drift: raw pixel positions of an
// nx x ny raster in a pitched array (row i at i*alignUp(ny, 32)).  one_over_dxs = (float)(1.0/dx_s).
int ref_cartesian_mesh(float2* pos, int nx, int ny, float stepx, float stepy, float one_over_dxs, int mirrorX,
                       int mirrorY) {
  if (nx < 1 || ny < 1 || ny > 1024) return int(cudaErrorInvalidValue);
  d_generateMesh<1><<<nx, align32(ny)>>>(pos, ny, stepx, stepy, one_over_dxs, 0, mirrorX != 0, mirrorY != 0, nullptr,
                                         make_float2(0.f, 0.f));
  return finish();
}

// d_generateMesh<type> (src/ScanMeshKernels.cu:46-93) with a scan drift, launched the way h_generateCartesianMesh,
// h_generateListMesh and h_generateSpiralMesh launch it (:153-180): one block of alignedY threads per mesh-array
// row, no jitter.  type 1 (Cartesian): rows = nx, meshY = ny, alignedY = alignUp(ny, 32); type 2 (list, the
// positions in metres in pos on entry, stepSizeY 0) and type 3 (spiral): rows = ceil(P / 1024), meshY = alignedY =
// 1024, no mirroring.  pos holds rows * alignedY float2.
int ref_mesh(int type, float2* pos, int rows, int meshY, float stepx, float stepy, float one_over_dxs, int mirrorX,
             int mirrorY, float driftx, float drifty) {
  if (rows < 1 || meshY < 1 || meshY > 1024 || type < 1 || type > 3 || (type != 1 && meshY != 1024))
    return int(cudaErrorInvalidValue);
  const float2 drift = make_float2(driftx, drifty);
  if (type == 1)
    d_generateMesh<1><<<rows, align32(meshY)>>>(pos, meshY, stepx, stepy, one_over_dxs, 0, mirrorX != 0,
                                                mirrorY != 0, nullptr, drift);
  else if (type == 2)
    d_generateMesh<2><<<rows, 1024>>>(pos, meshY, stepx, 0.f, one_over_dxs, 0, false, false, nullptr, drift);
  else
    d_generateMesh<3><<<rows, 1024>>>(pos, meshY, stepx, stepy, one_over_dxs, 0, false, false, nullptr, drift);
  return finish();
}

// h_symmetrizeDiffraction (src/DiffractionsKernels.cu:171-178): copy of a numX x numY block between pitched arrays.
int ref_symmetrize(const float* in, float* out, int dataOffX, int dataOffY, int dataAlignedY, int outOffX,
                   int outOffY, int outAlignedY, int numX, int numY) {
  if (numX < 1 || numY < 1 || numY > 1024) return int(cudaErrorInvalidValue);
  d_symmetrizeDiffraction<<<numX, numY>>>(in, out, dataOffX, dataOffY, dataAlignedY, outOffX, outOffY, outAlignedY);
  return finish();
}

// h_realRotate90 (src/utilitiesKernels.cu:2031-2049): `times` quarter turns of an N x N real array (only times % 4
// == 1 moves data in the reference).
int ref_rotate90(const float* in, float* out, int N, int times) {
  if (!pow2_window(N)) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  if (times % 4 == 1) d_rot90<real_t><<<dim3(div_up(N, slice)), dim3(N, slice)>>>(in, out, N, N, N);
  return finish();
}

// h_shiftFFT (src/utilitiesKernels.cu:1945-1964): fftshift of an N x N real array through `temp` (both axes).
int ref_shift_fft(float* data, float* temp, int N) {
  if (!pow2_window(N)) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  const dim3 grid(div_up(N, slice)), block(N, slice);
  d_shiftX<real_t, true><<<grid, block>>>(data, temp, float(N) / 2.0f, 0, N, N, N);
  int rc = finish();
  if (rc) return rc;
  d_shiftY<real_t, true><<<grid, block>>>(temp, data, float(N) / 2.0f, 0, N, N, N);
  return finish();
}

// h_squareRootDiffractions (src/Diffractions.cpp:244-248, src/DiffractionsKernels.cu:187-197): sqrt in place over
// P patterns of N x N.
int ref_sqrt_patterns(float* data, int P, int N) {
  if (!pow2_window(N) || P < 1) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  d_squareRootDiffractions<<<dim3(P, div_up(N, slice)), dim3(N, slice)>>>(data, N, N);
  return finish();
}

// d_preprocessDiffractions (src/DiffractionsKernels.cu:109-118) as h_preprocessDiffractions launches it (:180-187):
// non-finite values to 0, threshold subtracted (values below it to 0), optional sqrt.
int ref_preprocess(float* data, int P, int N, int squareRoot, float threshold) {
  if (!pow2_window(N) || P < 1) return int(cudaErrorInvalidValue);
  const unsigned slice = kMaxThreads / N;
  d_preprocessDiffractions<<<dim3(P, div_up(N, slice)), dim3(N, slice)>>>(data, squareRoot != 0, threshold, N, N);
  return finish();
}

}  // extern "C"
