// Definitions the reference's device functions expect from headers that do not exist under CUDA 12.9 (the
// CUDA-samples helper headers, the removed texture-reference API, the retired uint2float intrinsic).
// TEST INFRASTRUCTURE ONLY: included by oracle/ref_harness.cu ahead of the extracted reference functions.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>
#include <curand_kernel.h>
#include <math_constants.h>
#include <stdint.h>

#include "datatypes.h"  // the reference's own real_t / complex_t definitions (src/datatypes.h)

// src/reductions.cu:17-21 (no device emulation)
#define EMUSYNC

// retired device intrinsic: unsigned int -> float, round to nearest
#define uint2float __uint2float_rn

// dynamic shared memory the reference's reduction kernels use (src/utilitiesKernels.cu:61)
extern __shared__ real_t shared_array[];

// The reference samples its object through a legacy texture reference bound with clamp addressing, linear
// filtering and unnormalised coordinates (src/SampleKernels.cu:48,493-502).  The same sampler, on the same
// texture hardware, is a texture object; this overload lets the unchanged `tex2D(g_objArrayTex, x, y)` calls
// resolve to it.
__device__ cudaTextureObject_t g_objArrayTex;
__device__ __forceinline__ float2 tex2D(cudaTextureObject_t t, float x, float y) { return tex2D<float2>(t, x, y); }
