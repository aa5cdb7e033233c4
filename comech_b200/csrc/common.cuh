// Shared definitions of the feb200 device library (voxel linear-elastic FE solver for sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "../../include/feb200.h"

namespace feb {

// Error propagation: every host entry point returns an int status and never aborts.
struct FebError {
  int code;
  char msg[256];
};
void set_last_error(const char* fmt, ...);

#define FEB_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      ::feb::set_last_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return FEB_ERR_CUDA;                                                               \
    }                                                                                    \
  } while (0)

#define FEB_TRY(call)                          \
  do {                                         \
    const int feb_try_st_ = (call);            \
    if (feb_try_st_ != FEB_OK) return feb_try_st_; \
  } while (0)

// host-side count of kernel launches issued by the library (feb_launch_count)
void note_launch(int n = 1);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current device (the attribute is per
// device; set once per device and kernel, thread-safe); returns a status.
int set_dyn_smem(const void* kernel, int bytes);

// symmetric pseudo-inverse by cyclic Jacobi, numpy.linalg.pinv semantics (cutoff 1e-15 max |eigenvalue|);
// A is n x n row-major (host)
std::vector<double> sym_pinv(const std::vector<double>& A, int n);

constexpr int kThreads = 256;
constexpr int kSmCount = 148;

inline int div_up(int64_t a, int64_t b) { return int((a + b - 1) / b); }

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Material model of the matrix-free element operator.
//   ISO_SRI : D = mu-part integrated 2x2x2, lambda-part at the cell centre (rb/splitfe.py:58-69)
//   ISO_FULL: lambda and mu parts integrated 2x2x2 (fe/solver.py:77-90)
//   ORTHO   : six orthotropic pattern coefficients, 2x2x2 (fe/solver.py:43-74)
enum MatMode : int { MAT_ISO_SRI = 0, MAT_ISO_FULL = 1, MAT_ORTHO = 2 };

template <int MODE> struct MatWidth { static constexpr int value = (MODE == MAT_ORTHO) ? 6 : 2; };

__device__ __forceinline__ double atomic_add(double* p, double v) { return atomicAdd(p, v); }
__device__ __forceinline__ float atomic_add(float* p, float v) { return atomicAdd(p, v); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of one value per thread (blockDim.x a multiple of 32, <= 1024); result valid in thread 0.
template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T partial[32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) partial[wid] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? partial[threadIdx.x] : T(0);
  if (wid == 0) v = warp_sum(v);
  return v;
}

}  // namespace feb
