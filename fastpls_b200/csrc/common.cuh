// Shared helpers for the fastpls_b200 CUDA library (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace fpls {

// Error raised inside the library; the C-ABI layer converts it into a status
// code plus a message in the caller's buffer (no exception crosses the ABI).
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

enum Status : int {
  kOk = 0,
  kErrArgument = 1,
  kErrCuda = 2,
  kErrNumerical = 3,
  kErrNoDevice = 4,
  kErrInternal = 5,
};

#define FPLS_CUDA(call)                                                          \
  do {                                                                           \
    cudaError_t e__ = (call);                                                    \
    if (e__ != cudaSuccess) {                                                    \
      throw ::fpls::Error(::fpls::kErrCuda, std::string("CUDA error: ") +        \
                                               cudaGetErrorString(e__) + " at " + \
                                               __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                            \
  } while (0)

#define FPLS_CHECK_LAUNCH() FPLS_CUDA(cudaGetLastError())

#define FPLS_REQUIRE(cond, msg)                                                  \
  do {                                                                           \
    if (!(cond)) throw ::fpls::Error(::fpls::kErrArgument, (msg));               \
  } while (0)

constexpr int kSMCount = 148;  // B200: 2 dies x 74 SMs

// Host-side count of kernel launches issued by this library (every launch
// site calls note_launch() right after its <<<...>>>).
void note_launch();
long long launch_count();

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// D (8 x 8) += A (8 x 4) B (4 x 8) on the FP64 tensor cores (mma.sync m8n8k4):
// lane l holds a = A[l / 4][l % 4], b = B[l % 4][l / 4] and the accumulators
// c0, c1 = D[l / 4][2 (l % 4)], D[l / 4][2 (l % 4) + 1].
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Block-wide sum; `scratch` needs blockDim.x/32 doubles. Result valid in all threads.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  for (int i = 0; i < nwarps; ++i) r += scratch[i];
  __syncthreads();
  return r;
}

}  // namespace fpls
