// Gaussian sketches on the device, drawn exactly as the reference's host code
// draws them: std::mt19937(seed) feeding std::normal_distribution<double>(0, 1)
// as implemented by libstdc++ (src/svd_cpu_rsvd.cpp:10-22), column-major fill.
//
// One CTA replays one stream.  Per pass it twists the 624-word state in three
// dependency phases, tempers it, and consumes the words four at a time: two
// 53-bit canonical doubles (two 32-bit words each, low word first) form one
// polar-method attempt (x, y), accepted when 0 < x^2 + y^2 <= 1.  An accepted
// attempt yields y * mult and then x * mult (the distribution returns y first
// and keeps x for the next call).  624 words are a whole number of attempts,
// so passes never split one.  The arithmetic is IEEE double with every
// product and sum rounded separately (no contraction), so the stream matches
// the host bit for bit except where the device log differs from the host's
// in the last place.
#include "gaussian.cuh"

#include "../../include/fastpls_b200.h"

#include <algorithm>
#include <vector>

#include "capi_util.cuh"
#include "context.cuh"

namespace fpls {
namespace {

constexpr int kN = 624;
constexpr int kM = 397;
constexpr int kAttempts = kN / 4;  // 156
constexpr int kThreads = 256;
constexpr int kScanWarps = (kAttempts + 31) / 32;  // 5
static_assert(kScanWarps * 32 <= kThreads, "the flag scan needs whole warps");

__device__ __forceinline__ uint32_t twist_word(uint32_t cur, uint32_t next, uint32_t far) {
  const uint32_t y = (cur & 0x80000000u) | (next & 0x7fffffffu);
  return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ __forceinline__ uint32_t temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// generate_canonical<double, 53>: (lo + hi * 2^32) / 2^64, clamped below 1.
__device__ __forceinline__ double canonical53(uint32_t lo, uint32_t hi) {
  const double sum = __dadd_rn((double)lo, __dmul_rn((double)hi, 4294967296.0));
  double r = __ddiv_rn(sum, 18446744073709551616.0);
  if (r >= 1.0) r = 0.99999999999999988898;  // nextafter(1, 0)
  return r;
}

__global__ void __launch_bounds__(kThreads) mt_gaussian_kernel(double* __restrict__ out, long long len,
                                                               long long ld, const unsigned int* __restrict__ seeds) {
  __shared__ uint32_t mt[kN];
  __shared__ int flag[kAttempts];
  __shared__ double vx[kAttempts], vy[kAttempts];
  __shared__ int scan[kAttempts];
  __shared__ int wsum[kScanWarps];
  double* dst = out + (long long)blockIdx.x * ld;
  if (threadIdx.x == 0) {
    uint32_t x = seeds[blockIdx.x];
    mt[0] = x;
    for (int i = 1; i < kN; ++i) {
      x = 1812433253u * (x ^ (x >> 30)) + (uint32_t)i;
      mt[i] = x;
    }
  }
  __syncthreads();
  long long produced = 0;
  while (produced < len) {
    // twist: [0, 227) from old words; [227, 454) and [454, 624) from words
    // already renewed in the previous phase (k - 227), x[623] pairs with new x[0]
    uint32_t nw[3];
    int cnt = 0;
    for (int k = threadIdx.x; k < kN - kM; k += kThreads) nw[cnt++] = twist_word(mt[k], mt[k + 1], mt[k + kM]);
    __syncthreads();
    cnt = 0;
    for (int k = threadIdx.x; k < kN - kM; k += kThreads) mt[k] = nw[cnt++];
    __syncthreads();
    cnt = 0;
    for (int k = kN - kM + threadIdx.x; k < 2 * (kN - kM); k += kThreads)
      nw[cnt++] = twist_word(mt[k], mt[k + 1], mt[k - (kN - kM)]);
    __syncthreads();
    cnt = 0;
    for (int k = kN - kM + threadIdx.x; k < 2 * (kN - kM); k += kThreads) mt[k] = nw[cnt++];
    __syncthreads();
    cnt = 0;
    for (int k = 2 * (kN - kM) + threadIdx.x; k < kN; k += kThreads)
      nw[cnt++] = (k == kN - 1) ? twist_word(mt[kN - 1], mt[0], mt[kM - 1])
                                : twist_word(mt[k], mt[k + 1], mt[k - (kN - kM)]);
    __syncthreads();
    cnt = 0;
    for (int k = 2 * (kN - kM) + threadIdx.x; k < kN; k += kThreads) mt[k] = nw[cnt++];
    __syncthreads();
    // polar attempts over the tempered words
    if (threadIdx.x < kAttempts) {
      const int j = threadIdx.x;
      const double u1 = canonical53(temper(mt[4 * j]), temper(mt[4 * j + 1]));
      const double u2 = canonical53(temper(mt[4 * j + 2]), temper(mt[4 * j + 3]));
      const double x = __dsub_rn(__dmul_rn(2.0, u1), 1.0);
      const double y = __dsub_rn(__dmul_rn(2.0, u2), 1.0);
      const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
      const int ok = !(r2 > 1.0 || r2 == 0.0);
      flag[j] = ok;
      if (ok) {
        const double mult = __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
        vx[j] = __dmul_rn(x, mult);
        vy[j] = __dmul_rn(y, mult);
      }
    }
    __syncthreads();
    // exclusive scan of the accept flags: a ballot per warp over the first
    // kScanWarps warps (lanes past the last attempt vote 0), then the warp
    // totals added in warp order
    if (threadIdx.x < kScanWarps * 32) {
      const int j = threadIdx.x, lane = j & 31, w = j >> 5;
      const unsigned b = __ballot_sync(0xffffffffu, j < kAttempts && flag[j]);
      if (lane == 0) wsum[w] = __popc(b);
      __syncwarp();
      if (j < kAttempts) scan[j] = __popc(b & ((1u << lane) - 1u));
    }
    __syncthreads();
    if (threadIdx.x < kAttempts) {
      int off = 0;
      for (int w = 0; w < (threadIdx.x >> 5); ++w) off += wsum[w];
      scan[threadIdx.x] += off;
    }
    __syncthreads();
    if (threadIdx.x < kAttempts && flag[threadIdx.x]) {
      const long long o = produced + 2ll * scan[threadIdx.x];
      if (o < len) dst[o] = vy[threadIdx.x];
      if (o + 1 < len) dst[o + 1] = vx[threadIdx.x];
    }
    const int accepted = scan[kAttempts - 1] + flag[kAttempts - 1];
    produced += 2ll * accepted;
    __syncthreads();
  }
}

}  // namespace

void device_gaussian_streams(double* out, long long len, long long ld, const unsigned int* d_seeds, int nstreams,
                             cudaStream_t stream) {
  if (nstreams <= 0 || len <= 0) return;
  mt_gaussian_kernel<<<nstreams, kThreads, 0, stream>>>(out, len, ld, d_seeds); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void device_gaussian(double* out, long long n_elem, unsigned int seed) {
  Context& ctx = Context::get();
  unsigned int* d = ctx.arena.alloc_n<unsigned int>(1);
  h2d(d, &seed, sizeof(unsigned int));
  device_gaussian_streams(out, n_elem, n_elem, d, 1, ctx.stream);
}

}  // namespace fpls

extern "C" int fpls_gaussian_sketch(int rows, int cols, unsigned int seed, double* out, char* err,
                                    size_t errlen) {
  return fpls::capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(rows >= 0 && cols >= 0, "gaussian_sketch: negative size");
    fpls::Context& ctx = fpls::Context::get();
    ctx.begin_call();
    const long long n = (long long)rows * cols;
    if (n == 0) return;
    double* d = ctx.arena.alloc_n<double>((size_t)n);
    fpls::device_gaussian(d, n, seed);
    fpls::d2h(out, d, (size_t)n * sizeof(double));
    ctx.sync();
  });
}
