// FP64-accurate products on the sm_100a INT8 tensor cores.
//
//   C (M x N, FP64) = A (M x K) * B (N x K)^T
//
// Method: the error-free slice splitting of Ozaki, Ogita and Oishi ("Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59, 2012) in its
// integer form (Ootomo, Ozaki and Yokota, "DGEMM on integer matrix
// multiplication unit", IJHPCA 2024).  Each row r of A and of B (both
// K-contiguous) is scaled by 2^-e_r, e_r the binary exponent of its largest
// magnitude (so every scaled entry is below 1 in magnitude), and written as S
// signed 7-bit digits,
//     x = 2^e * sum_{s=1..S} d_s 2^{-7s} + r,   |d_s| <= 127,  |r| < 2^{e-7S},
// each digit taken exactly in FP64 (multiply by 128, truncate, subtract).  A
// product of two digit planes is exact in int32 (at most K * 127^2 per pair).
// The pairs with s + t <= S + 1 are summed per level l = s + t into their own
// int32 TMEM accumulator (several pairs share a level), and the levels are
// combined in FP64:
//     (A B^T)_ij = 2^{eA_i + eB_j} sum_l 2^{-7l} Acc_l(i, j) + error,
//     |error| <~ 3 K 2^{eA_i + eB_j - 7S}.
//
// Kernel (persistent, one CTA per SM, 6 warps; stream-K over (tile, K block)):
//   warp 0 lane 0  TMA producer.  Per 128-wide K block: the S digit planes of
//                  the 64-row B tile (8 KB each) into one of two B sets, and
//                  the S planes of the 128-row A tile (16 KB each) into S
//                  single-plane slots, each refilled as soon as its last MMA
//                  of the previous K block is done;
//   warp 1 lane 0  MMA issuer: for A plane s, the pairs with B planes
//                  t <= S + 1 - s as tcgen05.mma (kind::i8, M128 K32) over the
//                  B planes taken together (N = 64 per plane, up to 256): the
//                  level accumulators s + t are 64 TMEM columns apart, so each
//                  plane's block of D lands in its own level;
//   warps 2..5     epilogue: tcgen05.ld of the S level accumulators, FP64
//                  combination with the row and column scales, written to C
//                  when the segment covers its whole tile, else as an FP64
//                  stream-K partial; the CTA retiring a tile's last segment
//                  sums that tile's partials in segment order (deterministic).
// Every mbarrier wait is bounded (error flag, no endless spin); the copies and
// MMAs in flight are drained before the CTA releases TMEM and exits.  No
// cluster multicast is used.
#include "autotune.cuh"
#include "ozaki_gemm.cuh"
#include "xop_split.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <map>
#include <vector>

#include "context.cuh"
#include "tc_util.cuh"

namespace fpls {
namespace {

using tc::mbar_arrive;
using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mbar_wait;
using tc::smem_u32;
using tc::sw128_desc;
using tc::tma_load_2d;
using tc::umma_commit;

constexpr int OBM = 128;                 // A rows per tile
constexpr int OBN = 64;                  // B rows per tile
constexpr int OBK = 128;                 // K per block (one 128-byte swizzle row of int8)
constexpr int A_PLANE = OBM * OBK;       // 16 KB
constexpr int B_PLANE = OBN * OBK;       // 8 KB
// Warp 0 loads, warp 1 issues the MMAs, warps 2..9 are the epilogue: two warps
// per TMEM lane quarter (warp w reaches lanes 32 (w % 4) ..), each taking half
// of the tile's columns.
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kTmemCols = 512;
// int32 headroom: one level sums at most S pairs over one segment, so
// S * (64 * 128) * 127^2 < 2^31 for S <= 7.
constexpr int kMaxSegBlocks = 64;

template <int S>
struct OzLayout {
  static constexpr int A_BYTES = S * A_PLANE;
  static constexpr int B_SET = S * B_PLANE;
  static constexpr int BAR_OFF = A_BYTES + 2 * B_SET;
  static constexpr int SMEM_BYTES = BAR_OFF + 256 + 1024;
};
static_assert(OzLayout<kOzakiMaxSlices>::SMEM_BYTES <= 227 * 1024, "digit planes exceed shared memory");
static_assert(kOzakiMaxSlices * OBN <= kTmemCols, "level accumulators exceed TMEM");

// Instruction descriptor: D S32, A/B signed 8-bit, both K-major, M = 128, N = n.
constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(OBM >> 4) << 24);
}
// B planes per MMA: N = 64 * 4 = 256, the largest M = 128 int8 shape.
constexpr int kPlanesPerMma = 4;

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 2^e as a double, for -1022 <= e <= 1023.
__host__ __device__ __forceinline__ double pow2i(int e) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(static_cast<long long>(1023 + e) << 52);
#else
  return std::ldexp(1.0, e);
#endif
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1)
ozaki_gemm_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
                  int a_rows_pad, int b_rows_pad, const double* __restrict__ sA,
                  const double* __restrict__ sB, const int4* __restrict__ segs,
                  const int* __restrict__ cta_seg_begin, const int* __restrict__ tile_seg, int n_tiles_n,
                  double* __restrict__ part, double* __restrict__ C, int ldc, int M, int N, int* err,
                  int a_static, int c_accum) {
  __shared__ int epi_fail;   // raised by any epilogue warp whose wait gave up
  using L = OzLayout<S>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~static_cast<uintptr_t>(1023));
  uint8_t* sa = smem;                  // S single-plane A slots
  uint8_t* sb = smem + L::A_BYTES;     // two sets of S B planes
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
  uint64_t* fullA = bars;
  uint64_t* emptyA = bars + S;
  uint64_t* fullB = bars + 2 * S;
  uint64_t* emptyB = bars + 2 * S + 2;
  uint64_t* tfull = bars + 2 * S + 4;
  uint64_t* tempty = bars + 2 * S + 5;
  uint64_t* done = bars + 2 * S + 6;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 7);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int sbeg = cta_seg_begin[blockIdx.x];
  const int send = cta_seg_begin[blockIdx.x + 1];

  if (threadIdx.x == 0) {
    epi_fail = 0;
    for (int s = 0; s < S; ++s) {
      mbar_init(smem_u32(&fullA[s]), 1);
      mbar_init(smem_u32(&emptyA[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&fullB[b]), 1);
      mbar_init(smem_u32(&emptyB[b]), 1);
    }
    mbar_init(smem_u32(tfull), 1);
    mbar_init(smem_u32(tempty), 32 * kEpiWarps);
    mbar_init(smem_u32(done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  // With a_static the A planes were written before the previous kernel ran,
  // so the first K block's A planes are requested before waiting for it.
  if (warp == 0 && lane == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mB)) : "memory");
  }
  // the segment table is written when the plan is made: read before the wait
  int4 seg0 = make_int4(0, 0, 0, 0);
  if (lane == 0 && warp < 2 && sbeg < send) seg0 = segs[sbeg];
  const bool pre_a = a_static && warp == 0 && lane == 0 && sbeg < send;
  if (pre_a) {
    const int4 seg = seg0;
    const int mt = seg.x / n_tiles_n;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const uint32_t fa = smem_u32(&fullA[s]);
      mbar_expect_tx(fa, A_PLANE);
      tma_load_2d(&mA, smem_u32(sa + s * A_PLANE), fa, seg.y * OBK, s * a_rows_pad + mt * OBM);
    }
  }
  // The set-up above overlaps the previous kernel; its outputs (the B planes
  // and scales) are read only after it has completed.
  tc::grid_dep_wait();
  tc::grid_dep_launch();

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    int it = 0;         // K blocks of this CTA so far
    int b_loads = 0;    // B sets issued (iterations 0 .. b_loads - 1)
    int a_last[S];      // last iteration whose plane s was issued, or -1
#pragma unroll
    for (int s = 0; s < S; ++s) a_last[s] = pre_a ? 0 : -1;
    bool ok = true;
    for (int sg = sbeg; sg < send && ok; ++sg) {
      const int4 seg = sg == sbeg ? seg0 : segs[sg];
      const int mt = seg.x / n_tiles_n, nt = seg.x % n_tiles_n;
      for (int kb = seg.y; kb < seg.z && ok; ++kb, ++it) {
        const int b = it & 1;
        if (!mbar_wait(smem_u32(&emptyB[b]), ((it >> 1) & 1) ^ 1, err)) { ok = false; break; }
        const uint32_t fb = smem_u32(&fullB[b]);
        mbar_expect_tx(fb, S * B_PLANE);
#pragma unroll
        for (int t = 0; t < S; ++t)
          tma_load_2d(&mB, smem_u32(sb + b * L::B_SET + t * B_PLANE), fb, kb * OBK, t * b_rows_pad + nt * OBN);
        b_loads = it + 1;
#pragma unroll
        for (int s = 0; s < S; ++s) {
          if (!ok || (pre_a && it == 0)) break;   // first block's A planes already requested
          if (!mbar_wait(smem_u32(&emptyA[s]), (it & 1) ^ 1, err)) { ok = false; break; }
          const uint32_t fa = smem_u32(&fullA[s]);
          mbar_expect_tx(fa, A_PLANE);
          tma_load_2d(&mA, smem_u32(sa + s * A_PLANE), fa, kb * OBK, s * a_rows_pad + mt * OBM);
          a_last[s] = it;
        }
      }
    }
    // Drain: the last copy issued into every slot has landed before the CTA
    // can exit (bounded waits that ignore the error flag).
    for (int d = 1; d <= 2 && b_loads - d >= 0; ++d) {
      const int u = b_loads - d;
      mbar_wait(smem_u32(&fullB[u & 1]), (u >> 1) & 1, err, false);
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
      if (a_last[s] >= 0) mbar_wait(smem_u32(&fullA[s]), a_last[s] & 1, err, false);
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    int it = 0, j = 0;
    bool ok = true;
    for (int sg = sbeg; sg < send && ok; ++sg, ++j) {
      const int4 seg = sg == sbeg ? seg0 : segs[sg];
      if (!mbar_wait(smem_u32(tempty), (j & 1) ^ 1, err)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int kb = seg.y; kb < seg.z && ok; ++kb, ++it) {
        const int b = it & 1;
        if (!mbar_wait(smem_u32(&fullB[b]), (it >> 1) & 1, err)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t b0 = smem_u32(sb + b * L::B_SET);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          if (!mbar_wait(smem_u32(&fullA[s]), it & 1, err)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(sa + s * A_PLANE);
          // B planes t = 0 .. S-1-s are consecutive 64-row tiles, i.e. one
          // operand of 64 (S - s) rows; the D column block of plane t lands at
          // TMEM column 64 (s + t), the accumulator of level s + t.  Plane s = 0
          // touches every level and initialises them at a segment's first block.
#pragma unroll
          for (int t0 = 0; t0 < S - s; t0 += kPlanesPerMma) {
            const int np = (S - s - t0) < kPlanesPerMma ? (S - s - t0) : kPlanesPerMma;
            const uint32_t idesc = idesc_i8(OBN * np);
            const uint32_t acc = tmem + static_cast<uint32_t>((s + t0) * OBN);
#pragma unroll
            for (int k = 0; k < OBK / 32; ++k) {
              const uint32_t off = k * 32;  // 32 int8 along K per MMA inside the swizzle row
              umma_i8(acc, sw128_desc(a0 + off), sw128_desc(b0 + t0 * B_PLANE + off), idesc,
                      (k > 0 || s > 0 || kb > seg.y) ? 1u : 0u);
            }
          }
          umma_commit(smem_u32(&emptyA[s]));
        }
        if (!ok) break;
        umma_commit(smem_u32(&emptyB[b]));
      }
      if (!ok) break;
      umma_commit(smem_u32(tfull));
    }
    // Every MMA issued by this thread has completed before TMEM is released.
    umma_commit(smem_u32(done));
    mbar_wait(smem_u32(done), 0, err, false);
  } else if (warp >= 2) {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;  // TMEM lane quarter accessible to this warp
    const int half = (warp - 2) / 4;   // which half of the tile's columns
    int j = 0;
    for (int sg = sbeg; sg < send; ++sg, ++j) {
      const int4 seg = segs[sg];
      const int mt = seg.x / n_tiles_n, nt = seg.x % n_tiles_n;
      if (!mbar_wait(smem_u32(tfull), j & 1, err)) atomicOr(&epi_fail, 1);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // the epilogue warps leave together (they share named barrier 1)
      asm volatile("bar.sync 1, %0;" ::"r"(32 * kEpiWarps) : "memory");
      if (*(volatile int*)&epi_fail) {
        mbar_arrive(smem_u32(tempty));
        break;
      }
      const int tile = seg.x;
      const int t0 = tile_seg[tile], t1 = tile_seg[tile + 1];
      const bool whole = (t1 - t0) == 1;   // the tile's only segment: straight to C (when given)
      const int row = mt * OBM + q * 32 + lane;
      const double rs = sA[row];
      const double* cs = sB + nt * OBN;
      double* dst = part + static_cast<size_t>(sg) * OBN * OBM + q * 32 + lane;
      const uint32_t base = tmem + (static_cast<uint32_t>(q * 32) << 16);
#pragma unroll 1
      for (int c = half * (OBN / 32); c < (half + 1) * (OBN / 32); ++c) {
        uint32_t v[S][16];
#pragma unroll
        for (int l = 0; l < S; ++l) tc::tmem_ld16_raw(base + static_cast<uint32_t>(l * OBN + c * 16), v[l]);
        tc::tmem_wait_ld();
        // Levels three at a time, exactly in int64 (v_l 2^14 + v_{l+1} 2^7 +
        // v_{l+2} < 2^46), then one conversion and one scaling per group,
        // smallest group first.
        double acc[16];
#pragma unroll
        for (int x = 0; x < 16; ++x) acc[x] = 0.0;
#pragma unroll
        for (int g = (S - 1) / 3; g >= 0; --g) {
          const int l0 = 3 * g, l1 = (3 * g + 2 < S - 1) ? 3 * g + 2 : S - 1;
          const double w = pow2i(-7 * (l1 + 2));
#pragma unroll
          for (int x = 0; x < 16; ++x) {
            long long q = 0;
#pragma unroll
            for (int l = l0; l <= l1; ++l)
              q += static_cast<long long>(static_cast<int32_t>(v[l][x])) << (7 * (l1 - l));
            acc[x] += static_cast<double>(q) * w;
          }
        }
        if (whole && C) {
          if (row < M) {
#pragma unroll
            for (int x = 0; x < 16; ++x) {
              const int col = nt * OBN + c * 16 + x;
              if (col < N) {
                double* o = C + row + static_cast<size_t>(col) * ldc;
                *o = (c_accum ? *o : 0.0) + acc[x] * rs * cs[c * 16 + x];
              }
            }
          }
        } else {
#pragma unroll
          for (int x = 0; x < 16; ++x) dst[static_cast<size_t>(c * 16 + x) * OBM] = acc[x] * rs * cs[c * 16 + x];
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(smem_u32(tempty));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// C[m + n*ldc] = sum of the tile's partials in segment order (added to C when
// c_accum is set); tiles with one segment were written by the product kernel.
constexpr int kReducePieces = 8;

// tile_segs (when not null) lists each tile's segment ids in contraction
// order (plans whose segments of one tile are not consecutive).
__global__ void ozaki_reduce_kernel(const double* __restrict__ part, const int* __restrict__ tile_seg,
                                    const int* __restrict__ tile_segs, int n_tiles_n, int M, int N,
                                    double* __restrict__ C, int ldc, int c_accum = 0) {
  const int tile = blockIdx.x / kReducePieces;
  const int piece = blockIdx.x % kReducePieces;
  const int s0 = tile_seg[tile], s1 = tile_seg[tile + 1];
  if (s1 - s0 <= 1) return;   // a single segment went straight to C
  const int mt = tile / n_tiles_n, nt = tile % n_tiles_n;
  const int e0 = piece * (OBM * OBN / kReducePieces), e1 = e0 + OBM * OBN / kReducePieces;
  for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
    const int mm = e % OBM, nn = e / OBM;
    const int m = mt * OBM + mm, n = nt * OBN + nn;
    if (m >= M || n >= N) continue;
    double acc = 0.0;
    for (int j = s0; j < s1; ++j) {
      const int s = tile_segs ? tile_segs[j] : j;
      acc += part[(static_cast<size_t>(s) * OBN + nn) * OBM + mm];
    }
    double* o = C + m + static_cast<size_t>(n) * ldc;
    *o = (c_accum ? *o : 0.0) + acc;
  }
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One block per plane row j: the scale exponent from the largest |X[:, j]|,
// then the S digits of every entry (zeros in the padding).  Each thread takes
// four consecutive entries per pass and writes one 32-bit word per plane; the
// digits of a = x 2^-e (|a| < 1) are the 7-bit fields of trunc(a 2^(7S)), most
// significant first, with the sign of a (the same digits as S rounds of
// "times 128, take the integer part").
template <int S>
__global__ void __launch_bounds__(256) ozaki_split_kernel(const double* __restrict__ X, int klen, int cols,
                                                          int ldx, int8_t* __restrict__ P, int ldk,
                                                          size_t plane_stride, double* __restrict__ scale) {
  __shared__ double red[32];
  __shared__ int bad_any;
  const int j = blockIdx.x;
  const double* x = X + static_cast<size_t>(j) * ldx;
  if (threadIdx.x == 0) bad_any = 0;
  double m = 0.0;
  bool bad = false;
  if (j < cols)
    for (int i = threadIdx.x; i < klen; i += blockDim.x) {
      const double v = x[i];
      if (!isfinite(v)) bad = true;
      else m = fmax(m, fabs(v));
    }
  m = warp_max(m);
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
  __syncthreads();
  if (bad) bad_any = 1;
  if (ln == 0) red[w] = m;
  __syncthreads();
  if (w == 0) {
    double r = ln < (int)(blockDim.x >> 5) ? red[ln] : 0.0;
    r = warp_max(r);
    if (ln == 0) red[0] = r;
  }
  __syncthreads();
  m = red[0];
  int e = 0;
  if (m > 0.0) frexp(m, &e);       // m = f 2^e with 1/2 <= f < 1, so |x| 2^-e < 1
  if (e > 1000 && threadIdx.x == 0) bad_any = 1;   // beyond the scale range: NaN column
  e = max(-1000, min(1000, e));
  const double inv = pow2i(-e);
  if (threadIdx.x == 0) scale[j] = bad_any ? __longlong_as_double(0x7ff8000000000000ll) : pow2i(e);
  const double lift = static_cast<double>(1ll << (7 * S));
  int8_t* row = P + static_cast<size_t>(j) * ldk;
  for (int i0 = 4 * threadIdx.x; i0 < ldk; i0 += 4 * blockDim.x) {
    uint32_t wd[S];
#pragma unroll
    for (int s2 = 0; s2 < S; ++s2) wd[s2] = 0u;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u;
      double a = (j < cols && i < klen) ? x[i] * inv : 0.0;
      if (!isfinite(a)) a = 0.0;
      const long long q = __double2ll_rz(a * lift);
      const unsigned long long mag = static_cast<unsigned long long>(q < 0 ? -q : q);
#pragma unroll
      for (int s2 = 0; s2 < S; ++s2) {
        int d = static_cast<int>((mag >> (7 * (S - 1 - s2))) & 127ull);
        if (q < 0) d = -d;
        wd[s2] |= (static_cast<uint32_t>(d) & 0xffu) << (8 * u);
      }
    }
#pragma unroll
    for (int s2 = 0; s2 < S; ++s2)
      *reinterpret_cast<uint32_t*>(row + static_cast<size_t>(s2) * plane_stride + i0) = wd[s2];
  }
}

// Row exponents of a column-major matrix with the column means subtracted:
// thread (row i, column range of the block) takes the largest |x_ij - mean_j|
// and folds its binary exponent into rexp[i] by atomicMax (order-free);
// a non-finite entry raises bad[i].  Eight columns are loaded before any is
// used (eight independent loads in flight per thread), kept in four running
// maxima.
template <typename T>
__global__ void __launch_bounds__(256) ozaki_row_exp_kernel(const T* __restrict__ X, int n, int p, int ld,
                                                            const double* __restrict__ mean, int cols_per_block,
                                                            int* __restrict__ rexp, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j0 = blockIdx.y * cols_per_block, j1 = min(p, j0 + cols_per_block);
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  bool b = false;
  int j = j0;
  for (; j + 8 <= j1; j += 8) {
    T x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = X[i + static_cast<size_t>(j + u) * ld];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double v = static_cast<double>(x[u]) - (mean ? mean[j + u] : 0.0);
      if (!isfinite(v)) b = true;
      else m[u & 3] = fmax(m[u & 3], fabs(v));
    }
  }
  for (; j < j1; ++j) {
    const double v = static_cast<double>(X[i + static_cast<size_t>(j) * ld]) - (mean ? mean[j] : 0.0);
    if (!isfinite(v)) b = true;
    else m[0] = fmax(m[0], fabs(v));
  }
  const double mx = fmax(fmax(m[0], m[1]), fmax(m[2], m[3]));
  if (b) bad[i] = 1;
  if (mx > 0.0) {
    int e = 0;
    frexp(mx, &e);
    atomicMax(rexp + i, e);
  }
}

__global__ void ozaki_row_scale_kernel(const int* __restrict__ rexp, const int* __restrict__ bad, int n, int rows_pad,
                                       double* __restrict__ scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows_pad) return;
  if (i >= n) { scale[i] = 1.0; return; }
  const int e = max(-1000, min(1000, rexp[i] < -1000 ? 0 : rexp[i]));
  scale[i] = (bad[i] || rexp[i] > 1000) ? __longlong_as_double(0x7ff8000000000000ll) : pow2i(e);
}

// Digits of the rows of X - mean (n x p column-major) into the planes (row i of
// plane s at P + s * plane_stride + i * ldk, zero padded to rows_pad x ldk):
// tiles of R rows x 128 columns (R = 64 for FP32 input, 32 for FP64, 33 KB of
// shared memory either way).  Each warp loads 16 columns of the tile's rows
// (16 R / 32 independent coalesced loads per lane) into shared memory; then
// thread (row r, column group g) turns its row's 128 R / 256 consecutive
// entries of the group into digits and writes each plane's 16-byte runs.  The
// S signed 7-bit digits of a = (x - mean) / 2^e (|a| < 1, the scale a power of
// two, so every step is exact) are the base-128 digits of q = trunc(a *
// 2^(7S)), most significant first, carrying the sign of a: one FP64 -> int64
// truncation per entry, the same digits as S rounds of "times 128, take the
// integer part".
constexpr int kSplitCols = 128;
template <typename T>
constexpr int split_rows_per_tile() { return sizeof(T) == 4 ? 64 : 32; }

template <typename T, int S>
__global__ void __launch_bounds__(256) ozaki_split_rows_kernel(const T* __restrict__ X, int n, int p, int ld,
                                                               const double* __restrict__ mean,
                                                               const double* __restrict__ scale,
                                                               int8_t* __restrict__ P, int ldk, size_t plane_stride) {
  constexpr int R = split_rows_per_tile<T>();
  constexpr int H = R / 32;              // 32-row halves loaded per column
  constexpr int G = 256 / R;             // column groups
  constexpr int RUNS = kSplitCols / G / 16;
  __shared__ T tile[kSplitCols][R + 1];
  __shared__ double mj[kSplitCols];
  const int i0 = blockIdx.y * R, j0 = blockIdx.x * kSplitCols;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < kSplitCols) {
    const int j = j0 + threadIdx.x;
    mj[threadIdx.x] = (mean && j < p) ? mean[j] : 0.0;
  }
  {
    T v[16][H];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int j = j0 + warp * 16 + u;
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const int i = i0 + h * 32 + lane;
        v[u][h] = (j < p && i < n) ? X[i + static_cast<size_t>(j) * ld] : T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int h = 0; h < H; ++h) tile[warp * 16 + u][h * 32 + lane] = v[u][h];
  }
  __syncthreads();
  const int r = threadIdx.x % R, g = threadIdx.x / R;
  const int i = i0 + r;
  const double sc = scale[i];
  const double inv = (isfinite(sc) && sc > 0.0) ? 1.0 / sc : 0.0;   // a power of two: exact
  const double lift = static_cast<double>(1ll << (7 * S));
#pragma unroll
  for (int h = 0; h < RUNS; ++h) {
    uint32_t w[S][4];
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
      for (int q = 0; q < 4; ++q) w[s][q] = 0u;
    const int cb = g * (kSplitCols / G) + h * 16;
#pragma unroll
    for (int x = 0; x < 16; ++x) {
      const int c = cb + x;
      const int j = j0 + c;
      double a = (j < p && i < n) ? (static_cast<double>(tile[c][r]) - mj[c]) * inv : 0.0;
      if (!isfinite(a)) a = 0.0;
      const long long qv = __double2ll_rz(a * lift);
      const unsigned long long mag = static_cast<unsigned long long>(qv < 0 ? -qv : qv);
#pragma unroll
      for (int s = 0; s < S; ++s) {
        int d = static_cast<int>((mag >> (7 * (S - 1 - s))) & 127ull);
        if (qv < 0) d = -d;
        w[s][x >> 2] |= (static_cast<uint32_t>(d) & 0xffu) << (8 * (x & 3));
      }
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
      *reinterpret_cast<int4*>(P + static_cast<size_t>(s) * plane_stride + static_cast<size_t>(i) * ldk + j0 + cb) =
          make_int4(static_cast<int>(w[s][0]), static_cast<int>(w[s][1]), static_cast<int>(w[s][2]),
                    static_cast<int>(w[s][3]));
  }
}

template <typename T>
void launch_split_rows(const T* X, int n, int p, int ld, const double* mean, const double* scale, int8_t* P,
                       int ldk, int cols_pad, int rows_pad, size_t plane_stride, int S, cudaStream_t st) {
  const dim3 g(cols_pad / kSplitCols, rows_pad / split_rows_per_tile<T>());
  switch (S) {
    case 4: ozaki_split_rows_kernel<T, 4><<<g, 256, 0, st>>>(X, n, p, ld, mean, scale, P, ldk, plane_stride); break;
    case 5: ozaki_split_rows_kernel<T, 5><<<g, 256, 0, st>>>(X, n, p, ld, mean, scale, P, ldk, plane_stride); break;
    case 6: ozaki_split_rows_kernel<T, 6><<<g, 256, 0, st>>>(X, n, p, ld, mean, scale, P, ldk, plane_stride); break;
    default: ozaki_split_rows_kernel<T, 7><<<g, 256, 0, st>>>(X, n, p, ld, mean, scale, P, ldk, plane_stride); break;
  }
}

int round_up(int x, int a) { return (x + a - 1) / a * a; }

struct OzPlan {
  int tiles = 0, ntn = 0, ctas = 0;
  std::vector<int4> segs;
  std::vector<int> cta_begin, tile_begin;
  // Segment ids of each tile in contraction order (tile t: tile_segs[tile_begin[t]
  // .. tile_begin[t+1])); empty when a tile's segments are consecutive.
  std::vector<int> tile_segs;
};

// K blocks per chunk of a symmetric (Gram) plan: every CTA takes an equal share
// of each chunk, chunk after chunk, so that the CTAs running together read the
// same K-panel of the digit planes from L2 (32 blocks of 128 bytes per row and
// plane: 4096 columns, ~60 MB of planes at 3000 rows and 5 slices).
constexpr int kOzSymChunkBlocks = 32;

// Upper-triangle plan of a symmetric product C = A A^T (n x n): the tiles that
// reach the upper triangle, segments of at most kMaxSegBlocks K blocks cut at
// the chunk boundaries.
OzPlan plan_ozaki_sym(int n, int K, int sm_count) {
  OzPlan g;
  const int mt = (n + OBM - 1) / OBM;
  g.ntn = (n + OBN - 1) / OBN;
  g.tiles = mt * g.ntn;
  std::vector<int> inc;
  for (int t = 0; t < g.tiles; ++t)
    if ((t / g.ntn) * OBM < ((t % g.ntn) + 1) * OBN) inc.push_back(t);
  const int kbt = (K + OBK - 1) / OBK;
  const int kc = kOzSymChunkBlocks;
  const int nchunks = (kbt + kc - 1) / kc;
  const long long ninc = static_cast<long long>(inc.size());
  g.ctas = static_cast<int>(std::max<long long>(1, std::min<long long>(sm_count, ninc * kbt)));
  g.cta_begin.assign(g.ctas + 1, 0);
  g.tile_begin.assign(g.tiles + 1, 0);
  for (int c = 0; c < g.ctas; ++c) {
    g.cta_begin[c] = static_cast<int>(g.segs.size());
    for (int q = 0; q < nchunks; ++q) {
      const int w = std::min(kc, kbt - q * kc);
      const long long tq = ninc * w;
      long long a = tq * c / g.ctas, e = tq * (c + 1) / g.ctas;
      while (a < e) {
        const int t = inc[static_cast<size_t>(a / w)];
        const int kb0 = q * kc + static_cast<int>(a % w);
        int kb1 = static_cast<int>(std::min<long long>(q * kc + w, kb0 + (e - a)));
        kb1 = std::min(kb1, kb0 + kMaxSegBlocks);
        g.segs.push_back(make_int4(t, kb0, kb1, 0));
        a += kb1 - kb0;
      }
    }
  }
  g.cta_begin[g.ctas] = static_cast<int>(g.segs.size());
  std::vector<int> ids(g.segs.size());
  for (size_t i = 0; i < ids.size(); ++i) ids[i] = static_cast<int>(i);
  std::stable_sort(ids.begin(), ids.end(), [&](int x, int y) {
    return g.segs[x].x != g.segs[y].x ? g.segs[x].x < g.segs[y].x : g.segs[x].y < g.segs[y].y;
  });
  g.tile_segs = ids;
  int s = 0;
  for (int t = 0; t < g.tiles; ++t) {
    g.tile_begin[t] = s;
    while (s < static_cast<int>(ids.size()) && g.segs[ids[s]].x == t) ++s;
  }
  g.tile_begin[g.tiles] = s;
  return g;
}

// Stream-K plan: CTA c covers iterations [c*total/ctas, (c+1)*total/ctas) of
// the (tile, K block) space, cut into per-tile segments of at most
// kMaxSegBlocks K blocks.
OzPlan plan_ozaki(int M, int N, int K, int sm_count) {
  OzPlan g;
  const int mt = (M + OBM - 1) / OBM;
  g.ntn = (N + OBN - 1) / OBN;
  g.tiles = mt * g.ntn;
  const int kbt = (K + OBK - 1) / OBK;
  const long long total = static_cast<long long>(g.tiles) * kbt;
  g.ctas = static_cast<int>(std::max<long long>(1, std::min<long long>(sm_count, total)));
  g.cta_begin.assign(g.ctas + 1, 0);
  g.tile_begin.assign(g.tiles + 1, 0);
  for (int c = 0; c < g.ctas; ++c) {
    g.cta_begin[c] = static_cast<int>(g.segs.size());
    long long a = total * c / g.ctas, e = total * (c + 1) / g.ctas;
    while (a < e) {
      const int t = static_cast<int>(a / kbt);
      const int kb0 = static_cast<int>(a % kbt);
      int kb1 = static_cast<int>(std::min<long long>(kbt, kb0 + (e - a)));
      kb1 = std::min(kb1, kb0 + kMaxSegBlocks);
      g.segs.push_back(make_int4(t, kb0, kb1, 0));
      a += kb1 - kb0;
    }
  }
  g.cta_begin[g.ctas] = static_cast<int>(g.segs.size());
  int s = 0;
  for (int t = 0; t < g.tiles; ++t) {
    g.tile_begin[t] = s;
    while (s < static_cast<int>(g.segs.size()) && g.segs[s].x == t) ++s;
  }
  g.tile_begin[g.tiles] = s;
  return g;
}

struct OzCached {
  OzPlan g;
  char* dev = nullptr;
  int4* segs = nullptr;
  int* cta_begin = nullptr;
  int* tile_begin = nullptr;
  int* tile_segs = nullptr;   // null unless the plan lists each tile's segments
  double* part = nullptr;
};

std::map<std::array<int, 5>, OzCached>& oz_cache() {
  static std::map<std::array<int, 5>, OzCached> cache;
  return cache;
}

// Plans, their device tables and the partial buffers are kept per shape (and
// plan kind: general, or the upper tiles of a symmetric product), so the
// repeated products of an iteration issue no host-to-device copy.
const OzCached& oz_plan(int M, int N, int K, int sm_count, cudaStream_t st, bool sym = false) {
  auto& cache = oz_cache();
  const std::array<int, 5> key{M, N, K, sm_count, sym ? 1 : 0};
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  OzCached c;
  c.g = sym ? plan_ozaki_sym(M, K, sm_count) : plan_ozaki(M, N, K, sm_count);
  auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t b_segs = up(c.g.segs.size() * sizeof(int4));
  const size_t b_cta = up(c.g.cta_begin.size() * sizeof(int));
  const size_t b_tile = up(c.g.tile_begin.size() * sizeof(int));
  const size_t b_tsegs = up(std::max<size_t>(c.g.tile_segs.size(), 1) * sizeof(int));
  const size_t b_part = c.g.segs.size() * static_cast<size_t>(OBM) * OBN * sizeof(double);
  FPLS_CUDA(cudaMalloc(&c.dev, b_segs + b_cta + b_tile + b_tsegs + b_part));
  c.segs = reinterpret_cast<int4*>(c.dev);
  c.cta_begin = reinterpret_cast<int*>(c.dev + b_segs);
  c.tile_begin = reinterpret_cast<int*>(c.dev + b_segs + b_cta);
  c.tile_segs = c.g.tile_segs.empty() ? nullptr : reinterpret_cast<int*>(c.dev + b_segs + b_cta + b_tile);
  c.part = reinterpret_cast<double*>(c.dev + b_segs + b_cta + b_tile + b_tsegs);
  FPLS_CUDA(cudaMemcpyAsync(c.segs, c.g.segs.data(), c.g.segs.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  FPLS_CUDA(cudaMemcpyAsync(c.cta_begin, c.g.cta_begin.data(), c.g.cta_begin.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  FPLS_CUDA(cudaMemcpyAsync(c.tile_begin, c.g.tile_begin.data(), c.g.tile_begin.size() * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  if (c.tile_segs)
    FPLS_CUDA(cudaMemcpyAsync(c.tile_segs, c.g.tile_segs.data(), c.g.tile_segs.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
  return cache.emplace(key, std::move(c)).first->second;
}

// 2-D int8 tensor map over all planes stacked (rows_pad * slices rows of ldk
// bytes, row_stride() bytes apart).
CUtensorMap make_plane_map(const OzakiPlanes& p, int box_rows) {
  CUtensorMap m;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(p.ldk), static_cast<cuuint64_t>(p.rows_pad) * p.slices};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(p.row_stride())};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(OBK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tc::encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, p.data, dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(kErrCuda, "cuTensorMapEncodeTiled failed (digit planes)");
  return m;
}

template <int S>
void ensure_ozaki_attr() {
  static bool attr = false;
  if (!attr) {
    FPLS_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   OzLayout<S>::SMEM_BYTES));
    attr = true;
  }
}

void ensure_ozaki_attr_for(int slices) {
  switch (slices) {
    case 4: ensure_ozaki_attr<4>(); break;
    case 5: ensure_ozaki_attr<5>(); break;
    case 6: ensure_ozaki_attr<6>(); break;
    default: ensure_ozaki_attr<7>(); break;
  }
}

template <int S>
void launch_ozaki(const CUtensorMap& mA, const CUtensorMap& mB, const OzakiPlanes& A, const OzakiPlanes& B,
                  const OzCached& c, double* C, int ldc, int* err, cudaStream_t st, bool a_static,
                  bool c_accum) {
  ensure_ozaki_attr<S>();
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(c.g.ctas);
  lc.blockDim = dim3(kThreads);
  lc.dynamicSmemBytes = OzLayout<S>::SMEM_BYTES;
  lc.stream = st;
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = pdl;
  lc.numAttrs = tc::pdl_enabled() ? 1 : 0;
  const int a_rows_pad = A.rows_pad, b_rows_pad = B.rows_pad, ntn = c.g.ntn, m_rows = A.rows, n_rows = B.rows;
  FPLS_CUDA(cudaLaunchKernelEx(&lc, ozaki_gemm_kernel<S>, mA, mB, a_rows_pad, b_rows_pad,
                               static_cast<const double*>(A.scale), static_cast<const double*>(B.scale),
                               static_cast<const int4*>(c.segs), static_cast<const int*>(c.cta_begin),
                               static_cast<const int*>(c.tile_begin), ntn, c.part, C, ldc, m_rows, n_rows, err,
                               a_static ? 1 : 0, c_accum ? 1 : 0));
}

struct XOperatorOzakiSym : public XOperator {
  OzakiPlanes kp;
  int slices;
  XOperatorOzakiSym(const double* K, int n_, int s) : slices(s) {
    n = n_;
    p = n_;
    kp = ozaki_alloc(n, n, slices);
    ozaki_split(K, n, kp);   // row j of the planes = column j of K = row j (K symmetric)
  }
  void times(const double* M, int F, double* U) override {
    OzakiPlanes b = ozaki_alloc(F, n, slices);
    ozaki_split(M, n, b);
    ozaki_gemm(kp, b, U, n, true);
  }
  void t_times(const double* M, int F, double* U) override { times(M, F, U); }
  OzakiPartials times_partials(const double* M, int F) {
    OzakiPlanes b = ozaki_alloc(F, n, slices);
    ozaki_split(M, n, b);
    return ozaki_gemm_partials(kp, b, true);
  }
  void gram(double*) override { throw Error(kErrArgument, "the INT8 product operator has no Gram"); }
};

// X as its centred rows' digit planes: times() (X M for a p x F block M, the
// sketch product) and gram() (X X^T) on the INT8 tensor cores.
struct XOperatorOzakiRows : public XOperator {
  OzakiPlanes xp;
  XOperatorOzakiRows(const double* x64, const float* x32, const double* mean, int n_, int p_, int slices) {
    n = n_;
    p = p_;
    xp = ozaki_split_rows(x64, x32, n_, p_, mean, slices);
  }
  void times(const double* M, int F, double* U) override {
    OzakiPlanes b = ozaki_alloc(F, p, xp.slices);
    ozaki_split(M, p, b);
    ozaki_gemm(xp, b, U, n);
  }
  void t_times(const double*, int, double*) override {
    throw Error(kErrArgument, "the INT8 row operator has no transposed product");
  }
  void gram(double* K) override { ozaki_gram(xp, K, n); }
};

}  // namespace

namespace {

// Runs the product kernel (defined below).
const OzCached& run_ozaki(const OzakiPlanes& A, const OzakiPlanes& B, double* C, int ldc, bool a_static,
                          bool sym = false, bool c_accum = false);

// Row scales of the n x p column-major matrix X - mean (x64 or x32, ld n) into
// scale (rows_pad entries: 2^e above each row's largest magnitude, 1 on the
// padding rows, NaN for a row with a non-finite entry), then its digits into
// the planes at P (rows ld_planes bytes apart, planes plane_stride apart),
// columns [0, cols_pad) with zeros past p.
void split_rows_range(const double* x64, const float* x32, int n, int p, const double* mean, int slices,
                      int rows_pad, double* scale, int8_t* P, int ld_planes, int cols_pad, size_t plane_stride) {
  Context& ctx = Context::get();
  int* rexp = ctx.arena.alloc_n<int>(n);
  int* bad = ctx.arena.alloc_n<int>(n);
  FPLS_CUDA(cudaMemsetAsync(rexp, 0x80, n * sizeof(int), ctx.stream));   // a very negative sentinel
  dzero(bad, n * sizeof(int));
  constexpr int kCols = 160;
  const dim3 g1(ceil_div(n, 256), ceil_div(p, kCols));
  if (x64) ozaki_row_exp_kernel<double><<<g1, 256, 0, ctx.stream>>>(x64, n, p, n, mean, kCols, rexp, bad);
  else ozaki_row_exp_kernel<float><<<g1, 256, 0, ctx.stream>>>(x32, n, p, n, mean, kCols, rexp, bad);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  ozaki_row_scale_kernel<<<ceil_div(rows_pad, 256), 256, 0, ctx.stream>>>(rexp, bad, n, rows_pad, scale);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  static_assert(OBM % 64 == 0 && OBK % kSplitCols == 0, "split tiles must divide the plane padding");
  if (x64) launch_split_rows<double>(x64, n, p, n, mean, scale, P, ld_planes, cols_pad, rows_pad, plane_stride,
                                     slices, ctx.stream);
  else launch_split_rows<float>(x32, n, p, n, mean, scale, P, ld_planes, cols_pad, rows_pad, plane_stride, slices,
                                ctx.stream);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

// The upper tiles of C = A A^T (set, or increased when accumulate is set); the
// lower triangle is left to the caller.
void ozaki_gram_upper(const OzakiPlanes& A, double* C, int ldc, bool accumulate) {
  FPLS_REQUIRE(ldc == A.rows, "INT8 Gram: the output must be n x n with ld n");
  Context& ctx = Context::get();
  const int slot = ctx.prof_begin("gram_int8", ctx.stream);
  const OzCached& c = run_ozaki(A, A, C, ldc, false, true, accumulate);
  // the upper tiles' partials summed in contraction order (tiles with a single
  // segment were written by the product kernel)
  ozaki_reduce_kernel<<<c.g.tiles * kReducePieces, 256, 0, ctx.stream>>>(c.part, c.tile_begin, c.tile_segs, c.g.ntn,
                                                                         A.rows, A.rows, C, ldc, accumulate ? 1 : 0);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  if (slot >= 0) {
    // algorithmic work: the S (S + 1) / 2 digit-plane pairs over the planned
    // (upper) tiles; bytes: every plane of A once and C once
    const double S = A.slices, n = A.rows, K = A.k;
    int planned = 0;
    for (int t = 0; t < c.g.tiles; ++t) planned += c.g.tile_begin[t + 1] > c.g.tile_begin[t];
    const double frac = static_cast<double>(planned) / c.g.tiles;
    ctx.prof_end(slot, ctx.stream, S * n * K + 8.0 * n * n * frac, 0.5 * S * (S + 1.0) * 2.0 * n * n * K * frac);
  }
}

// X as column chunks of digit planes, each chunk with its own row scales.
struct XOperatorOzakiRowsChunked : public XOperator {
  OzakiPlanes xp;                  // all columns; xp.scale unused
  std::vector<int> bounds;
  std::vector<double*> scales;     // per chunk, rows_pad entries
  XOperatorOzakiRowsChunked(int n_, int p_, int slices, const std::vector<int>& b) : bounds(b) {
    n = n_;
    p = p_;
    FPLS_REQUIRE(bounds.size() >= 2 && bounds.front() == 0 && bounds.back() == p_,
                 "INT8 chunks: bounds must run from 0 to p");
    for (size_t c = 1; c + 1 < bounds.size(); ++c)
      FPLS_REQUIRE(bounds[c] % OBK == 0 && bounds[c] > bounds[c - 1], "INT8 chunks: inner bounds must be multiples of 128");
    xp = ozaki_alloc(n_, p_, slices);
    for (size_t c = 0; c + 1 < bounds.size(); ++c) scales.push_back(Context::get().arena.alloc_n<double>(xp.rows_pad));
  }
  int chunks() const { return static_cast<int>(bounds.size()) - 1; }
  // columns [bounds[c], bounds[c+1]) of `full` as planes of their own
  OzakiPlanes view(const OzakiPlanes& full, int c, double* scale) const {
    OzakiPlanes v = full;
    v.data = full.data + bounds[c];
    v.k = bounds[c + 1] - bounds[c];
    v.ldk = round_up(v.k, OBK);
    v.ld = full.row_stride();
    v.scale = scale;
    return v;
  }
  void times(const double* M, int F, double* U) override {
    OzakiPlanes b = ozaki_alloc(F, p, xp.slices);
    ozaki_split(M, p, b);
    Context& ctx = Context::get();
    for (int c = 0; c < chunks(); ++c) {
      const OzakiPlanes a = view(xp, c, scales[c]);
      const OzakiPlanes bc = view(b, c, b.scale);
      const OzCached& cc = run_ozaki(a, bc, U, n, false, false, c > 0);
      ozaki_reduce_kernel<<<cc.g.tiles * kReducePieces, 256, 0, ctx.stream>>>(cc.part, cc.tile_begin, nullptr,
                                                                              cc.g.ntn, n, F, U, n, c > 0 ? 1 : 0);
      ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
  }
  void t_times(const double*, int, double*) override {
    throw Error(kErrArgument, "the INT8 row operator has no transposed product");
  }
  void gram(double*) override { throw Error(kErrArgument, "the chunked INT8 row operator forms its Gram by chunks"); }
};

XOperatorOzakiRowsChunked& as_chunked(XOperator& op) {
  auto* o = dynamic_cast<XOperatorOzakiRowsChunked*>(&op);
  FPLS_REQUIRE(o != nullptr, "INT8 chunks: not a chunked INT8 row operator");
  return *o;
}

}  // namespace

OzakiPlanes ozaki_split_rows(const double* x64, const float* x32, int n, int p, const double* mean, int slices) {
  OzakiPlanes pl = ozaki_alloc(n, p, slices);
  split_rows_range(x64, x32, n, p, mean, slices, pl.rows_pad, pl.scale, pl.data, pl.ldk, pl.ldk,
                   static_cast<size_t>(pl.rows_pad) * pl.ldk);
  return pl;
}

std::unique_ptr<XOperator> make_ozaki_rows_chunked(int n, int p, int slices, const std::vector<int>& bounds) {
  return std::unique_ptr<XOperator>(new XOperatorOzakiRowsChunked(n, p, slices, bounds));
}

void ozaki_rows_fill_chunk(XOperator& op, const double* c64, const float* c32, const double* mean, int c) {
  XOperatorOzakiRowsChunked& o = as_chunked(op);
  FPLS_REQUIRE(c >= 0 && c < o.chunks(), "INT8 chunks: chunk index out of range");
  const int j0 = o.bounds[c], w = o.bounds[c + 1] - j0;
  split_rows_range(c64, c32, o.n, w, mean, o.xp.slices, o.xp.rows_pad, o.scales[c], o.xp.data + j0, o.xp.ldk,
                   round_up(w, OBK), static_cast<size_t>(o.xp.rows_pad) * o.xp.ldk);
}

void ozaki_rows_gram_chunk(XOperator& op, double* K, int c, bool accumulate) {
  XOperatorOzakiRowsChunked& o = as_chunked(op);
  FPLS_REQUIRE(c >= 0 && c < o.chunks(), "INT8 chunks: chunk index out of range");
  ozaki_gram_upper(o.view(o.xp, c, o.scales[c]), K, o.n, accumulate);
}

std::unique_ptr<XOperator> make_ozaki_rows_operator(const double* x64, const float* x32, const double* mean, int n,
                                                    int p, int slices) {
  return std::unique_ptr<XOperator>(new XOperatorOzakiRows(x64, x32, mean, n, p, slices));
}

OzakiPlanes ozaki_alloc(int rows, int k, int slices) {
  FPLS_REQUIRE(slices >= kOzakiMinSlices && slices <= kOzakiMaxSlices, "INT8 products: slices must be in 4..7");
  FPLS_REQUIRE(rows >= 1 && k >= 1, "INT8 products: empty operand");
  OzakiPlanes p;
  p.rows = rows;
  p.k = k;
  p.slices = slices;
  p.rows_pad = round_up(rows, OBM);
  p.ldk = round_up(k, OBK);
  Arena& ar = Context::get().arena;
  p.data = ar.alloc_n<int8_t>(static_cast<size_t>(slices) * p.rows_pad * p.ldk);
  p.scale = ar.alloc_n<double>(p.rows_pad);
  return p;
}

void ozaki_split(const double* X, int ldx, const OzakiPlanes& out) {
  Context& ctx = Context::get();
  const size_t stride = static_cast<size_t>(out.rows_pad) * out.ldk;
  switch (out.slices) {
    case 4: ozaki_split_kernel<4><<<out.rows_pad, 256, 0, ctx.stream>>>(X, out.k, out.rows, ldx, out.data, out.ldk,
                                                                        stride, out.scale); break;
    case 5: ozaki_split_kernel<5><<<out.rows_pad, 256, 0, ctx.stream>>>(X, out.k, out.rows, ldx, out.data, out.ldk,
                                                                        stride, out.scale); break;
    case 6: ozaki_split_kernel<6><<<out.rows_pad, 256, 0, ctx.stream>>>(X, out.k, out.rows, ldx, out.data, out.ldk,
                                                                        stride, out.scale); break;
    default: ozaki_split_kernel<7><<<out.rows_pad, 256, 0, ctx.stream>>>(X, out.k, out.rows, ldx, out.data, out.ldk,
                                                                         stride, out.scale); break;
  }
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

namespace {

// Runs the product kernel: whole tiles straight to C (when C is given), the
// others as partials in the cached plan.
const OzCached& run_ozaki(const OzakiPlanes& A, const OzakiPlanes& B, double* C, int ldc, bool a_static,
                          bool sym, bool c_accum) {
  FPLS_REQUIRE(A.slices == B.slices && A.k == B.k && A.ldk == B.ldk, "INT8 products: operands do not match");
  Context& ctx = Context::get();
  cudaStream_t st = ctx.stream;
  const OzCached& c = oz_plan(A.rows, B.rows, A.k, ctx.sm_count, st, sym);
  const CUtensorMap mA = make_plane_map(A, OBM);
  const CUtensorMap mB = make_plane_map(B, OBN);
  int* err = ctx.d_status + 16;
  switch (A.slices) {
    case 4: launch_ozaki<4>(mA, mB, A, B, c, C, ldc, err, st, a_static, c_accum); break;
    case 5: launch_ozaki<5>(mA, mB, A, B, c, C, ldc, err, st, a_static, c_accum); break;
    case 6: launch_ozaki<6>(mA, mB, A, B, c, C, ldc, err, st, a_static, c_accum); break;
    default: launch_ozaki<7>(mA, mB, A, B, c, C, ldc, err, st, a_static, c_accum); break;
  }
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  return c;
}

}  // namespace

void ozaki_gemm(const OzakiPlanes& A, const OzakiPlanes& B, double* C, int ldc, bool a_static) {
  const OzCached& c = run_ozaki(A, B, C, ldc, a_static);
  ozaki_reduce_kernel<<<c.g.tiles * kReducePieces, 256, 0, Context::get().stream>>>(c.part, c.tile_begin, nullptr,
                                                                                 c.g.ntn, A.rows, B.rows, C, ldc);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void ozaki_gram(const OzakiPlanes& A, double* C, int ldc) {
  ozaki_gram_upper(A, C, ldc, false);
  mirror_upper_triangle(C, A.rows);
}

OzakiPartials ozaki_gemm_partials(const OzakiPlanes& A, const OzakiPlanes& B, bool a_static) {
  const OzCached& c = run_ozaki(A, B, nullptr, 0, a_static);
  OzakiPartials p;
  p.part = c.part;
  p.tile_seg = c.tile_begin;
  p.n_tiles_n = c.g.ntn;
  return p;
}

void ozaki_release_cache() {
  for (auto& kv : oz_cache()) cudaFree(kv.second.dev);
  oz_cache().clear();
}

std::unique_ptr<XOperator> make_ozaki_sym_operator(const double* K, int n, int slices) {
  return std::unique_ptr<XOperator>(new XOperatorOzakiSym(K, n, slices));
}

OzakiPartials ozaki_sym_partials_from_planes(XOperator& op, const OzakiPlanes& b) {
  auto* oz = dynamic_cast<XOperatorOzakiSym*>(&op);
  FPLS_REQUIRE(oz != nullptr, "INT8 partial products need the INT8 operator");
  return ozaki_gemm_partials(oz->kp, b, true);
}

void ozaki_sym_prepare_partials(XOperator& op, const OzakiPlanes& b) {
  auto* oz = dynamic_cast<XOperatorOzakiSym*>(&op);
  FPLS_REQUIRE(oz != nullptr, "INT8 partial products need the INT8 operator");
  FPLS_REQUIRE(oz->kp.slices == b.slices && oz->kp.k == b.k, "INT8 products: operands do not match");
  Context& ctx = Context::get();
  oz_plan(oz->kp.rows, b.rows, oz->kp.k, ctx.sm_count, ctx.stream);
  ensure_ozaki_attr_for(b.slices);
  tc::encode_fn();
}

OzakiPartials ozaki_sym_times_partials(XOperator& op, const double* M, int F) {
  auto* oz = dynamic_cast<XOperatorOzakiSym*>(&op);
  FPLS_REQUIRE(oz != nullptr, "INT8 partial products need the INT8 operator");
  return oz->times_partials(M, F);
}

int ozaki_default_slices() {
  if (const char* e = std::getenv("FASTPLS_OZAKI_SLICES")) {
    const int v = std::atoi(e);
    if (v >= kOzakiMinSlices && v <= kOzakiMaxSlices) return v;
  }
  const int t = active_tune().ozaki_slices;
  if (t >= kOzakiMinSlices && t <= kOzakiMaxSlices) return t;
  // 2^-35 of the row scales, about four orders of magnitude below the error
  // the BF16x3 row Gram already carries: on the omics double-CV grid 5, 6 and 7
  // slices give the same predictions as FP64 products (5 and 6 the same to the
  // last inner prediction) and 4 do not.
  return 5;
}

}  // namespace fpls
