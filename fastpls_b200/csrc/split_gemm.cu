// BF16 split-precision GEMM on the sm_100a tensor cores (tcgen05 + TMA + TMEM).
//
//   C (M x N, FP64) = A (M x K) * B (N x K)^T
//
// where A and B are each held as a pair of BF16 matrices (hi = bf16(x),
// lo = bf16(x - hi)), K-contiguous.  Every 16-wide K step issues three UMMAs
// into the same FP32 TMEM accumulator: hi*hi + hi*lo + lo*hi.
//
// Kernel structure (persistent, one CTA per SM, 6 warps):
//   warp 0 lane 0  TMA producer: A_hi, A_lo (128 x 64) and B_hi, B_lo (64 x 64)
//                  tiles per 64-wide K block into a 4-stage SWIZZLE_128B ring;
//   warp 1 lane 0  MMA issuer: 12 tcgen05.mma (M128 N64 K16) per K block,
//                  tcgen05.commit frees the stage; accumulators double-buffered
//                  in TMEM (2 x 64 columns) so the epilogue overlaps the next tile;
//   warps 2..5     epilogue: tcgen05.ld of the 128 x 64 FP32 accumulator, one
//                  TMEM lane quarter per warp, stored as a stream-K partial.
// Work is split stream-K: the (tile, K block) iteration space is cut into
// equal contiguous ranges per CTA; a second kernel sums each tile's partials in
// FP64.  All mbarrier waits are bounded by a clock budget and raise an error
// flag instead of spinning forever.  No cluster multicast is used.
#include <atomic>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <array>
#include <map>
#include <memory>
#include <vector>
#include <string>
#include <cstdlib>

#include "autotune.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "tc_util.cuh"
#include "xop_split.cuh"

namespace fpls {
namespace {

using tc::encode_fn;
using tc::mbar_arrive;
using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mbar_wait;
using tc::smem_u32;
using tc::sw128_desc;
using tc::tma_load_2d;
using tc::umma_commit;

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  tc::tmem_ld16_raw(taddr, r);
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

constexpr int BM = 128;
constexpr int BN = 64;     // N tile of the general products
constexpr int BN_SYM = 128;  // N tile of the symmetric (Gram) products
constexpr int BK = 64;
constexpr int A_TILE = BM * BK * 2;                 // 16 KB
constexpr int BAR_BYTES = 256;
// NP BF16 planes per operand, TN columns per output tile.  TN = 64: 48 KB
// (two planes) or 72 KB (three) stages, 4 or 3 deep; TN = 128: 64 KB or 96 KB
// stages, 3 or 2 deep.
template <int NP, int TN> struct Planes {
  static constexpr int B_BYTES = TN * BK * 2;
  static constexpr int STAGES = TN == 64 ? (NP == 2 ? 4 : 3) : (NP == 2 ? 3 : 2);
  static constexpr int STAGE_BYTES = NP * (A_TILE + B_BYTES);
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + BAR_BYTES + 1024;
  static constexpr int TMEM_COLS = 2 * TN;
  // Instruction descriptor: D F32, A/B BF16, both K-major, N = TN, M = 128.
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) |
                                    (uint32_t(TN >> 3) << 17) | (uint32_t(BM >> 4) << 24);
};
static_assert(Planes<3, 64>::SMEM_BYTES <= 227 * 1024, "three-plane stages exceed shared memory");
static_assert(Planes<2, 128>::SMEM_BYTES <= 227 * 1024, "wide-tile stages exceed shared memory");
static_assert(Planes<3, 128>::SMEM_BYTES <= 227 * 1024, "three-plane wide-tile stages exceed shared memory");
constexpr int NUM_THREADS = 192;

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}


template <int NP, int TN>
__global__ void __launch_bounds__(NUM_THREADS, 1)
split_gemm_kernel(const __grid_constant__ CUtensorMap mA0, const __grid_constant__ CUtensorMap mA1,
                  const __grid_constant__ CUtensorMap mA2, const __grid_constant__ CUtensorMap mB0,
                  const __grid_constant__ CUtensorMap mB1, const __grid_constant__ CUtensorMap mB2,
                  const int4* __restrict__ segs, const int* __restrict__ cta_seg_begin,
                  int n_tiles_n, float* __restrict__ part, int* err, int withhold_loads) {
  using P = Planes<NP, TN>;
  constexpr int STAGES = P::STAGES;
  constexpr int STAGE_BYTES = P::STAGE_BYTES;
  constexpr int B_T = P::B_BYTES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* tfull = bars + 2 * STAGES;
  uint64_t* tempty = bars + 2 * STAGES + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 4);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int sbeg = cta_seg_begin[blockIdx.x];
  const int send = cta_seg_begin[blockIdx.x + 1];

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&tfull[b]), 1);
      mbar_init(smem_u32(&tempty[b]), 128);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(P::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    int it = 0;
    bool ok = !withhold_loads;  // test hook: no stage is ever filled, so the MMA
                                // issuer's first wait runs out its budget while
                                // no copy or MMA is in flight
    for (int sg = sbeg; sg < send && ok; ++sg) {
      const int4 seg = segs[sg];
      const int mt = seg.x / n_tiles_n, nt = seg.x % n_tiles_n;
      for (int kb = seg.y; kb < seg.z; ++kb, ++it) {
        const int s = it % STAGES;
        const uint32_t ph = (it / STAGES) & 1;
        if (!mbar_wait(smem_u32(&empty[s]), ph ^ 1, err)) {
          ok = false;
          // Error path: let the copies already issued into the ring land before
          // the CTA exits (bounded waits that ignore the error flag).
          for (int d = 1; d <= STAGES && it - d >= 0; ++d) {
            const int ps = (it - d) % STAGES;
            mbar_wait(smem_u32(&full[ps]), ((it - d) / STAGES) & 1, err, false);
          }
          break;
        }
        const uint32_t fb = smem_u32(&full[s]);
        mbar_expect_tx(fb, STAGE_BYTES);
        uint8_t* st = smem + s * STAGE_BYTES;
        tma_load_2d(&mA0, smem_u32(st), fb, kb * BK, mt * BM);
        tma_load_2d(&mA1, smem_u32(st + A_TILE), fb, kb * BK, mt * BM);
        if (NP == 3) tma_load_2d(&mA2, smem_u32(st + 2 * A_TILE), fb, kb * BK, mt * BM);
        tma_load_2d(&mB0, smem_u32(st + NP * A_TILE), fb, kb * BK, nt * TN);
        tma_load_2d(&mB1, smem_u32(st + NP * A_TILE + B_T), fb, kb * BK, nt * TN);
        if (NP == 3) tma_load_2d(&mB2, smem_u32(st + NP * A_TILE + 2 * B_T), fb, kb * BK, nt * TN);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    int it = 0, j = 0;
    bool ok = true;
    for (int sg = sbeg; sg < send && ok; ++sg, ++j) {
      const int4 seg = segs[sg];
      const int b = j & 1;
      const uint32_t jph = (j >> 1) & 1;
      if (!mbar_wait(smem_u32(&tempty[b]), jph ^ 1, err)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + static_cast<uint32_t>(b * TN);
      for (int kb = seg.y; kb < seg.z; ++kb, ++it) {
        const int s = it % STAGES;
        const uint32_t ph = (it / STAGES) & 1;
        if (!mbar_wait(smem_u32(&full[s]), ph, err)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(smem + s * STAGE_BYTES);
        const uint32_t b0 = a0 + NP * A_TILE;
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) {
          const uint32_t off = k * 32;  // 16 BF16 = 32 bytes along K inside the swizzle atom
          const uint64_t da0 = sw128_desc(a0 + off), da1 = sw128_desc(a0 + A_TILE + off);
          const uint64_t db0 = sw128_desc(b0 + off), db1 = sw128_desc(b0 + B_T + off);
          // products down to 2^-16 (two planes) or 2^-24 (three planes) of hi*hi
          umma_bf16(acc, da0, db0, P::IDESC, (kb > seg.y || k > 0) ? 1u : 0u);
          umma_bf16(acc, da0, db1, P::IDESC, 1u);
          umma_bf16(acc, da1, db0, P::IDESC, 1u);
          if (NP == 3) {
            const uint64_t da2 = sw128_desc(a0 + 2 * A_TILE + off);
            const uint64_t db2 = sw128_desc(b0 + 2 * B_T + off);
            umma_bf16(acc, da0, db2, P::IDESC, 1u);
            umma_bf16(acc, da2, db0, P::IDESC, 1u);
            umma_bf16(acc, da1, db1, P::IDESC, 1u);
          }
        }
        umma_commit(smem_u32(&empty[s]));
      }
      umma_commit(smem_u32(&tfull[b]));
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;  // TMEM lane quarter accessible to this warp
    int j = 0;
    for (int sg = sbeg; sg < send; ++sg, ++j) {
      const int b = j & 1;
      const uint32_t jph = (j >> 1) & 1;
      const bool ok = mbar_wait(smem_u32(&tfull[b]), jph, err);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float v[TN];
      const uint32_t base = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(b * TN);
#pragma unroll
      for (int c = 0; c < TN / 16; ++c) tmem_ld16(base + c * 16, v + c * 16);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(smem_u32(&tempty[b]));
      if (!ok) break;
      float* dst = part + static_cast<size_t>(sg) * TN * BM + q * 32 + lane;
#pragma unroll
      for (int c = 0; c < TN; ++c) dst[static_cast<size_t>(c) * BM] = v[c];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P::TMEM_COLS)
                 : "memory");
  }
}

// C[m + n*ldc] = alpha * sum_{segments of the tile} part + beta * C   (FP64)
constexpr int kReduceSplit = 8;

// tile_segs (when not null) lists each tile's segment ids in contraction
// order; otherwise a tile's segments are the consecutive ids s0 .. s1 - 1.
// skip_empty (upper-triangle plans, whose lower tiles are mirrored afterwards):
// tiles without segments are left as they are.
template <int TN>
__global__ void split_reduce_kernel(const float* __restrict__ part, const int* __restrict__ tile_seg,
                                    const int* __restrict__ tile_segs, int n_tiles_n, int M, int N,
                                    double alpha, double beta, double* __restrict__ C, int ldc,
                                    int skip_empty) {
  constexpr int BN = TN;
  // kReduceSplit blocks per tile, each covering BN / kReduceSplit columns.
  const int tile = blockIdx.x / kReduceSplit;
  const int part_idx = blockIdx.x % kReduceSplit;
  const int mt = tile / n_tiles_n, nt = tile % n_tiles_n;
  const int s0 = tile_seg[tile], s1 = tile_seg[tile + 1];
  if (skip_empty && s0 == s1) return;
  // four consecutive rows of one column per thread (16-byte partial loads),
  // the segments summed in contraction order
  const int e0 = part_idx * (BM * BN / kReduceSplit), e1 = e0 + BM * BN / kReduceSplit;
  for (int e = e0 + 4 * threadIdx.x; e < e1; e += 4 * blockDim.x) {
    const int mm = e % BM, nn = e / BM;
    const int m = mt * BM + mm, n = nt * BN + nn;
    if (m >= M || n >= N) continue;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const float* pc = part + static_cast<size_t>(nn) * BM + mm;
    for (int j = s0; j < s1; ++j) {
      const int s = tile_segs ? tile_segs[j] : j;
      const float4 v = *reinterpret_cast<const float4*>(pc + static_cast<size_t>(s) * BN * BM);
      acc[0] += static_cast<double>(v.x);
      acc[1] += static_cast<double>(v.y);
      acc[2] += static_cast<double>(v.z);
      acc[3] += static_cast<double>(v.w);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (m + u >= M) break;
      double* cp = C + m + u + static_cast<size_t>(n) * ldc;
      *cp = (beta == 0.0) ? alpha * acc[u] : alpha * acc[u] + beta * *cp;
    }
  }
}

// hi/lo split of a column-major FP64 matrix (rows x cols, ld) written as
// cols x ldo row-major BF16 pairs (row j = column j), zero padded to ldo.
// Two planes: hi = bf16(x), lo = bf16(x - hi).  Three planes (mid non-null):
// hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid).
__device__ __forceinline__ void split_value(double x, __nv_bfloat16& h, __nv_bfloat16* m, __nv_bfloat16& l) {
  h = __double2bfloat16(x);
  const double r = x - static_cast<double>(__bfloat162float(h));
  if (m) {
    *m = __double2bfloat16(r);
    l = __double2bfloat16(r - static_cast<double>(__bfloat162float(*m)));
  } else {
    l = __double2bfloat16(r);
  }
}

__global__ void split_cols_kernel(const double* __restrict__ X, int rows, int cols, int ld,
                                  __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                  int ldo, __nv_bfloat16* __restrict__ mid) {
  const size_t total = static_cast<size_t>(cols) * ldo;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t % ldo);
    const int j = static_cast<int>(t / ldo);
    double x = (i < rows) ? X[i + static_cast<size_t>(j) * ld] : 0.0;
    __nv_bfloat16 h, l, md;
    split_value(x, h, mid ? &md : nullptr, l);
    hi[t] = h;
    lo[t] = l;
    if (mid) mid[t] = md;
  }
}

// hi/lo split with transpose: X (rows x cols col-major, ld) -> rows x ldo
// row-major pairs (row i holds X[i, :]), columns [cols, wcols) written as zero
// padding (wcols <= ldo; a column chunk of a wider matrix writes just its
// columns).  32 x 32 tiles via smem.
// With `mean` the column means are subtracted (in FP64) before the split, so a
// single-precision or uncentred caller matrix is centred and split in one pass
// with the same values as centring an FP64 copy first.
template <typename T>
__global__ void split_rows_kernel(const T* __restrict__ X, int rows, int cols, int ld,
                                  __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                  int ldo, __nv_bfloat16* __restrict__ mid,
                                  const double* __restrict__ mean, int wcols) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + tx, j = j0 + r;
    double v = 0.0;
    if (i < rows && j < cols) {
      v = static_cast<double>(X[i + static_cast<size_t>(j) * ld]);
      if (mean) v -= mean[j];
    }
    tile[r][tx] = v;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + tx;
    if (i < rows && j < wcols) {
      const double x = tile[tx][r];
      __nv_bfloat16 h, l, md;
      split_value(x, h, mid ? &md : nullptr, l);
      hi[static_cast<size_t>(i) * ldo + j] = h;
      lo[static_cast<size_t>(i) * ldo + j] = l;
      if (mid) mid[static_cast<size_t>(i) * ldo + j] = md;
    }
  }
}


// The same split with TR x 64 tiles (TR rows of X, 64 columns): each warp reads
// columns of the tile as TR / 32 runs of 128 bytes, and writes rows of the
// planes as BF16 pairs (128 bytes per warp and plane).  Needs ldo and the
// column offset of hi / lo / mid even (4-byte pairs).
template <typename T, int TR>
__global__ void __launch_bounds__(256) split_rows_tile_kernel(const T* __restrict__ X, int rows, int cols, int ld,
                                                               __nv_bfloat16* __restrict__ hi,
                                                               __nv_bfloat16* __restrict__ lo, int ldo,
                                                               __nv_bfloat16* __restrict__ mid,
                                                               const double* __restrict__ mean, int wcols) {
  __shared__ T tile[64][TR + 1];   // tile[column][row] of the block
  const int i0 = blockIdx.y * TR, j0 = blockIdx.x * 64;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int jj = warp + 8 * c, j = j0 + jj;
    T v[TR / 32];
#pragma unroll
    for (int u = 0; u < TR / 32; ++u) v[u] = T(0);
    if (j < cols) {
      const T* col = X + static_cast<size_t>(j) * ld + i0;
#pragma unroll
      for (int u = 0; u < TR / 32; ++u)
        if (i0 + lane + 32 * u < rows) v[u] = col[lane + 32 * u];
    }
#pragma unroll
    for (int u = 0; u < TR / 32; ++u) tile[jj][lane + 32 * u] = v[u];
  }
  __syncthreads();
  const int jj = 2 * lane, j = j0 + jj;
  if (j >= wcols) return;
  const double m0 = (mean && j < cols) ? mean[j] : 0.0;
  const double m1 = (mean && j + 1 < cols) ? mean[j + 1] : 0.0;
  const bool pair = j + 1 < wcols;
#pragma unroll 4
  for (int r = 0; r < TR / 8; ++r) {
    const int ii = warp + 8 * r, i = i0 + ii;
    if (i >= rows) break;
    const double x0 = j < cols ? static_cast<double>(tile[jj][ii]) - m0 : 0.0;
    const double x1 = j + 1 < cols ? static_cast<double>(tile[jj + 1][ii]) - m1 : 0.0;
    __nv_bfloat16 h0, l0, d0, h1, l1, d1;
    split_value(x0, h0, mid ? &d0 : nullptr, l0);
    split_value(x1, h1, mid ? &d1 : nullptr, l1);
    const size_t o = static_cast<size_t>(i) * ldo + j;
    if (pair) {
      *reinterpret_cast<__nv_bfloat162*>(hi + o) = __halves2bfloat162(h0, h1);
      *reinterpret_cast<__nv_bfloat162*>(lo + o) = __halves2bfloat162(l0, l1);
      if (mid) *reinterpret_cast<__nv_bfloat162*>(mid + o) = __halves2bfloat162(d0, d1);
    } else {
      hi[o] = h0;
      lo[o] = l0;
      if (mid) mid[o] = d0;
    }
  }
}

// 2-D BF16 tensor map: `rows` rows of `k` elements, row pitch ld elements.
CUtensorMap make_map(const __nv_bfloat16* base, int rows, int k, int ld, int box_rows) {
  CUtensorMap m;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(kErrCuda, "cuTensorMapEncodeTiled failed");
  return m;
}

int round_up(int x, int a) { return (x + a - 1) / a * a; }

// BF16 planes of one operand (hi, lo and, with three planes, mid), each
// rows x ld K-contiguous, stored one after the other.
struct SplitPair {
  __nv_bfloat16* hi = nullptr;
  __nv_bfloat16* lo = nullptr;
  __nv_bfloat16* mid = nullptr;
  int rows = 0, k = 0, ld = 0, np = 2;
};

SplitPair pair_at(__nv_bfloat16* base, int rows, int k, int np = 2) {
  SplitPair s;
  s.rows = rows;
  s.k = k;
  s.np = np;
  s.ld = round_up(std::max(k, 1), BK);
  s.hi = base;
  s.lo = base + static_cast<size_t>(rows) * s.ld;
  if (np == 3) s.mid = base + 2 * static_cast<size_t>(rows) * s.ld;
  return s;
}

size_t pair_elems(int rows, int k, int np = 2) {
  return np * static_cast<size_t>(rows) * round_up(std::max(k, 1), BK);
}

SplitPair alloc_pair(int rows, int k, int np = 2) {
  return pair_at(Context::get().arena.alloc_n<__nv_bfloat16>(pair_elems(rows, k, np)), rows, k, np);
}

// Stream-K work plan: CTA c covers iterations [c*total/ctas, (c+1)*total/ctas)
// of the (tile, K block) space, cut into per-tile segments.
struct GemmPlan {
  int tiles = 0, ntn = 0, ctas = 0;
  int bn = BN;   // output tile width (64, or 128 for symmetric products)
  std::vector<int4> segs;
  std::vector<int> cta_begin, tile_begin;
  // Segment ids of each tile (tile t: tile_segs[tile_begin[t] .. tile_begin[t+1])),
  // in contraction order; empty when the segments are already grouped by tile.
  std::vector<int> tile_segs;
};

// Stream-K plan over the output tiles.  With `upper` only the tiles that
// reach the upper triangle (tile row start < tile column end) are planned, for
// symmetric products whose lower triangle is mirrored afterwards.
constexpr int kSymSegBlocks = 16;
// Segments of the symmetric (row Gram) plan: 32 K-blocks (2048 terms in FP32;
// sqrt(2) more rounding than 16 blocks, still far below the BF16 split error)
// halve the FP32 partials written and summed.
constexpr int kGramSegBlocks = 32;
constexpr int kSymChunkBlocks = 64;   // K-blocks per chunk of a symmetric plan (a multiple of kGramSegBlocks)
// Products that take the split path in the mixed precision mode.
constexpr int kMixedMinK = 256;
constexpr double kMixedMinWork = 1e7;

GemmPlan plan_gemm(int M, int N, int K, int sm_count, bool upper = false, bool short_segments = false,
                   int bn = BN) {
  GemmPlan g;
  g.bn = bn;
  const int mt = (M + BM - 1) / BM;
  g.ntn = (N + bn - 1) / bn;
  g.tiles = mt * g.ntn;
  std::vector<int> inc;
  inc.reserve(g.tiles);
  for (int t = 0; t < g.tiles; ++t)
    if (!upper || (t / g.ntn) * BM < ((t % g.ntn) + 1) * bn) inc.push_back(t);
  const int kbt = (K + BK - 1) / BK;
  // A symmetric (Gram) product sums the whole contraction of each tile in one
  // CTA; cutting it into segments of at most kGramSegBlocks K-blocks (every
  // three-plane product into kSymSegBlocks) keeps each FP32 accumulation short
  // and adds the segments in FP64.
  const int kseg = upper ? kGramSegBlocks : (short_segments ? kSymSegBlocks : kbt);
  const long long total = static_cast<long long>(inc.size()) * kbt;
  g.ctas = static_cast<int>(std::max<long long>(1, std::min<long long>(sm_count, total)));
  g.cta_begin.assign(g.ctas + 1, 0);
  g.tile_begin.assign(g.tiles + 1, 0);
  // A symmetric plan walks the contraction in chunks of kSymChunkBlocks
  // K-blocks and gives every CTA an equal share of each chunk, chunk after
  // chunk, so that the CTAs running at the same time read the same K-panel of
  // both operands (it stays in L2) instead of the whole operands.
  const int kc = upper ? kSymChunkBlocks : kbt;
  const int nchunks = (kbt + kc - 1) / kc;
  const long long ninc = static_cast<long long>(inc.size());
  for (int c = 0; c < g.ctas; ++c) {
    g.cta_begin[c] = static_cast<int>(g.segs.size());
    for (int q = 0; q < nchunks; ++q) {
      const int w = std::min(kc, kbt - q * kc);
      const long long tq = ninc * w;   // (tile, K block) pairs of chunk q
      long long a = tq * c / g.ctas, e = tq * (c + 1) / g.ctas;
      while (a < e) {
        const int t = inc[static_cast<size_t>(a / w)];
        const int kb0 = q * kc + static_cast<int>(a % w);
        int kb1 = static_cast<int>(std::min<long long>(q * kc + w, kb0 + (e - a)));
        kb1 = std::min(kb1, (kb0 / kseg + 1) * kseg);
        g.segs.push_back(make_int4(t, kb0, kb1, 0));
        a += kb1 - kb0;
      }
    }
  }
  g.cta_begin[g.ctas] = static_cast<int>(g.segs.size());
  if (kc == kbt) {
    int s = 0;
    for (int t = 0; t < g.tiles; ++t) {
      g.tile_begin[t] = s;
      while (s < static_cast<int>(g.segs.size()) && g.segs[s].x == t) ++s;
    }
    g.tile_begin[g.tiles] = s;
  } else {
    // group the segment ids by tile, each tile's in contraction order
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
  }
  return g;
}

// Number of output tiles that received at least one segment.
int planned_tiles(const GemmPlan& g) {
  int c = 0;
  for (int t = 0; t < g.tiles; ++t) c += g.tile_begin[t + 1] > g.tile_begin[t];
  return c;
}

// True when the plan skips tiles (a symmetric, upper-triangle plan).
bool upper_hint(const GemmPlan& g) { return planned_tiles(g) < g.tiles; }

// Device scratch of one GEMM: segment tables and the FP32 stream-K partials.
struct GemmScratch {
  int4* segs = nullptr;
  int* cta_begin = nullptr;
  int* tile_begin = nullptr;
  int* tile_segs = nullptr;   // null when the plan has no per-tile segment list
  float* part = nullptr;
};

size_t gemm_scratch_bytes(const GemmPlan& g) {
  auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  return up(g.segs.size() * sizeof(int4)) + up(g.cta_begin.size() * sizeof(int)) +
         up(g.tile_begin.size() * sizeof(int)) + up(g.tile_segs.size() * sizeof(int)) +
         up(g.segs.size() * static_cast<size_t>(BM) * g.bn * sizeof(float));
}

GemmScratch carve_gemm_scratch(const GemmPlan& g, char* base) {
  auto up = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  GemmScratch s;
  s.segs = reinterpret_cast<int4*>(base);
  base += up(g.segs.size() * sizeof(int4));
  s.cta_begin = reinterpret_cast<int*>(base);
  base += up(g.cta_begin.size() * sizeof(int));
  s.tile_begin = reinterpret_cast<int*>(base);
  base += up(g.tile_begin.size() * sizeof(int));
  if (!g.tile_segs.empty()) {
    s.tile_segs = reinterpret_cast<int*>(base);
    base += up(g.tile_segs.size() * sizeof(int));
  }
  s.part = reinterpret_cast<float*>(base);
  return s;
}

template <int NP, int TN>
void ensure_smem_attr() {
  // The attribute applies to the device current when it is set: one flag per device.
  static std::atomic<bool> attr[64];
  int dev = 0;
  FPLS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    FPLS_CUDA(cudaFuncSetAttribute(split_gemm_kernel<NP, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   Planes<NP, TN>::SMEM_BYTES));
    return;
  }
  if (!attr[dev].load(std::memory_order_acquire)) {
    FPLS_CUDA(cudaFuncSetAttribute(split_gemm_kernel<NP, TN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   Planes<NP, TN>::SMEM_BYTES));
    attr[dev].store(true, std::memory_order_release);
  }
}

template <int NP, int TN>
void launch_split_kernel(const CUtensorMap (&m)[6], const GemmPlan& g, const GemmScratch& s, int* err,
                         cudaStream_t st) {
  ensure_smem_attr<NP, TN>();
  // FASTPLS_TEST_WITHHOLD_LOADS=1 (tests of the timeout path only): the
  // producer issues no load, the pipeline's bounded wait expires and the call
  // returns FPLS_ERR_CUDA with the tensor memory released.
  const char* w = std::getenv("FASTPLS_TEST_WITHHOLD_LOADS");
  const int withhold = (w && w[0] == '1') ? 1 : 0;
  split_gemm_kernel<NP, TN><<<g.ctas, NUM_THREADS, Planes<NP, TN>::SMEM_BYTES, st>>>(
      m[0], m[1], m[2], m[3], m[4], m[5], s.segs, s.cta_begin, g.ntn, s.part, err, withhold);
}

// C (M x N) = alpha * A B^T + beta C on stream `st` with the given scratch; no allocation.
void upload_plan_tables(const GemmPlan& g, const GemmScratch& s, cudaStream_t st) {
  FPLS_CUDA(cudaMemcpyAsync(s.segs, g.segs.data(), g.segs.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  FPLS_CUDA(cudaMemcpyAsync(s.cta_begin, g.cta_begin.data(), g.cta_begin.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  FPLS_CUDA(cudaMemcpyAsync(s.tile_begin, g.tile_begin.data(), g.tile_begin.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  if (!g.tile_segs.empty())
    FPLS_CUDA(cudaMemcpyAsync(s.tile_segs, g.tile_segs.data(), g.tile_segs.size() * sizeof(int), cudaMemcpyHostToDevice,
                              st));
}

// Launches the GEMM and its reduction; the plan tables must already be in `s`.
void split_gemm_run(const SplitPair& A, const SplitPair& B, int M, int N, int K, double alpha,
                    double beta, double* C, int ldc, const GemmPlan& g, const GemmScratch& s,
                    int* err, cudaStream_t st, Context* prof) {
  FPLS_REQUIRE(A.np == B.np && (A.np == 2 || A.np == 3), "split GEMM: operands with different plane counts");
  FPLS_REQUIRE(g.bn == BN || g.bn == BN_SYM, "split GEMM: unsupported tile width");
  const CUtensorMap maps[6] = {make_map(A.hi, M, K, A.ld, BM),
                               make_map(A.np == 3 ? A.mid : A.lo, M, K, A.ld, BM),
                               make_map(A.lo, M, K, A.ld, BM),
                               make_map(B.hi, N, K, B.ld, g.bn),
                               make_map(B.np == 3 ? B.mid : B.lo, N, K, B.ld, g.bn),
                               make_map(B.lo, N, K, B.ld, g.bn)};
  const bool upper_plan = g.tiles > 0 && static_cast<int>(g.tile_begin.size()) == g.tiles + 1 &&
                          g.tile_begin[g.tiles] > 0 && upper_hint(g);
  const int slot = prof ? prof->prof_begin(upper_plan ? (A.np == 3 ? "gram_bf16x6" : "gram_bf16x3")
                                                      : (A.np == 3 ? "split_gemm_bf16x6" : "split_gemm_bf16x3"),
                                           st)
                        : -1;
  if (A.np == 3) {
    if (g.bn == BN_SYM) launch_split_kernel<3, BN_SYM>(maps, g, s, err, st);
    else launch_split_kernel<3, BN>(maps, g, s, err, st);
  } else if (g.bn == BN_SYM) {
    launch_split_kernel<2, BN_SYM>(maps, g, s, err, st);
  } else {
    launch_split_kernel<2, BN>(maps, g, s, err, st);
  }
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  if (prof) {
    // Algorithmic bytes: every BF16 plane of A and B once, the FP64 result once;
    // flops: three (two planes) or six (three planes) products over the planned tiles.
    const double tiles_frac = static_cast<double>(planned_tiles(g)) / g.tiles;
    const double planes = A.np, products = A.np == 3 ? 6.0 : 3.0;
    prof->prof_end(slot, st,
                   2.0 * planes * (static_cast<double>(M) * K + static_cast<double>(N) * K) +
                       8.0 * static_cast<double>(M) * N * tiles_frac,
                   products * 2.0 * static_cast<double>(M) * N * K * tiles_frac);
  }
  if (g.bn == BN_SYM)
    split_reduce_kernel<BN_SYM><<<g.tiles * kReduceSplit, 256, 0, st>>>(s.part, s.tile_begin, s.tile_segs, g.ntn, M, N,
                                                                         alpha, beta, C, ldc, upper_plan ? 1 : 0);
  else
    split_reduce_kernel<BN><<<g.tiles * kReduceSplit, 256, 0, st>>>(s.part, s.tile_begin, s.tile_segs, g.ntn, M, N,
                                                                     alpha, beta, C, ldc, upper_plan ? 1 : 0);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

// Plans (with their device tables and partial buffers) are kept per GEMM shape
// so that the repeated products of the SIMPLS loop issue no host-to-device copy
// (a pageable copy would synchronise the stream on every call).
struct CachedPlan {
  GemmPlan g;
  char* dev = nullptr;
  GemmScratch s;
};
std::map<std::array<int, 7>, CachedPlan>& plan_cache() {
  static std::map<std::array<int, 7>, CachedPlan> cache;
  return cache;
}

const CachedPlan& cached_plan(int M, int N, int K, int sm_count, cudaStream_t st, bool upper = false,
                              bool short_segments = false, int bn = BN) {
  auto& cache = plan_cache();
  const std::array<int, 7> key{M, N, K, sm_count, upper ? 1 : 0, short_segments ? 1 : 0, bn};
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  CachedPlan c;
  c.g = plan_gemm(M, N, K, sm_count, upper, short_segments, bn);
  FPLS_CUDA(cudaMalloc(&c.dev, gemm_scratch_bytes(c.g)));
  c.s = carve_gemm_scratch(c.g, c.dev);
  upload_plan_tables(c.g, c.s, st);
  return cache.emplace(key, std::move(c)).first->second;
}

// General products with at least this many rows and columns run on 128 x 128
// tiles (FASTPLS_WIDE_TILES=0: 128 x 64): twice the multiply-adds per operand
// byte of the 128 x 64 tiles, which the fat predictor-by-response products
// (X^T Y of the OPLS filter: 20000 x 5000 over 50000 rows) are bound by.
constexpr int kWideMinM = 2048, kWideMinN = 512;
bool general_wide_tiles(int M, int N) {
  static const int v = [] {
    const char* e = std::getenv("FASTPLS_WIDE_TILES");
    return (e && e[0] == '0') ? 0 : 1;
  }();
  return v && M >= kWideMinM && N >= kWideMinN;
}

bool sym_wide_tiles() {
  if (const char* e = std::getenv("FASTPLS_GRAM_TILE")) return std::string(e) != "64";
  return active_tune().gram_tile != 64;
}

void split_gemm(const SplitPair& A, const SplitPair& B, int M, int N, int K, double alpha,
                double beta, double* C, int ldc, bool upper = false) {
  Context& ctx = Context::get();
  // Symmetric two-plane products (the row Gram) on 128 x 128 tiles: half the
  // B re-reads of the 128 x 64 tiles and twice the MACs per operand byte read
  // by the tensor core.
  const int bn = ((upper && A.np == 2 && sym_wide_tiles()) || (!upper && general_wide_tiles(M, N))) ? BN_SYM : BN;
  const CachedPlan& c = cached_plan(M, N, K, ctx.sm_count, ctx.stream, upper, A.np == 3, bn);
  split_gemm_run(A, B, M, N, K, alpha, beta, C, ldc, c.g, c.s, ctx.d_status + 16, ctx.stream,
                 ctx.profile ? &ctx : nullptr);
}

// Block (ti, tj), ti <= tj, reads the upper 32 x 32 tile (rows ti, columns tj)
// with column reads, and writes its transpose into the lower tile (rows tj,
// columns ti) with column writes; a diagonal block writes only below the
// diagonal.  Blocks below the diagonal have nothing to do.
__global__ void __launch_bounds__(256) mirror_upper_kernel(double* K, int n) {
  __shared__ double t[32][33];
  const int ti = blockIdx.x, tj = blockIdx.y;
  if (ti > tj) return;
  const int x = threadIdx.x & 31, y0 = threadIdx.x >> 5;
  for (int y = y0; y < 32; y += 8) {
    const int r = ti * 32 + x, c = tj * 32 + y;
    if (r < n && c < n) t[y][x] = K[r + static_cast<size_t>(c) * n];
  }
  __syncthreads();
  for (int y = y0; y < 32; y += 8) {
    const int r = tj * 32 + x, c = ti * 32 + y;   // lower entry (r, c) = upper entry (c, r)
    if (r < n && c < n && r > c) K[r + static_cast<size_t>(c) * n] = t[x][y];
  }
}

// K[i, j] = K[j, i] for i > j (n x n).
void mirror_upper(double* K, int n) {
  Context& ctx = Context::get();
  const int nt = (n + 31) / 32;
  mirror_upper_kernel<<<dim3(nt, nt), 256, 0, ctx.stream>>>(K, n); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void split_cols_on(const double* X, int rows, int cols, int ld, const SplitPair& out, cudaStream_t st,
                   int sm_count) {
  split_cols_kernel<<<4 * sm_count, 256, 0, st>>>(X, rows, cols, ld, out.hi, out.lo, out.ld, out.mid); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

template <typename T>
void split_rows_on(const T* X, int rows, int cols, int ld, const SplitPair& out, cudaStream_t st,
                   const double* mean = nullptr, int col0 = 0, int wcols = -1) {
  if (wcols < 0) wcols = out.ld - col0;
  if (((out.ld | col0) & 1) == 0) {
    // 128-row tiles for FP32 (33 KB of shared memory), 64-row tiles for FP64
    constexpr int TR = sizeof(T) == 4 ? 128 : 64;
    dim3 grid((wcols + 63) / 64, (rows + TR - 1) / TR);
    split_rows_tile_kernel<T, TR><<<grid, 256, 0, st>>>(X, rows, cols, ld, out.hi + col0, out.lo + col0, out.ld,
                                                        out.mid ? out.mid + col0 : nullptr, mean, wcols);
  } else {
    dim3 grid((wcols + 31) / 32, (rows + 31) / 32);
    split_rows_kernel<T><<<grid, dim3(32, 8), 0, st>>>(X, rows, cols, ld, out.hi + col0, out.lo + col0, out.ld,
                                                       out.mid ? out.mid + col0 : nullptr, mean, wcols);
  }
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void split_cols(const double* X, int rows, int cols, int ld, const SplitPair& out) {
  Context& ctx = Context::get();
  split_cols_on(X, rows, cols, ld, out, ctx.stream, ctx.sm_count);
}

void split_rows(const double* X, int rows, int cols, int ld, const SplitPair& out) {
  split_rows_on(X, rows, cols, ld, out, Context::get().stream);
}

struct XOperatorSplit : public XOperator {
  SplitPair xr;   // n x p  (A of X * R)
  SplitPair xc;   // p x n  (A of X^T * T)
  bool has_t = true;
  int np = 2;
  XOperatorSplit(const double* X, int n_, int p_, bool need_t, int np_) : has_t(need_t), np(np_) {
    n = n_;
    p = p_;
    xr = alloc_pair(n, p, np);
    split_rows(X, n, p, n, xr);
    if (has_t) {
      xc = alloc_pair(p, n, np);
      split_cols(X, n, p, n, xc);
    }
  }
  // Row-major planes only, split straight from the caller's matrix with the
  // column means (or none) subtracted on the way.
  template <typename T>
  XOperatorSplit(const T* X, const double* mean, int n_, int p_, int np_) : has_t(false), np(np_) {
    n = n_;
    p = p_;
    xr = alloc_pair(n, p, np);
    split_rows_on(X, n, p, n, xr, Context::get().stream, mean);
  }
  // Row-major planes allocated only; filled column chunk by column chunk.
  XOperatorSplit(int n_, int p_, int np_) : has_t(false), np(np_) {
    n = n_;
    p = p_;
    xr = alloc_pair(n, p, np);
  }
  // Columns [j0, j1) of the planes from the chunk X (n x (j1 - j0), ld n) minus
  // mean[0 .. j1-j0) (or nothing); the last chunk also writes the zero padding.
  template <typename T>
  void fill_columns(const T* X, const double* mean, int j0, int j1) {
    const int w = (j1 >= p) ? xr.ld - j0 : j1 - j0;
    split_rows_on(X, n, j1 - j0, n, xr, Context::get().stream, mean, j0, w);
  }
  // K (upper tiles) = Xc[:, j0:j1] Xc[:, j0:j1]^T, added to K when accumulate.
  void gram_columns(double* K, int j0, int j1, bool accumulate) {
    SplitPair v = xr;
    v.hi = xr.hi + j0;
    v.lo = xr.lo + j0;
    if (v.mid) v.mid = xr.mid + j0;
    v.k = j1 - j0;
    split_gemm(v, v, n, n, j1 - j0, 1.0, accumulate ? 1.0 : 0.0, K, n, true);
  }
  void times(const double* Rhat, int F, double* U) override {
    SplitPair b = alloc_pair(F, p, np);
    split_cols(Rhat, p, F, p, b);
    split_gemm(xr, b, n, F, p, 1.0, 0.0, U, n);
  }
  void gram(double* K) override {
    // upper-triangle tiles only; the lower triangle is mirrored
    split_gemm(xr, xr, n, n, p, 1.0, 0.0, K, n, true);
    mirror_upper(K, n);
  }
  void t_times(const double* T, int F, double* P) override {
    FPLS_REQUIRE(has_t, "split operator built without its transposed copy");
    SplitPair b = alloc_pair(F, n, np);
    split_cols(T, n, F, n, b);
    split_gemm(xc, b, p, F, n, 1.0, 0.0, P, p);
  }
};

}  // namespace

void xgemm(bool transA, int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
           int ldc) {
  Context& ctx = Context::get();
  const bool mixed = ctx.precision >= 1 && K >= kMixedMinK &&
                     static_cast<double>(M) * N * K >= kMixedMinWork;
  const int np = ctx.precision == 2 ? 3 : 2;
  if (!mixed) {
    gemm(transA, false, M, N, K, 1.0, A, lda, B, ldb, 0.0, C, ldc);
    return;
  }
  // A operand as M x K K-contiguous rows: op(A) = A (M x K col-major) needs
  // the row split, op(A) = A^T (A is K x M) is already K-contiguous per row.
  SplitPair a = alloc_pair(M, K, np);
  if (transA) split_cols(A, K, M, lda, a);
  else split_rows(A, M, K, lda, a);
  SplitPair b = alloc_pair(N, K, np);
  split_cols(B, K, N, ldb, b);
  split_gemm(a, b, M, N, K, 1.0, 0.0, C, ldc);
}

void split_gemm_release_cache() {
  for (auto& kv : plan_cache()) cudaFree(kv.second.dev);
  plan_cache().clear();
}

std::unique_ptr<XOperator> make_split_operator(const double* X, int n, int p, bool need_t, int planes) {
  return std::unique_ptr<XOperator>(new XOperatorSplit(X, n, p, need_t, planes));
}

std::unique_ptr<XOperator> make_split_operator_chunked(int n, int p, int planes) {
  return std::unique_ptr<XOperator>(new XOperatorSplit(n, p, planes));
}

void split_operator_fill_columns(XOperator& op, const double* x64, const float* x32, const double* mean, int j0,
                                 int j1) {
  auto* sp = dynamic_cast<XOperatorSplit*>(&op);
  FPLS_REQUIRE(sp != nullptr, "column chunks need the split operator");
  FPLS_REQUIRE(j0 % 8 == 0 && j0 >= 0 && j1 > j0 && j1 <= sp->p, "column chunk out of range");
  if (x64) sp->fill_columns(x64, mean, j0, j1);
  else sp->fill_columns(x32, mean, j0, j1);
}

void split_operator_gram_columns(XOperator& op, double* K, int j0, int j1, bool accumulate) {
  auto* sp = dynamic_cast<XOperatorSplit*>(&op);
  FPLS_REQUIRE(sp != nullptr, "column chunks need the split operator");
  FPLS_REQUIRE(j0 % 8 == 0 && j0 >= 0 && j1 > j0 && j1 <= sp->p, "column chunk out of range");
  sp->gram_columns(K, j0, j1, accumulate);
}

void mirror_upper_triangle(double* K, int n) { mirror_upper(K, n); }

std::unique_ptr<XOperator> make_split_operator_centered(const double* x64, const float* x32, const double* mean,
                                                        int n, int p, int planes) {
  if (x64) return std::unique_ptr<XOperator>(new XOperatorSplit(x64, mean, n, p, planes));
  return std::unique_ptr<XOperator>(new XOperatorSplit(x32, mean, n, p, planes));
}

void split_gemm_test(const double* A, const double* B, int M, int N, int K, double* C) {
  // A: M x K col-major, B: K x N col-major; C = A B.
  SplitPair a = alloc_pair(M, K);
  SplitPair b = alloc_pair(N, K);
  split_rows(A, M, K, M, a);
  split_cols(B, K, N, K, b);
  split_gemm(a, b, M, N, K, 1.0, 0.0, C, M);
}

size_t split_gemm_scratch_need(int M, int N, int K, int sm_count) {
  const GemmPlan g = plan_gemm(M, N, K, sm_count);
  return 2 * (pair_elems(M, K) + pair_elems(N, K)) + gemm_scratch_bytes(g) + 256;
}

void split_gemm_in_scratch(const double* A, const double* B, int M, int N, int K, double* C,
                           void* scratch, size_t scratch_bytes, int* err, cudaStream_t st,
                           int sm_count) {
  const GemmPlan g = plan_gemm(M, N, K, sm_count);
  const size_t need = 2 * (pair_elems(M, K) + pair_elems(N, K)) + gemm_scratch_bytes(g) + 256;
  if (need > scratch_bytes) throw Error(kErrArgument, "split GEMM shape exceeds the fixed scratch size");
  char* base = static_cast<char*>(scratch);
  SplitPair a = pair_at(reinterpret_cast<__nv_bfloat16*>(base), M, K);
  base += 2 * pair_elems(M, K);
  SplitPair b = pair_at(reinterpret_cast<__nv_bfloat16*>(base), N, K);
  base += 2 * pair_elems(N, K);
  base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(base) + 255) & ~static_cast<uintptr_t>(255));
  split_rows_on(A, M, K, M, a, st);
  split_cols_on(B, K, N, K, b, st, sm_count);
  const GemmScratch gs = carve_gemm_scratch(g, base);
  upload_plan_tables(g, gs, st);
  split_gemm_run(a, b, M, N, K, 1.0, 0.0, C, M, g, gs, err, st, nullptr);
}

}  // namespace fpls
