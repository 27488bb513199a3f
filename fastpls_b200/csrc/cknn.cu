// Candidate-kNN classifier on the device: latent score space, class centroids,
// candidate classes by centroid similarity, and the smoothed class-kNN rerank.
//
// Reference behaviour (R package fastPLS):
//   score space / row L2 / centroids   R/main.R:657-730
//   candidate_knn_predict_cuda         src/fastPLS.cpp:1653-1711 -> 1322-1467
//   per-(row, candidate) class kNN     src/lda_cuda_kernels.cu:180-243 (at most
//                                      32 neighbour similarities are kept)
//
// The reference scores every (test row, candidate class) pair with one thread
// that walks the whole class serially.  Here the pairs are grouped by class:
// for each class the test rows that list it as a candidate form 64-row tiles,
// the class's training rows (gathered class-contiguous, row-major) are cut into
// chunks, and one CTA computes the 64 x 64 similarity tiles of a (class, tile,
// chunk) item with FP64 tensor-core MMA, folding each tile into per-row top-k
// lists held in shared memory.  A merge pass combines the chunk lists of a pair
// and applies the smoothed score; a rerank pass keeps the top classes.
#include "../../include/fastpls_b200.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <limits>
#include <vector>

#include <cuda_bf16.h>

#include "blas_f64.cuh"
#include "capi_util.cuh"
#include "cknn.cuh"
#include "context.cuh"
#include "tc_util.cuh"

namespace fpls {
namespace {

constexpr int kKnnMax = 32;      // neighbour list cap of the replaced CUDA scorer
constexpr int kTileM = 64;       // test rows per tile
constexpr int kTileN = 64;       // training rows per similarity tile
constexpr int kBK = 16;
constexpr int kPad = 4;
constexpr int kTileThreads = 128;
constexpr int kMaxChunks = 64;   // chunk lists merged per pair
constexpr int kMinChunkRows = 2048;

// Strict '>' insertion into a descending list of length k (earlier entries win
// ties), list entries strided by `stride` (src/fastPLS.cpp:1249-1267).
template <typename V, typename I>
__device__ __forceinline__ void insert_desc(V* vals, I* idx, int k, size_t stride, V v, I id) {
  if (!(v > vals[(size_t)(k - 1) * stride])) return;
  int j = 0;
  while (!(v > vals[(size_t)j * stride])) ++j;
  for (int h = k - 1; h > j; --h) {
    vals[(size_t)h * stride] = vals[(size_t)(h - 1) * stride];
    if (idx) idx[(size_t)h * stride] = idx[(size_t)(h - 1) * stride];
  }
  vals[(size_t)j * stride] = v;
  if (idx) idx[(size_t)j * stride] = id;
}

// ---------------------------------------------------------------- fit side

// Tn = row_l2(T Ck) or row_l2(T); zero / non-finite row norms become 1
// (R/main.R:657-662).  One thread per row, sums in column order.
__global__ void row_l2_kernel(const double* __restrict__ A, int n, int k, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < k; ++j) {
    const double v = A[i + (size_t)j * n];
    s += v * v;
  }
  double nr = sqrt(s);
  if (!isfinite(nr) || nr == 0.0) nr = 1.0;
  for (int j = 0; j < k; ++j) out[i + (size_t)j * n] = A[i + (size_t)j * n] / nr;
}

__global__ void class_hist_kernel(const int* __restrict__ codes, int n, int C, int* counts) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = codes[i];
    if (c >= 1 && c <= C) atomicAdd(counts + (c - 1), 1);
  }
}

// dest[i] = slot of row i in class-contiguous order (-1 for codes outside 1..C).
__global__ void class_slot_kernel(const int* __restrict__ codes, int n, int C,
                                  const int* __restrict__ offs, int* cursor, int* dest) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = codes[i];
    dest[i] = (c >= 1 && c <= C) ? offs[c - 1] + atomicAdd(cursor + (c - 1), 1) : -1;
  }
}

// Column-major A (n x k) -> row-major rows out[dest[i] * k + j] (rows with
// dest < 0 dropped); dest == null keeps the order.  32 x 32 tiles through
// shared memory so both sides are coalesced.
__global__ void transpose_scatter_kernel(const double* __restrict__ A, int n, int k,
                                         const int* __restrict__ dest, double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (i < n && j < k) tile[r][threadIdx.x] = A[i + (size_t)j * n];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (i < n && j < k) {
      const int d = dest ? dest[i] : i;
      if (d >= 0) out[(size_t)d * k + j] = tile[threadIdx.x][r];
    }
  }
}

// Class sums of class-contiguous row-major rows (R/main.R:686-698): each CTA
// walks a fixed range of rows, locating its first class by binary search in
// the class offsets; each thread keeps up to 4 column sums in registers and
// flushes them (atomicAdd into sums, C x k column-major) at class boundaries,
// so a very large class is spread over many CTAs.
constexpr int kCentCols = 4;
__global__ void __launch_bounds__(128) class_rowsum_kernel(const double* __restrict__ Ts, int k, int nrows,
                                                           const int* __restrict__ offs, int C, int rows,
                                                           int col0, double* __restrict__ sums) {
  const int s0 = blockIdx.x * rows;
  const int s1 = min(nrows, s0 + rows);
  int lo = 0, hi = C - 1;  // last class with offs[c] <= s0
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (offs[mid] <= s0) lo = mid; else hi = mid - 1;
  }
  int c = lo;
  int cend = offs[c + 1];
  int jc[kCentCols];
  double acc[kCentCols];
#pragma unroll
  for (int u = 0; u < kCentCols; ++u) {
    jc[u] = col0 + threadIdx.x + u * blockDim.x;
    acc[u] = 0.0;
  }
  for (int r = s0; r < s1; ++r) {
    if (r >= cend) {
#pragma unroll
      for (int u = 0; u < kCentCols; ++u) {
        if (jc[u] < k) atomicAdd(sums + c + (size_t)jc[u] * C, acc[u]);
        acc[u] = 0.0;
      }
      while (r >= offs[c + 1]) ++c;
      cend = offs[c + 1];
    }
    const double* row = Ts + (size_t)r * k;
#pragma unroll
    for (int u = 0; u < kCentCols; ++u)
      if (jc[u] < k) acc[u] += __ldg(row + jc[u]);
  }
#pragma unroll
  for (int u = 0; u < kCentCols; ++u)
    if (jc[u] < k) atomicAdd(sums + c + (size_t)jc[u] * C, acc[u]);
}

// centroid = row_l2(sums / max(count, 1)); one thread per class.
__global__ void centroid_finish_kernel(const double* __restrict__ sums, int k, const int* __restrict__ offs,
                                       int C, double* __restrict__ cent) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  const int cnt = offs[c + 1] - offs[c];
  const double den = cnt > 0 ? (double)cnt : 1.0;
  double sq = 0.0;
  for (int j = 0; j < k; ++j) {
    const double t = sums[c + (size_t)j * C] / den;
    sq += t * t;
  }
  double nr = sqrt(sq);
  if (!isfinite(nr) || nr == 0.0) nr = 1.0;
  for (int j = 0; j < k; ++j) cent[c + (size_t)j * C] = (sums[c + (size_t)j * C] / den) / nr;
}

// ---------------------------------------------------------------- predict side

// Top-m classes of each test row by centroid similarity (insertion order of
// src/fastPLS.cpp:1401-1415): cand = class code (1-based) or -1.
__global__ void select_candidates_kernel(const double* __restrict__ base, int ntest, int C, int top_m,
                                         int* __restrict__ cand, double* __restrict__ cbase) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntest) return;
  double* vals = cbase + i;
  int* idx = cand + i;
  for (int j = 0; j < top_m; ++j) {
    vals[(size_t)j * ntest] = -INFINITY;
    idx[(size_t)j * ntest] = -1;
  }
  for (int c = 0; c < C; ++c)
    insert_desc(vals, idx, top_m, (size_t)ntest, base[i + (size_t)c * ntest], c + 1);
}

__global__ void pair_hist_kernel(const int* __restrict__ cand, long long npairs, int C, int* counts) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    const int c = cand[p];
    if (c >= 1 && c <= C) atomicAdd(counts + (c - 1), 1);
  }
}

// pairs[slot] = flat (row + slot_j * ntest) index into the candidate matrix.
__global__ void pair_scatter_kernel(const int* __restrict__ cand, long long npairs, int C,
                                    const int* __restrict__ offs, int* cursor, int* pairs) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    const int c = cand[p];
    if (c >= 1 && c <= C) pairs[offs[c - 1] + atomicAdd(cursor + (c - 1), 1)] = (int)p;
  }
}

struct KnnItem {
  int cls;    // 0-based class
  int tile;   // 64-pair tile within the class's pair list
  int chunk;  // training-row chunk within the class
  int pad;
};

struct KnnClassInfo {
  const int* row_offs;         // C + 1 class-contiguous training row offsets
  const int* pair_offs;        // C + 1 class-sorted pair offsets
  const int* chunk_rows;       // C rows per chunk
  const int* nchunks;          // C
  const long long* part_base;  // C partial-list base offsets (in doubles)
};

// One (class, 64-pair tile, training chunk) item: 64 x 64 FP64 MMA similarity
// tiles over the chunk, folded into per-row top-k lists (two half-row lists
// per test row, merged at the end) and written as one sorted list per pair.
__global__ void __launch_bounds__(kTileThreads)
knn_tile_kernel(const KnnItem* __restrict__ items, KnnClassInfo ci, const int* __restrict__ pairs,
                int ntest, const double* __restrict__ Tq, const double* __restrict__ Ts, int K,
                int use_k, double* __restrict__ part) {
  extern __shared__ double smem[];
  double (*As)[kBK][kTileM + kPad] = reinterpret_cast<double (*)[kBK][kTileM + kPad]>(smem);
  double (*Bs)[kBK][kTileN + kPad] =
      reinterpret_cast<double (*)[kBK][kTileN + kPad]>(smem + 2 * kBK * (kTileM + kPad));
  double (*sim)[kTileN + 1] =
      reinterpret_cast<double (*)[kTileN + 1]>(smem + 2 * kBK * (kTileM + kPad) + 2 * kBK * (kTileN + kPad));
  double* lv = smem + 2 * kBK * (kTileM + kPad) + 2 * kBK * (kTileN + kPad) + kTileM * (kTileN + 1);
  __shared__ int prow[kTileM];

  const KnnItem it = items[blockIdx.x];
  const int c = it.cls;
  const int p0 = ci.pair_offs[c] + it.tile * kTileM;
  const int np = min(kTileM, ci.pair_offs[c + 1] - p0);
  const int cr = ci.chunk_rows[c];
  const int r0 = ci.row_offs[c] + it.chunk * cr;
  const int r1 = min(ci.row_offs[c + 1], r0 + cr);
  const int tid = threadIdx.x;
  if (tid < kTileM) prow[tid] = (tid < np) ? (int)(pairs[p0 + tid] % ntest) : -1;
  for (int e = 0; e < use_k; ++e) lv[e * kTileThreads + tid] = -INFINITY;
  double tail = -INFINITY;

  const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  __syncthreads();

  for (int n0 = r0; n0 < r1; n0 += kTileN) {
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[8], rb[8];
    auto load = [&](int k0) {
      const int kk = tid & 15;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int mn = (tid >> 4) + 8 * i;
        const int gk = k0 + kk;
        const int tr = prow[mn];
        ra[i] = (tr >= 0 && gk < K) ? __ldg(Tq + (size_t)tr * K + gk) : 0.0;
        rb[i] = (n0 + mn < r1 && gk < K) ? __ldg(Ts + (size_t)(n0 + mn) * K + gk) : 0.0;
      }
    };
    auto store = [&](int b) {
      const int kk = tid & 15;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int mn = (tid >> 4) + 8 * i;
        As[b][kk][mn] = ra[i];
        Bs[b][kk][mn] = rb[i];
      }
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += kBK) {
      const bool has_next = k0 + kBK < K;
      if (has_next) load(k0 + kBK);
#pragma unroll
      for (int kk = 0; kk < kBK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[buf][kk + tig][wm + i * 8 + gid];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk + tig][wn + j * 8 + gid];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
      if (has_next) store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) sim[wm + i * 8 + gid][wn + j * 8 + tig * 2 + e] = acc[i][j][e];
    __syncthreads();
    {
      const int m = tid & (kTileM - 1), h = tid >> 6;
      const int ncol = min(32, r1 - n0 - h * 32);
      for (int cidx = 0; cidx < ncol; ++cidx) {
        const double v = sim[m][h * 32 + cidx];
        if (v > tail) {
          insert_desc<double, int>(lv + tid, nullptr, use_k, kTileThreads, v, 0);
          tail = lv[(use_k - 1) * kTileThreads + tid];
        }
      }
    }
    __syncthreads();
  }

  // Merge the two half-row lists of each test row; write the pair's list.
  if (tid < kTileM && tid < np) {
    const int q = p0 + tid - ci.pair_offs[c];
    double* out = part + ci.part_base[c] + ((long long)q * ci.nchunks[c] + it.chunk) * use_k;
    const double* la = lv + tid;
    const double* lb = lv + tid + kTileM;
    int ia = 0, ib = 0;
    for (int e = 0; e < use_k; ++e) {
      const double va = la[ia * kTileThreads], vb = lb[ib * kTileThreads];
      if (!(vb > va)) { out[e] = va; ++ia; } else { out[e] = vb; ++ib; }
    }
  }
}

// The same items with the whole contraction staged at once: the item's 64
// test rows are copied into shared memory once (cp.async, rows of K doubles
// at a stride S = K rounded up to 4 with S = 4 mod 16, so that the fragment
// loads of a warp hit distinct banks), the class's training rows stream
// through two 64-row buffers (the next tile's copy in flight while this one is
// multiplied), eight warps each take a 32 x 16 block of the 64 x 64 tile
// (FP64 m8n8k4), and the finished buffer holds the similarity tile for the
// top-k epilogue.  Up to K = 116.
constexpr int kV2Threads = 256;
constexpr int kV2MaxStride = 116;

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int NB>
__global__ void __launch_bounds__(kV2Threads, NB == 1 ? 2 : 1)
knn_tile_kernel_v2(const KnnItem* __restrict__ items, KnnClassInfo ci, const int* __restrict__ pairs,
                   int ntest, const double* __restrict__ Tq, const double* __restrict__ Ts, int K, int KP, int S,
                   int use_k, double* __restrict__ part) {
  extern __shared__ double smem[];
  // a training-row buffer also holds the 64 x 65 similarity tile
  const int BS = max(S, kTileN + 1);
  double* As = smem;                   // 64 x S (test rows)
  // NB = 2: two buffers, the next tile's copy in flight during this tile;
  // NB = 1: one buffer (half the shared memory: two CTAs per SM, one CTA's
  // epilogue overlapping the other's products)
  double* Bb[2] = {smem + kTileM * S, smem + kTileM * S + (NB - 1) * kTileN * BS};   // rows of stride S
  double* lv = smem + kTileM * S + NB * kTileN * BS;                                 // use_k x 128 lists
  __shared__ int prow[kTileM];

  const KnnItem it = items[blockIdx.x];
  const int c = it.cls;
  const int p0 = ci.pair_offs[c] + it.tile * kTileM;
  const int np = min(kTileM, ci.pair_offs[c + 1] - p0);
  const int cr = ci.chunk_rows[c];
  const int r0 = ci.row_offs[c] + it.chunk * cr;
  const int r1 = min(ci.row_offs[c + 1], r0 + cr);
  const int tid = threadIdx.x;
  if (tid < kTileM) prow[tid] = (tid < np) ? (int)(pairs[p0 + tid] % ntest) : -1;
  if (tid < 2 * kTileM)
    for (int e = 0; e < use_k; ++e) lv[e * (2 * kTileM) + tid] = -INFINITY;
  double tail = -INFINITY;
  __syncthreads();

  const uint32_t sA = static_cast<uint32_t>(__cvta_generic_to_shared(As));
  const uint32_t sB[2] = {static_cast<uint32_t>(__cvta_generic_to_shared(Bb[0])),
                          static_cast<uint32_t>(__cvta_generic_to_shared(Bb[1]))};
  for (int idx = tid; idx < kTileM * KP; idx += kV2Threads) {
    const int r = idx / KP, k = idx % KP;
    const int src = prow[r];
    const bool ok = src >= 0 && k < K;
    cp_async8(sA + 8u * (r * S + k), ok ? Tq + (size_t)src * K + k : Tq, ok);
  }
  auto copy_tile = [&](int n0, int b) {
    for (int idx = tid; idx < kTileN * KP; idx += kV2Threads) {
      const int r = idx / KP, k = idx % KP;
      const bool ok = n0 + r < r1 && k < K;
      cp_async8(sB[b] + 8u * (r * S + k), ok ? Ts + (size_t)(n0 + r) * K + k : Ts, ok);
    }
  };
  copy_tile(r0, 0);
  cp_async_commit();

  const int warp = tid >> 5, lane = tid & 31, gid = lane >> 2, tig = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  int j = 0;
  for (int n0 = r0; n0 < r1; n0 += kTileN, ++j) {
    const int b = NB == 2 ? (j & 1) : 0;
    const bool more = n0 + kTileN < r1;
    if (NB == 2 && more) {
      copy_tile(n0 + kTileN, b ^ 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* Bs = Bb[b];
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 2; ++q) acc[i][q][0] = acc[i][q][1] = 0.0;
    const double* ap = As + (wm + gid) * S + tig;
    const double* bp = Bs + (wn + gid) * S + tig;
#pragma unroll 5
    for (int kk = 0; kk < KP; kk += 4) {
      double a[4], bq[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = ap[i * 8 * S + kk];
#pragma unroll
      for (int q = 0; q < 2; ++q) bq[q] = bp[q * 8 * S + kk];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 2; ++q) dmma_8x8x4(acc[i][q][0], acc[i][q][1], a[i], bq[q]);
    }
    __syncthreads();   // every warp is done with this tile's training rows: the buffer holds the similarities
    double* sim = Bb[b];   // 64 x 65
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int e = 0; e < 2; ++e) sim[(wm + i * 8 + gid) * (kTileN + 1) + wn + q * 8 + tig * 2 + e] = acc[i][q][e];
    __syncthreads();
    if (tid < 2 * kTileM) {
      const int m = tid & (kTileM - 1), h = tid >> 6;
      const int ncol = min(32, r1 - n0 - h * 32);
      for (int cidx = 0; cidx < ncol; ++cidx) {
        const double v = sim[m * (kTileN + 1) + h * 32 + cidx];
        if (v > tail) {
          insert_desc<double, int>(lv + tid, nullptr, use_k, 2 * kTileM, v, 0);
          tail = lv[(use_k - 1) * (2 * kTileM) + tid];
        }
      }
    }
    __syncthreads();   // the buffer is refilled by the copy issued next
    if (NB == 1 && more) {
      copy_tile(n0 + kTileN, 0);
      cp_async_commit();
    }
  }

  // Merge the two half-row lists of each test row; write the pair's list.
  if (tid < kTileM && tid < np) {
    const int q = p0 + tid - ci.pair_offs[c];
    double* out = part + ci.part_base[c] + ((long long)q * ci.nchunks[c] + it.chunk) * use_k;
    const double* la = lv + tid;
    const double* lb = lv + tid + kTileM;
    int ia = 0, ib = 0;
    for (int e = 0; e < use_k; ++e) {
      const double va = la[ia * (2 * kTileM)], vb = lb[ib * (2 * kTileM)];
      if (!(vb > va)) { out[e] = va; ++ia; } else { out[e] = vb; ++ib; }
    }
  }
}

// ----------------------------------------------------- tensor-core filter
// The same (class, pair tile, training chunk) items on the BF16 tensor cores,
// with results equal to the FP64 tiles':
//   pass 1  128 pairs x 128 training rows of approximate similarities per
//           tile: both score rows split into BF16 planes hi = bf16(x),
//           lo = bf16(x - hi), three products hi.hi + hi.lo + lo.hi
//           (tcgen05.mma kind::f16, M128 N128 K16, FP32 accumulation in TMEM,
//           double-buffered so the epilogue overlaps the next tile); each pair
//           row keeps running maxima of 64 disjoint buckets of its values and
//           writes the k largest of them per chunk;
//   bar     per pair, theta = the k-th largest of those values over all its
//           chunks.  They are approximate values of distinct training rows, so
//           theta is at most the k-th largest approximate value of the class.
//           Every approximate value is within eps = 2^-14 |x| max|y| of the
//           exact dot: the split leaves x - hi - lo below 2^-18 |x| and drops
//           terms below 3 2^-18 |x||y| in all (1.2e-5 |x||y|); the BF16
//           products are exact in FP32 and the FP32 accumulation of the 3 x 128
//           products loses at most 384 2^-23 sum|x_k y_k| <= 4.6e-5 |x||y|
//           even with every addition truncated; 5.7e-5 < 2^-14.  So each row
//           of the pair's exact top k has an approximate value of at least
//           theta - 2 eps;
//   pass 2  the same products again; every training row whose approximate
//           value reaches that bar is scored exactly (FP64 dot of the two score
//           rows) and folded into the pair's top-k list, which is what the
//           FP64 tiles write and knn_merge_kernel reads.
// Score rows up to 128 wide, neighbour lists up to 16 long, up to 2^24
// training rows.  Warp 0 loads (TMA, SWIZZLE_128B boxes of 64 x 128 BF16: the
// A tile once, the B tiles through two stages), warp 1 issues the MMAs,
// warps 2..9 are the epilogue (two per TMEM lane quarter).  Every mbarrier
// wait is bounded; no cluster multicast.
constexpr int kFT = 128;                  // pairs per tile = training rows per tile
constexpr int kFK = 128;                  // contraction width (rows zero padded)
constexpr int kFBox = 64 * kFT * 2;       // one 64-wide box of 128 BF16 rows: 16 KB
constexpr int kFOperand = 4 * kFBox;      // two planes x two boxes: 64 KB
constexpr int kFEpiWarps = 8;             // two per TMEM lane quarter, half the columns each
constexpr int kFThreads = 64 + 32 * kFEpiWarps;
constexpr int kFBarOff = 3 * kFOperand;   // A, then two B stages
constexpr int kFList = 16;                // longest neighbour list of the filter
constexpr int kFBuckets = 32;             // pass 1: running maxima per thread
constexpr int kFCap = 128;                // pass 2: candidate rows kept per pair
constexpr int kFSmem = kFBarOff + 256 + 1024;
constexpr uint32_t kFIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(kFT >> 3) << 17) |
                             (uint32_t(kFT >> 4) << 24);
static_assert(kFSmem <= 227 * 1024, "filter tiles exceed shared memory");

__device__ __forceinline__ void umma_bf16_f32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kFIdesc), "r"(acc)
      : "memory");
}

template <int PASS>
__global__ void __launch_bounds__(kFThreads, 1)
knn_filter_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                  const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                  const KnnItem* __restrict__ items, KnnClassInfo ci, const int* __restrict__ pairs, int ntest,
                  const double* __restrict__ Tq, const double* __restrict__ Ts, int K, int use_k,
                  float* __restrict__ apart, const float* __restrict__ bar, int* __restrict__ ccount,
                  int* __restrict__ crow, int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~static_cast<uintptr_t>(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kFBarOff);
  uint64_t* fullA = bars;
  uint64_t* full = bars + 1;     // [2]
  uint64_t* empty = bars + 3;    // [2]
  uint64_t* tfull = bars + 5;    // [2]
  uint64_t* tempty = bars + 7;   // [2]
  uint64_t* done = bars + 9;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 10);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const KnnItem it = items[blockIdx.x];
  const int c = it.cls;
  const int p0 = ci.pair_offs[c] + it.tile * kFT;
  const int np = min(kFT, ci.pair_offs[c + 1] - p0);
  const int r0 = ci.row_offs[c] + it.chunk * ci.chunk_rows[c];
  const int r1 = min(ci.row_offs[c + 1], r0 + ci.chunk_rows[c]);
  const int ntiles = (r1 - r0 + kFT - 1) / kFT;

  if (threadIdx.x == 0) {
    tc::mbar_init(tc::smem_u32(fullA), 1);
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(tc::smem_u32(&full[b]), 1);
      tc::mbar_init(tc::smem_u32(&empty[b]), 1);
      tc::mbar_init(tc::smem_u32(&tfull[b]), 1);
      tc::mbar_init(tc::smem_u32(&tempty[b]), 32 * kFEpiWarps);
    }
    tc::mbar_init(tc::smem_u32(done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(2 * kFT)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    const uint32_t sa = tc::smem_u32(smem);
    tc::mbar_expect_tx(tc::smem_u32(fullA), kFOperand);
    tc::tma_load_2d(&mAh, sa, tc::smem_u32(fullA), 0, p0);
    tc::tma_load_2d(&mAh, sa + kFBox, tc::smem_u32(fullA), 64, p0);
    tc::tma_load_2d(&mAl, sa + 2 * kFBox, tc::smem_u32(fullA), 0, p0);
    tc::tma_load_2d(&mAl, sa + 3 * kFBox, tc::smem_u32(fullA), 64, p0);
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
      const int s = t & 1;
      if (!tc::mbar_wait(tc::smem_u32(&empty[s]), ((t >> 1) & 1) ^ 1, err)) break;
      const uint32_t fb = tc::smem_u32(&full[s]);
      const uint32_t sb = tc::smem_u32(smem + (1 + s) * kFOperand);
      const int row = r0 + t * kFT;
      tc::mbar_expect_tx(fb, kFOperand);
      tc::tma_load_2d(&mBh, sb, fb, 0, row);
      tc::tma_load_2d(&mBh, sb + kFBox, fb, 64, row);
      tc::tma_load_2d(&mBl, sb + 2 * kFBox, fb, 0, row);
      tc::tma_load_2d(&mBl, sb + 3 * kFBox, fb, 64, row);
      issued = t + 1;
    }
    // the copies in flight land before the CTA exits (bounded waits)
    tc::mbar_wait(tc::smem_u32(fullA), 0, err, false);
    for (int d = 1; d <= 2 && issued - d >= 0; ++d) {
      const int u = issued - d;
      tc::mbar_wait(tc::smem_u32(&full[u & 1]), (u >> 1) & 1, err, false);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------- MMA issuer
    bool ok = tc::mbar_wait(tc::smem_u32(fullA), 0, err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t sa = tc::smem_u32(smem);
    for (int t = 0; t < ntiles && ok; ++t) {
      const int b = t & 1;
      if (!tc::mbar_wait(tc::smem_u32(&tempty[b]), ((t >> 1) & 1) ^ 1, err)) { ok = false; break; }
      if (!tc::mbar_wait(tc::smem_u32(&full[b]), (t >> 1) & 1, err)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sb = tc::smem_u32(smem + (1 + b) * kFOperand);
      const uint32_t acc = tmem + static_cast<uint32_t>(b * kFT);
#pragma unroll
      for (int kk = 0; kk < kFK / 16; ++kk) {
        const uint32_t off = (kk >> 2) * kFBox + (kk & 3) * 32;   // box, then 32 bytes per K16 step
        const uint64_t ah = tc::sw128_desc(sa + off), al = tc::sw128_desc(sa + 2 * kFBox + off);
        const uint64_t bh = tc::sw128_desc(sb + off), bl = tc::sw128_desc(sb + 2 * kFBox + off);
        umma_bf16_f32(acc, ah, bh, kk > 0 ? 1u : 0u);
        umma_bf16_f32(acc, ah, bl, 1u);
        umma_bf16_f32(acc, al, bh, 1u);
      }
      tc::umma_commit(tc::smem_u32(&empty[b]));
      tc::umma_commit(tc::smem_u32(&tfull[b]));
    }
    // every MMA issued has completed before TMEM is released
    tc::umma_commit(tc::smem_u32(done));
    tc::mbar_wait(tc::smem_u32(done), 0, err, false);
  } else if (warp >= 2) {
    // ---------------------------------------------------------- epilogue
    // Two warps per TMEM lane quarter, each with half of the tile's columns:
    // thread (row r, half h) loads its 64 values in one round and releases
    // the accumulator before using them.
    //   pass 1: 32 running maxima of disjoint buckets of the half row's
    //           values (one max per value).  They are values of distinct
    //           training rows, so the k-th largest of them is at most the
    //           k-th largest approximate value, which is all the bar needs;
    //   pass 2: the rows whose value reaches the bar are noted in the pair's
    //           candidate slots (scored exactly by knn_exact_kernel, outside
    //           this pipeline).
    // The two halves of a pair row's bucket maxima are merged at the end.
    const int q = warp & 3;
    const int h = (warp - 2) / 4;
    const int r = q * 32 + lane;          // pair row of the tile (TMEM lane)
    const bool row_ok = r < np;
    const int tr = row_ok ? pairs[p0 + r] % ntest : 0;
    float M[kFBuckets];
#pragma unroll
    for (int e = 0; e < kFBuckets; ++e) M[e] = -INFINITY;
    const float thr = (PASS == 2 && row_ok) ? bar[p0 + r] : INFINITY;
    for (int t = 0; t < ntiles; ++t) {
      const int b = t & 1;
      const bool ok = tc::mbar_wait(tc::smem_u32(&tfull[b]), (t >> 1) & 1, err);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int n0 = r0 + t * kFT;
      const int ncol = min(kFT, r1 - n0);
      const uint32_t base = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(b * kFT + h * 64);
      uint32_t v[4][16];
      __syncwarp();
#pragma unroll
      for (int c = 0; c < 4; ++c) tc::tmem_ld16_raw(base + c * 16, v[c]);
      tc::tmem_wait_ld();
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      tc::mbar_arrive(tc::smem_u32(&tempty[b]));
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        // values past the class's last training row (or of an absent pair
        // row) are NaN: they fail every comparison, so they neither raise a
        // bucket maximum nor become candidates (not even for a bar of -inf)
        float f[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const bool in = ok && row_ok && h * 64 + g * 16 + i < ncol;
          f[i] = in ? __uint_as_float(v[g][i]) : __int_as_float(0x7fc00000);
        }
        if (PASS == 1) {
#pragma unroll
          for (int i = 0; i < 16; ++i) M[(g * 16 + i) % kFBuckets] = fmaxf(M[(g * 16 + i) % kFBuckets], f[i]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (f[i] >= thr) {
              const int slot = atomicAdd(ccount + p0 + r, 1);
              if (slot < kFCap) crow[(size_t)(p0 + r) * kFCap + slot] = n0 + h * 64 + g * 16 + i;
            }
        }
      }
      if (!ok) break;
    }
    // the two halves meet in the (now idle) A-tile buffer after the closing
    // barrier below
    if (PASS == 1) {
      float* ls = reinterpret_cast<float*>(smem);
#pragma unroll
      for (int e = 0; e < kFBuckets; ++e) ls[(h * kFBuckets + e) * kFT + r] = M[e];
    }
  }
  // every MMA has completed (the issuer waited for them) and every epilogue
  // thread has stored its values: one thread per pair row writes its list
  __syncthreads();
  if (PASS == 1 && warp >= 2 && warp < 6) {
    const int r = (warp & 3) * 32 + lane;
    if (r < np) {
      const int qi = p0 + r - ci.pair_offs[c];
      const long long o = ci.part_base[c] + ((long long)qi * ci.nchunks[c] + it.chunk) * use_k;
      // the use_k largest of the row's 64 bucket maxima, in descending order
      float* ls = reinterpret_cast<float*>(smem);
      for (int e = 0; e < use_k; ++e) {
        int best = 0;
        float bv = ls[r];
        for (int x = 1; x < 2 * kFBuckets; ++x) {
          const float vx = ls[x * kFT + r];
          if (vx > bv) { bv = vx; best = x; }
        }
        apart[o + e] = bv;
        ls[best * kFT + r] = -INFINITY;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kFT) : "memory");
  }
}

// Row i of the BF16 planes (rows_pad x kFK, zero padded) = the hi / lo split
// of row src(i) of S (row-major, K doubles per row): src(i) = pairs[i] % ntest
// when pairs is given (the test row of class-sorted pair i), else i.
__global__ void knn_split_rows_kernel(const double* __restrict__ S, int rows, int K, const int* __restrict__ pairs,
                                      int ntest, int rows_pad, __nv_bfloat16* __restrict__ hi,
                                      __nv_bfloat16* __restrict__ lo) {
  const size_t total = (size_t)rows_pad * kFK;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t / kFK), k = static_cast<int>(t % kFK);
    double x = 0.0;
    if (i < rows && k < K) {
      const int src = pairs ? pairs[i] % ntest : i;
      x = S[(size_t)src * K + k];
    }
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[t] = h;
    lo[t] = __double2bfloat16(x - static_cast<double>(__bfloat162float(h)));
  }
}

// Largest row norm of S (rows x K, row-major) as float bits (non-negative
// floats order as their bit patterns; a NaN norm wins and disables the filter).
__global__ void knn_row_norm_max_kernel(const double* __restrict__ S, int rows, int K, unsigned* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  double s = 0.0;
  for (int k = 0; k < K; ++k) s = fma(S[(size_t)i * K + k], S[(size_t)i * K + k], s);
  atomicMax(out, __float_as_uint(__double2float_ru(sqrt(s))));
}

// Per class-sorted pair: theta = the k-th largest approximate similarity over
// all its chunk lists, bar = theta - 2 eps (rounded down), -inf when the
// class has fewer than k rows.
__global__ void knn_filter_bar_kernel(const float* __restrict__ apart, KnnClassInfo ci, int C,
                                      const int* __restrict__ pairs, long long total_pairs, int ntest,
                                      const double* __restrict__ Tq, int K, int use_k,
                                      const unsigned* __restrict__ ymax_bits, float* __restrict__ bar) {
  const long long P = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (P >= total_pairs) return;
  int lo = 0, hi = C - 1;   // the last class whose pair offset is <= P
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ci.pair_offs[mid] <= P) lo = mid;
    else hi = mid - 1;
  }
  const int c = lo;
  const long long qi = P - ci.pair_offs[c];
  const int nch = ci.nchunks[c];
  float lst[kKnnMax];
  for (int e = 0; e < use_k; ++e) lst[e] = -INFINITY;
  for (int s = 0; s < nch; ++s) {
    const float* l = apart + ci.part_base[c] + (qi * nch + s) * use_k;
    for (int e = 0; e < use_k; ++e) {
      const float v = l[e];
      if (!(v > lst[use_k - 1])) break;   // chunk lists are sorted
      insert_desc<float, int>(lst, nullptr, use_k, 1, v, 0);
    }
  }
  const float theta = lst[use_k - 1];
  if (theta == -INFINITY) {
    bar[P] = -INFINITY;
    return;
  }
  const double* x = Tq + (size_t)(pairs[P] % ntest) * K;
  double s2 = 0.0;
  for (int k = 0; k < K; ++k) s2 = fma(x[k], x[k], s2);
  const double eps = ldexp(sqrt(s2) * static_cast<double>(__uint_as_float(*ymax_bits)), -14);
  bar[P] = __double2float_rd(static_cast<double>(theta) - 2.0 * eps);
}

// Exact scores of the candidates of every pair (one warp per class-sorted
// pair): up to 32 candidates, the lanes split each FP64 dot; more, each lane
// takes candidates lane, lane + 32, ... and forms their dots (k in order).  The
// use_k largest go to plist[P * use_k ..] in descending order (-inf when there
// are fewer).  A pair with more than kFCap
// candidates raises *overflow (its list would be incomplete).
__global__ void knn_exact_kernel(const int* __restrict__ ccount, const int* __restrict__ crow,
                                 const int* __restrict__ pairs, long long total_pairs, int ntest,
                                 const double* __restrict__ Tq, const double* __restrict__ Ts, int K, int use_k,
                                 double* __restrict__ plist, int* overflow) {
  const long long P = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (P >= total_pairs) return;   // whole warps
  int cnt = ccount[P];
  if (cnt > kFCap) {
    if (lane == 0) atomicExch(overflow, 1);
    cnt = kFCap;
  }
  const double* xr = Tq + (size_t)(pairs[P] % ntest) * K;
  if (cnt <= 32) {
    // The common case: the warp's lanes split every dot (four candidates at a
    // time, the test row loaded once), lane c keeps candidate c's value, and
    // each value goes to its rank in the descending list (ties by lane).
    double xv[kFK / 32];
#pragma unroll
    for (int m = 0; m < kFK / 32; ++m) xv[m] = (lane + 32 * m < K) ? xr[lane + 32 * m] : 0.0;
    double mine = -INFINITY;
    for (int c0 = 0; c0 < cnt; c0 += 4) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c0 + c < cnt) {
          const double* yr = Ts + (size_t)crow[(size_t)P * kFCap + c0 + c] * K;
#pragma unroll
          for (int m = 0; m < kFK / 32; ++m)
            if (lane + 32 * m < K) acc[c] = fma(xv[m], yr[lane + 32 * m], acc[c]);
        }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (lane == c0 + c && c0 + c < cnt) mine = acc[c];
    }
    if (!(mine == mine)) mine = -INFINITY;   // a NaN never enters a list
    int rank = 0;
    for (int j = 0; j < 32; ++j) {
      const double vj = __shfl_sync(0xffffffffu, mine, j);
      rank += (vj > mine || (vj == mine && j < lane)) ? 1 : 0;
    }
    if (rank < use_k) plist[P * use_k + rank] = mine;
    return;
  }
  double v[kFCap / 32];
#pragma unroll
  for (int u = 0; u < kFCap / 32; ++u) {
    v[u] = -INFINITY;
    const int idx = lane + 32 * u;
    if (idx < cnt) {
      const double* yr = Ts + (size_t)crow[(size_t)P * kFCap + idx] * K;
      double d = 0.0;
#pragma unroll 4
      for (int k = 0; k < K; ++k) d = fma(xr[k], yr[k], d);
      v[u] = d;
    }
  }
  for (int e = 0; e < use_k; ++e) {
    // the warp's largest remaining value; the lowest lane holding it gives it up
    double m = v[0];
#pragma unroll
    for (int u = 1; u < kFCap / 32; ++u) m = fmax(m, v[u]);
    double wm = m;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wm = fmax(wm, __shfl_xor_sync(0xffffffffu, wm, o));
    const unsigned holders = __ballot_sync(0xffffffffu, m == wm && wm > -INFINITY);
    if (holders && lane == __ffs(holders) - 1) {
      bool done = false;
#pragma unroll
      for (int u = 0; u < kFCap / 32; ++u)
        if (!done && v[u] == wm) {
          v[u] = -INFINITY;
          done = true;
        }
    }
    if (lane == 0) plist[P * use_k + e] = holders ? wm : -INFINITY;
  }
}

CUtensorMap make_bf16_rows_map(const __nv_bfloat16* p, int rows_pad) {
  CUtensorMap m;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(kFK), static_cast<cuuint64_t>(rows_pad)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(kFK) * 2};
  cuuint32_t box[2] = {64, static_cast<cuuint32_t>(kFT)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tc::encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(p), dims, strides,
                               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(kErrCuda, "cuTensorMapEncodeTiled failed (cKNN score planes)");
  return m;
}

// Per pair: merge its chunk lists, smoothed class score (src/fastPLS.cpp:1287-1320,
// src/lda_cuda_kernels.cu:225-242), add alpha * base + bias.
__global__ void knn_merge_kernel(const int* __restrict__ pairs, long long total_pairs,
                                 const int* __restrict__ cand, const double* __restrict__ cbase,
                                 KnnClassInfo ci, const double* __restrict__ part, int use_k,
                                 double tau, double alpha, const double* __restrict__ bias,
                                 double* __restrict__ cscore) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= total_pairs) return;
  const int flat = pairs[q];
  const int c = cand[flat] - 1;
  const int found = ci.row_offs[c + 1] - ci.row_offs[c];
  double top[kKnnMax];
  for (int e = 0; e < use_k; ++e) top[e] = -INFINITY;
  const int S = ci.nchunks[c];
  const double* src = part + ci.part_base[c] + (q - ci.pair_offs[c]) * (long long)S * use_k;
  for (int s = 0; s < S; ++s)
    for (int e = 0; e < use_k; ++e) {
      const double v = src[(size_t)s * use_k + e];
      if (!(v > top[use_k - 1])) break;  // lists are sorted: the rest is smaller
      insert_desc<double, int>(top, nullptr, use_k, 1, v, 0);
    }
  double local;
  if (found < 1 || !isfinite(top[0])) {
    local = -INFINITY;
  } else {
    const int denom = max(1, min(use_k, found));
    const double mx = top[0];
    double acc = 0.0;
    for (int j = 0; j < denom; ++j) acc += exp((top[j] - mx) / tau);
    local = mx + tau * log(acc / (double)denom);
  }
  cscore[flat] = __dadd_rn(__dadd_rn(local, __dmul_rn(alpha, cbase[flat])), bias[c]);
}

// Rerank the candidates of each row by score (src/fastPLS.cpp:1447-1466).
__global__ void knn_rerank_kernel(const int* __restrict__ cand, const double* __restrict__ cscore,
                                  int ntest, int C, int top_m, int top_k, int* __restrict__ top_index,
                                  double* __restrict__ top_score) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntest) return;
  for (int j = 0; j < top_k; ++j) {
    top_score[i + (size_t)j * ntest] = -INFINITY;
    top_index[i + (size_t)j * ntest] = -1;
  }
  for (int j = 0; j < top_m; ++j) {
    const int cls = cand[i + (size_t)j * ntest];
    if (cls < 1 || cls > C) continue;
    insert_desc(top_score + i, top_index + i, top_k, (size_t)ntest, cscore[i + (size_t)j * ntest], cls);
  }
}

__global__ void fill_int_kernel(int* x, size_t n, int v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = v;
}

// Class-contiguous, row-major copy of the rows of T (n x k, column-major) by
// class code; returns the C + 1 row offsets on the host and device.
struct ClassRows {
  double* Ts = nullptr;       // rows in class order, row-major (nvalid x k)
  int* d_offs = nullptr;      // C + 1
  std::vector<int> offs;      // C + 1 (host)
};

ClassRows group_rows_by_class(const double* dT, int n, int k, const int* dcodes, int C) {
  Context& ctx = Context::get();
  ClassRows cr;
  int* counts = ctx.arena.alloc_n<int>(C);
  int* cursor = ctx.arena.alloc_n<int>(C);
  int* dest = ctx.arena.alloc_n<int>(std::max(n, 1));
  fill_int_kernel<<<ceil_div(C, 256), 256, 0, ctx.stream>>>(counts, C, 0); ::fpls::note_launch();
  fill_int_kernel<<<ceil_div(C, 256), 256, 0, ctx.stream>>>(cursor, C, 0); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  const int g = std::max(1, std::min(ceil_div(n, 256), 8 * ctx.sm_count));
  class_hist_kernel<<<g, 256, 0, ctx.stream>>>(dcodes, n, C, counts); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  std::vector<int> h(C);
  d2h(h.data(), counts, C * sizeof(int));
  ctx.sync();
  cr.offs.assign(C + 1, 0);
  for (int c = 0; c < C; ++c) cr.offs[c + 1] = cr.offs[c] + h[c];
  cr.d_offs = ctx.arena.alloc_n<int>(C + 1);
  h2d(cr.d_offs, cr.offs.data(), (C + 1) * sizeof(int));
  class_slot_kernel<<<g, 256, 0, ctx.stream>>>(dcodes, n, C, cr.d_offs, cursor, dest); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  const int nvalid = cr.offs[C];
  cr.Ts = ctx.arena.alloc_n<double>((size_t)std::max(nvalid, 1) * k);
  dim3 grid(ceil_div(n, 32), ceil_div(k, 32));
  transpose_scatter_kernel<<<grid, dim3(32, 8), 0, ctx.stream>>>(dT, n, k, dest, cr.Ts); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  return cr;
}

}  // namespace

using capi::upload;

void candidate_scores_device(const double* dT, int n, int k, const double* dCk, double* dTn) {
  Context& ctx = Context::get();
  const double* src = dT;
  if (dCk) {
    double* prod = ctx.arena.alloc_n<double>((size_t)n * k);
    gemm(false, false, n, k, k, 1.0, dT, n, dCk, k, 0.0, prod, n);
    src = prod;
  }
  row_l2_kernel<<<ceil_div(n, 128), 128, 0, ctx.stream>>>(src, n, k, dTn); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void candidate_centroids_device(const double* dTn, int n, int k, const int* dy, int C, double* dCent) {
  Context& ctx = Context::get();
  ClassRows cr = group_rows_by_class(dTn, n, k, dy, C);
  const int nvalid = cr.offs[C];
  double* sums = ctx.arena.alloc_n<double>((size_t)C * k);
  fill(sums, (size_t)C * k, 0.0);
  if (nvalid > 0) {
    const int rows = std::min(2048, std::max(64, ceil_div(nvalid, 4 * ctx.sm_count)));
    for (int col0 = 0; col0 < k; col0 += 128 * kCentCols) {
      class_rowsum_kernel<<<ceil_div(nvalid, rows), 128, 0, ctx.stream>>>(cr.Ts, k, nvalid, cr.d_offs, C, rows,
                                                                         col0, sums); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
  }
  centroid_finish_kernel<<<ceil_div(C, 128), 128, 0, ctx.stream>>>(sums, k, cr.d_offs, C, dCent); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void candidate_knn_predict_device(const double* dTt, int ntest, const double* dTr, int ntrain, int kdim,
                                  const int* dy, const double* dC, int C, const double* dbias, int top_k,
                                  int top_m, int knn_k, double tau, double alpha, int* d_ti, double* d_ts,
                                  bool allow_filter) {
  Context& ctx = Context::get();
  const int tk = std::max(1, std::min(top_k, C));
  const int tm = std::max(tk, std::min(std::max(1, top_m), C));
  const int use_k = std::max(1, std::min(std::max(1, knn_k), kKnnMax));
  const double tau_e = (std::isfinite(tau) && tau > 0.0) ? tau : 0.2;
  const double alpha_e = std::isfinite(alpha) ? alpha : 0.5;
  const long long npairs = (long long)ntest * tm;
  FPLS_REQUIRE(npairs < (1ll << 31), "candidate-kNN: ntest * top_m must stay below 2^31");
  double* bias0 = nullptr;
  if (!dbias) {
    bias0 = ctx.arena.alloc_n<double>(C);
    fill(bias0, C, 0.0);
    dbias = bias0;
  }
  PhaseTimer pt("candidate-kNN predict");
  // base scores and candidate classes
  double* base = ctx.arena.alloc_n<double>((size_t)ntest * C);
  gemm(false, true, ntest, C, kdim, 1.0, dTt, ntest, dC, C, 0.0, base, ntest);
  int* cand = ctx.arena.alloc_n<int>((size_t)npairs);
  double* cbase = ctx.arena.alloc_n<double>((size_t)npairs);
  select_candidates_kernel<<<ceil_div(ntest, 128), 128, 0, ctx.stream>>>(base, ntest, C, tm, cand, cbase); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();

  // training rows grouped by class (row-major), test rows row-major
  pt.mark("base scores + candidates");
  ClassRows cr = group_rows_by_class(dTr, ntrain, kdim, dy, C);
  double* Tq = ctx.arena.alloc_n<double>((size_t)ntest * kdim);
  {
    dim3 grid(ceil_div(ntest, 32), ceil_div(kdim, 32));
    transpose_scatter_kernel<<<grid, dim3(32, 8), 0, ctx.stream>>>(dTt, ntest, kdim, nullptr, Tq); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }

  // (row, candidate) pairs grouped by class
  int* pcount = ctx.arena.alloc_n<int>(C);
  int* pcursor = ctx.arena.alloc_n<int>(C);
  fill_int_kernel<<<ceil_div(C, 256), 256, 0, ctx.stream>>>(pcount, C, 0); ::fpls::note_launch();
  fill_int_kernel<<<ceil_div(C, 256), 256, 0, ctx.stream>>>(pcursor, C, 0); ::fpls::note_launch();
  const int g = std::max(1, std::min(ceil_div(npairs, 256), 8 * ctx.sm_count));
  pair_hist_kernel<<<g, 256, 0, ctx.stream>>>(cand, npairs, C, pcount); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  std::vector<int> hp(C);
  d2h(hp.data(), pcount, C * sizeof(int));
  ctx.sync();
  // Tile kernel (FASTPLS_CKNN_TILES): 4 or unset the BF16 tensor-core filter
  // with exact FP64 rescoring (score rows up to 128 wide), 1 the 16-wide
  // k-step FP64 kernel, 2 / 3 the staged FP64 kernels with two / one
  // training-row buffers.
  const char* tv = std::getenv("FASTPLS_CKNN_TILES");
  const char sel = (tv && tv[0]) ? tv[0] : '4';
  const bool use_filter = allow_filter && sel == '4' && kdim <= kFK && use_k <= kFList;
  const int tile_m = use_filter ? kFT : kTileM;   // pairs per item
  const int gran = use_filter ? kFT : kTileN;     // chunk rows are a multiple of this
  std::vector<int> poffs(C + 1, 0), chunk_rows(C, 0), nchunks(C, 0);
  std::vector<long long> part_base(C, 0);
  std::vector<KnnItem> items;
  long long part_total = 0;
  for (int c = 0; c < C; ++c) {
    poffs[c + 1] = poffs[c] + hp[c];
    const int rows = cr.offs[c + 1] - cr.offs[c];
    int S = 0, cr_rows = 0;
    if (rows > 0) {
      S = std::min(kMaxChunks, std::max(1, ceil_div(rows, kMinChunkRows)));
      cr_rows = ceil_div(ceil_div(rows, S), gran) * gran;
      S = ceil_div(rows, cr_rows);
    }
    chunk_rows[c] = cr_rows;
    nchunks[c] = S;
    part_base[c] = part_total;
    part_total += (long long)hp[c] * S * use_k;
    if (rows > 0 && hp[c] > 0) {
      const int tiles = ceil_div(hp[c], tile_m);
      for (int t = 0; t < tiles; ++t)
        for (int s = 0; s < S; ++s) items.push_back(KnnItem{c, t, s, 0});
    }
  }
  const long long total_pairs = poffs[C];
  if (pt.enabled()) {
    double work = 0.0;
    for (int c = 0; c < C; ++c) work += (double)hp[c] * (cr.offs[c + 1] - cr.offs[c]);
    std::fprintf(stderr, "[fastpls trace] candidate-kNN: %lld pairs, %.3e pair-rows (%.3e flop), %zu items\n",
                 total_pairs, work, 2.0 * work * kdim, items.size());
  }
  int* pairs = ctx.arena.alloc_n<int>((size_t)std::max<long long>(total_pairs, 1));
  int* d_poffs = ctx.arena.alloc_n<int>(C + 1);
  h2d(d_poffs, poffs.data(), (C + 1) * sizeof(int));
  pair_scatter_kernel<<<g, 256, 0, ctx.stream>>>(cand, npairs, C, d_poffs, pcursor, pairs); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();

  KnnClassInfo ci;
  ci.row_offs = cr.d_offs;
  ci.pair_offs = d_poffs;
  ci.chunk_rows = upload(chunk_rows.data(), C);
  ci.nchunks = upload(nchunks.data(), C);
  ci.part_base = upload(part_base.data(), C);
  double* part = ctx.arena.alloc_n<double>((size_t)std::max<long long>(part_total, 1));
  double* cscore = ctx.arena.alloc_n<double>((size_t)npairs);
  pt.mark("class rows + pair lists");
  // the lists the merge reads: (pair, chunk) lists of the FP64 tiles, or one
  // exact list per pair from the filter
  KnnClassInfo ci_merge = ci;
  const double* merge_part = part;
  if (!items.empty() && use_filter) {
    const KnnItem* ditems = upload(items.data(), items.size());
    FPLS_REQUIRE(items.size() < (1u << 31), "candidate-kNN: too many work items");
    const int slot = ctx.prof_begin("cknn_filter", ctx.stream);
    const int nvalid = cr.offs[C];
    const long long a_rows = (total_pairs + kFT - 1) / kFT * kFT + kFT;
    const long long b_rows = ((long long)nvalid + kFT - 1) / kFT * kFT + kFT;
    FPLS_REQUIRE(a_rows < (1ll << 31) && b_rows < (1ll << 31), "candidate-kNN: too many rows for the filter");
    __nv_bfloat16* ah = ctx.arena.alloc_n<__nv_bfloat16>((size_t)a_rows * kFK);
    __nv_bfloat16* al = ctx.arena.alloc_n<__nv_bfloat16>((size_t)a_rows * kFK);
    __nv_bfloat16* bh = ctx.arena.alloc_n<__nv_bfloat16>((size_t)b_rows * kFK);
    __nv_bfloat16* bl = ctx.arena.alloc_n<__nv_bfloat16>((size_t)b_rows * kFK);
    const int gs = 8 * ctx.sm_count;
    knn_split_rows_kernel<<<gs, 256, 0, ctx.stream>>>(Tq, (int)total_pairs, kdim, pairs, ntest, (int)a_rows, ah, al);
    ::fpls::note_launch();
    knn_split_rows_kernel<<<gs, 256, 0, ctx.stream>>>(cr.Ts, nvalid, kdim, nullptr, 1, (int)b_rows, bh, bl);
    ::fpls::note_launch();
    unsigned* ymax = ctx.arena.alloc_n<unsigned>(1);
    dzero(ymax, sizeof(unsigned));
    if (nvalid > 0) {
      knn_row_norm_max_kernel<<<ceil_div(nvalid, 256), 256, 0, ctx.stream>>>(cr.Ts, nvalid, kdim, ymax);
      ::fpls::note_launch();
    }
    FPLS_CHECK_LAUNCH();
    pt.mark("filter planes");
    const CUtensorMap mAh = make_bf16_rows_map(ah, (int)a_rows), mAl = make_bf16_rows_map(al, (int)a_rows);
    const CUtensorMap mBh = make_bf16_rows_map(bh, (int)b_rows), mBl = make_bf16_rows_map(bl, (int)b_rows);
    float* apart = ctx.arena.alloc_n<float>((size_t)std::max<long long>(part_total, 1));
    float* barv = ctx.arena.alloc_n<float>((size_t)std::max<long long>(total_pairs, 1));
    int* ferr = ctx.d_status + 24;
    dzero(ferr, sizeof(int));
    int* ccount = ctx.arena.alloc_n<int>((size_t)std::max<long long>(total_pairs, 1));
    int* crow = ctx.arena.alloc_n<int>((size_t)std::max<long long>(total_pairs, 1) * kFCap);
    dzero(ccount, (size_t)std::max<long long>(total_pairs, 1) * sizeof(int));
    static bool fattr = false;
    if (!fattr) {
      FPLS_CUDA(cudaFuncSetAttribute(knn_filter_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
      FPLS_CUDA(cudaFuncSetAttribute(knn_filter_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
      fattr = true;
    }
    const unsigned ng = (unsigned)items.size();
    knn_filter_kernel<1><<<ng, kFThreads, kFSmem, ctx.stream>>>(mAh, mAl, mBh, mBl, ditems, ci, pairs, ntest, Tq,
                                                               cr.Ts, kdim, use_k, apart, nullptr, nullptr, nullptr,
                                                               ferr);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    pt.mark("filter pass 1");
    knn_filter_bar_kernel<<<(unsigned)ceil_div(total_pairs, 256), 256, 0, ctx.stream>>>(
        apart, ci, C, pairs, total_pairs, ntest, Tq, kdim, use_k, ymax, barv);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    pt.mark("filter bar");
    knn_filter_kernel<2><<<ng, kFThreads, kFSmem, ctx.stream>>>(mAh, mAl, mBh, mBl, ditems, ci, pairs, ntest, Tq,
                                                               cr.Ts, kdim, use_k, nullptr, barv, ccount, crow,
                                                               ferr);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    pt.mark("filter pass 2");
    // exact scores of the candidates, one list per pair
    double* plist = ctx.arena.alloc_n<double>((size_t)std::max<long long>(total_pairs, 1) * use_k);
    int* fover = ctx.d_status + 25;
    dzero(fover, sizeof(int));
    knn_exact_kernel<<<(unsigned)ceil_div(total_pairs * 32, 256), 256, 0, ctx.stream>>>(
        ccount, crow, pairs, total_pairs, ntest, Tq, cr.Ts, kdim, use_k, plist, fover);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    pt.mark("filter exact scores");
    std::vector<int> ones(C, 1);
    std::vector<long long> pbase(C);
    for (int c = 0; c < C; ++c) pbase[c] = (long long)poffs[c] * use_k;
    ci_merge.nchunks = upload(ones.data(), C);
    ci_merge.part_base = upload(pbase.data(), C);
    merge_part = plist;
    if (slot >= 0) {
      // algorithmic work: the three BF16 products of both passes over every
      // (candidate pair, class row); bytes: the score planes of every class's
      // training rows once per 128-pair tile and pass, the pair planes once
      // (the class's time includes the planes, the bar and the exact scores)
      double work = 0.0, bytes = 2.0 * 4.0 * kFK * (double)total_pairs;
      for (int c = 0; c < C; ++c) {
        const double rows = cr.offs[c + 1] - cr.offs[c];
        work += (double)hp[c] * rows;
        bytes += 2.0 * 4.0 * kFK * rows * (double)ceil_div(hp[c], kFT);
      }
      ctx.prof_end(slot, ctx.stream, bytes, 2.0 * 3.0 * 2.0 * work * kdim);
    }
    int flags[2] = {0, 0};
    d2h(flags, ferr, 2 * sizeof(int));
    ctx.sync();
    if (flags[0]) throw Error(kErrCuda, "candidate-kNN: a filter tile's pipeline wait timed out");
    if (flags[1]) {
      // a pair had more rows within the error bar than its candidate slots
      // hold: the call runs again on the FP64 tiles
      candidate_knn_predict_device(dTt, ntest, dTr, ntrain, kdim, dy, dC, C, dbias, top_k, top_m, knn_k, tau,
                                   alpha, d_ti, d_ts, false);
      return;
    }
  } else if (!items.empty()) {
    const KnnItem* ditems = upload(items.data(), items.size());
    FPLS_REQUIRE(items.size() < (1u << 31), "candidate-kNN: too many work items");
    const int slot = ctx.prof_begin("cknn_tiles", ctx.stream);
    // stride of the staged rows: K rounded up to 4, then to 4 mod 16
    const int KP = (kdim + 3) / 4 * 4;
    const int S = KP + (4 - KP % 16 + 16) % 16;
    // FP64 tile kernels: on the large-class workload (K = 100) the
    // similarity tiles took 123.4 ms (k-step), 162.6 ms (two buffers: one
    // 8-warp CTA per SM, the tensor pipe idles while the top-k epilogue runs)
    // and 107.2 ms (one buffer: two CTAs per SM, one CTA's epilogue overlapping
    // the other's products).  The filter takes score rows up to 128 wide and
    // lists up to 16 long; past that the staged kernel runs, and rows wider
    // than 116 doubles take the k-step kernel.
    if (S <= kV2MaxStride && sel != '1') {
      const int nb = sel == '2' ? 2 : 1;
      const size_t smem = sizeof(double) * ((size_t)kTileM * S + nb * (size_t)kTileN * std::max(S, kTileN + 1) +
                                            (size_t)use_k * 2 * kTileM);
      const int smem_max = (int)(sizeof(double) * ((size_t)(kTileM + nb * kTileN) * kV2MaxStride +
                                                   (size_t)kKnnMax * 2 * kTileM));
      static bool attr2[2] = {false, false};
      if (!attr2[nb - 1]) {
        if (nb == 2)
          FPLS_CUDA(cudaFuncSetAttribute(knn_tile_kernel_v2<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
        else {
          FPLS_CUDA(cudaFuncSetAttribute(knn_tile_kernel_v2<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
          // all of the SM's unified memory as shared memory: two 113 KB CTAs at K = 100
          FPLS_CUDA(cudaFuncSetAttribute(knn_tile_kernel_v2<1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared));
        }
        attr2[nb - 1] = true;
      }
      if (nb == 2)
        knn_tile_kernel_v2<2><<<(unsigned)items.size(), kV2Threads, smem, ctx.stream>>>(
            ditems, ci, pairs, ntest, Tq, cr.Ts, kdim, KP, S, use_k, part);
      else
        knn_tile_kernel_v2<1><<<(unsigned)items.size(), kV2Threads, smem, ctx.stream>>>(
            ditems, ci, pairs, ntest, Tq, cr.Ts, kdim, KP, S, use_k, part);
    } else {
      const size_t smem = sizeof(double) * (2 * kBK * (kTileM + kPad) + 2 * kBK * (kTileN + kPad) +
                                            kTileM * (kTileN + 1) + (size_t)kKnnMax * kTileThreads);
      static bool attr_set = false;
      if (!attr_set) {
        FPLS_CUDA(cudaFuncSetAttribute(knn_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set = true;
      }
      knn_tile_kernel<<<(unsigned)items.size(), kTileThreads, smem, ctx.stream>>>(
          ditems, ci, pairs, ntest, Tq, cr.Ts, kdim, use_k, part);
    }
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    if (slot >= 0) {
      // algorithmic work: one kdim-long FP64 dot per (candidate pair, class row);
      // bytes: every class's training rows once per 64-row tile of its pairs,
      // the test rows once
      double work = 0.0, bytes = 8.0 * (double)ntest * kdim;
      for (int c = 0; c < C; ++c) {
        const double rows = cr.offs[c + 1] - cr.offs[c];
        work += (double)hp[c] * rows;
        bytes += 8.0 * kdim * rows * (double)ceil_div(hp[c], kTileM);
      }
      ctx.prof_end(slot, ctx.stream, bytes, 2.0 * work * kdim);
    }
  }
  pt.mark("similarity tiles");
  fill(cscore, (size_t)npairs, -INFINITY);
  if (total_pairs > 0) {
    knn_merge_kernel<<<ceil_div(total_pairs, 128), 128, 0, ctx.stream>>>(
        pairs, total_pairs, cand, cbase, ci_merge, merge_part, use_k, tau_e, alpha_e, dbias, cscore);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  knn_rerank_kernel<<<ceil_div(ntest, 128), 128, 0, ctx.stream>>>(cand, cscore, ntest, C, tm, tk, d_ti, d_ts); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  pt.mark("merge + rerank");
  pt.report();
}

}  // namespace fpls

using namespace fpls;

extern "C" {

int fpls_candidate_scores(const double* T, int n, int k, const double* Ck, double* Tn, char* err,
                          size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && k > 0, "candidate-kNN requires at least one latent component");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dT = upload(T, (size_t)n * k);
    const double* dC = Ck ? upload(Ck, (size_t)k * k) : nullptr;
    double* out = ctx.arena.alloc_n<double>((size_t)n * k);
    candidate_scores_device(dT, n, k, dC, out);
    d2h(Tn, out, (size_t)n * k * sizeof(double));
    ctx.sync();
  });
}

int fpls_candidate_centroids(const double* Tn, int n, int k, const int* y_codes, int n_classes,
                             double* centroids, char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && k > 0, "candidate centroids: empty score matrix");
    FPLS_REQUIRE(n_classes >= 1, "candidate-kNN requires at least one class");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dT = upload(Tn, (size_t)n * k);
    const int* dy = upload(y_codes, n);
    double* dC = ctx.arena.alloc_n<double>((size_t)n_classes * k);
    candidate_centroids_device(dT, n, k, dy, n_classes, dC);
    d2h(centroids, dC, (size_t)n_classes * k * sizeof(double));
    ctx.sync();
  });
}

int fpls_candidate_knn_predict(const double* Ttest_norm, int ntest, const double* Ttrain_norm,
                               int ntrain, int kdim, const int* y_codes, const double* centroids,
                               int n_classes, const double* candidate_bias, int top_k, int top_m,
                               int knn_k, double tau, double alpha, int* top_index,
                               double* top_score, char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(n_classes >= 1, "candidate-kNN requires at least one class");
    FPLS_REQUIRE(ntest > 0 && ntrain > 0 && kdim > 0, "candidate-kNN: empty score matrices");
    Context& ctx = Context::get();
    ctx.begin_call();
    const int C = n_classes;
    const int tk = std::max(1, std::min(top_k, C));
    const double* dTt = upload(Ttest_norm, (size_t)ntest * kdim);
    const double* dTr = upload(Ttrain_norm, (size_t)ntrain * kdim);
    const int* dy = upload(y_codes, ntrain);
    const double* dC = upload(centroids, (size_t)C * kdim);
    const double* dbias = candidate_bias ? upload(candidate_bias, C) : nullptr;
    int* d_ti = ctx.arena.alloc_n<int>((size_t)ntest * tk);
    double* d_ts = ctx.arena.alloc_n<double>((size_t)ntest * tk);
    candidate_knn_predict_device(dTt, ntest, dTr, ntrain, kdim, dy, dC, C, dbias, top_k, top_m, knn_k,
                                 tau, alpha, d_ti, d_ts);
    d2h(top_index, d_ti, (size_t)ntest * tk * sizeof(int));
    d2h(top_score, d_ts, (size_t)ntest * tk * sizeof(double));
    ctx.sync();
  });
}

}  // extern "C"
