#include "dual_engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>

#include "autotune.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "ozaki_gemm.cuh"
#include "tc_util.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace fpls {
namespace {

constexpr int kMaxN = 8192;     // n-vectors staged in shared memory
constexpr int kMaxM = 128;
constexpr int kMaxK = 256;

struct DualEng {
  int n, m, F, K, iters, m1, center;
  int merge;     // refresh merged into the previous component's reduction (m <= kFuseM)
  const double* x0;
  const double* XOmega;
  const uint8_t* mask;
  const int* labels;
  const double* mY_all;
  const double* dY;
  const int* ntrain;
  const double* class_cnt;   // F x m train rows per class
  double* CS;    // F x n x m
  double* KCS;   // F x n x m
  double* CV;    // F x n x K
  double* KCV;   // F x n x K
  double* Kcy;   // F x n   K image of the warm start r / ||t|| of the last component
  double* cp;    // n x F   loading coefficients (input of the K product)
  double* Gp;    // n x F   K cp
  // K cp as INT8-product partials (when kpart is set): entry (i, f) is the sum
  // over segments s of tile (i / 128) * kntn + f / 64 of
  // kpart[(s * 64 + f % 64) * 128 + i % 128], in segment order.
  const double* kpart;
  const int* kseg;
  int kntn;
  // Digit planes of cp written by the step (when cpd is set): plane sl, row f
  // at cpd + sl * cpstride + f * cpldk, scale 2^e in cps[f].
  int8_t* cpd;
  double* cps;
  int cpldk, cpS;
  size_t cpstride;
  double* scal;  // F x 2   ||t||, sum(t)
  double* qs;    // F x m   Y^T t
  double* Q;
  double* tnorm;
  double* Tkeep;
  int* ncomp_done;
  int* status;
};

constexpr int kRedMax = kMaxK > kMaxM + 3 ? kMaxK : kMaxM + 3;
// Class counts up to which a step launch merges the refresh of component a
// into the Gram-Schmidt of component a - 1 (the merged reduction's columns,
// m + 1 and m + 2 of them, fit one 8 x 8 FP64 MMA tile).
constexpr int kFuseM = 6;

// C_S of every fit: mask_f * (onehot(label) - (mY_all + dY_f)).
__global__ void k_dual_cs0(DualEng e) {
  const size_t total = (size_t)e.F * e.n * e.m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % e.n);
    const size_t col = t / e.n;
    const int f = static_cast<int>(col / e.m), j = static_cast<int>(col % e.m);
    double v = 0.0;
    if (e.mask[(size_t)f * e.n + i]) {
      const double off = e.mY_all[j] + (e.dY ? e.dY[(size_t)f * e.m + j] : 0.0);
      v = (e.labels[i] == j ? 1.0 : 0.0) - off;
    }
    e.CS[t] = v;
  }
}

// Each fit is handled by CL CTAs of T threads (a thread-block cluster when
// CL > 1); CTA r owns rows [r * rows_per, (r + 1) * rows_per) of every
// n-vector of the fit and keeps them in registers (LR rows per thread, so
// n <= CL * T * LR).  Reductions over the n rows are per-CTA (warp shuffles,
// shared memory) and then across the cluster through distributed shared
// memory, summed in rank order so every CTA of the cluster sees bit-identical
// results and takes the same branches.  With CL = 1 a fit lives in one CTA and
// every reduction ends at a block barrier.
template <int CL, int T, int LR, bool MG>
struct Step {
static constexpr int kCl = CL;
static constexpr int kT = T;
static constexpr int kW = T / 32;
static constexpr int kLR = LR;


static constexpr int kDotChunk = 64;   // columns of one pass of per-warp dot partials
static constexpr int kDotCols = LR <= 4 ? 8 : 4;   // columns whose loads are in flight together
static constexpr int kColUnroll = LR <= 4 ? 8 : 4;
struct ClusterRed {
  double warp[kW][kDotChunk];
  double xw[kW];                     // per-warp sums of an extra scalar reduced with the dots
  double part[2][kRedMax];           // this CTA's partials (alternating between exchanges)
  double res[kRedMax];
  double fv[kFuseM];                 // merged launch: S'^T v / |v| and the refresh start z
  double fz[2][kFuseM];
  int buf;
};

// Per-fit data that no launch changes, staged in shared memory before the
// dependency wait: x0 and the label of every owned row (-1 outside the fit's
// training rows) at slot k * T + thread, the class counts and the training
// row count.
struct Fixed {
  double x0[kT * kLR];
  signed char lab[kT * kLR];
  double cnt[kMaxM];
  double nf;
};

struct Rows {
  int r0, nl;  // first owned row, owned row count
  __device__ __forceinline__ bool ok(int k) const { return (int)threadIdx.x + k * kT < nl; }
  __device__ __forceinline__ int row(int k) const { return r0 + (int)threadIdx.x + k * kT; }
};

// part[buf][0..count) holds this CTA's partials (after a barrier): combine
// them over the cluster into res[0..count) (sums, or maxima for k >=
// max_from), in rank order; ends with res visible to the CTA.  A peer reads
// part[buf] after the cluster barrier, so the next exchange writes the other
// buffer.
static __device__ void cluster_exchange(ClusterRed& R, int count, int max_from = kRedMax) {
  const int b = R.buf;
  if constexpr (CL == 1) {
    __syncthreads();
    for (int k = threadIdx.x; k < count; k += kT) R.res[k] = R.part[b][k];
    __syncthreads();
    if (threadIdx.x == 0) R.buf = b ^ 1;
    __syncthreads();
  } else {
    // The cluster barrier also orders this CTA's own partial writes (every
    // thread of every CTA arrives with release semantics), and every thread
    // has read buf before it, so the flip can follow at once; the closing
    // block barrier publishes res and the new buf.
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    if (threadIdx.x == 0) R.buf = b ^ 1;
    for (int k = threadIdx.x; k < count; k += kT) {
      double v = cl.map_shared_rank(&R.part[b][0], 0)[k];
      if (k >= max_from) {
        for (int r = 1; r < kCl; ++r) v = fmax(v, cl.map_shared_rank(&R.part[b][0], r)[k]);
      } else {
        for (int r = 1; r < kCl; ++r) v += cl.map_shared_rank(&R.part[b][0], r)[k];
      }
      R.res[k] = v;
    }
    __syncthreads();
  }
}

// res[0..count) = cluster sums of the per-thread values v[0..count) (count <= 4).
static __device__ void cluster_sum(ClusterRed& R, double (&v)[4], int count) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = 0; k < count; ++k) {
    const double w = warp_sum(v[k]);
    if (lane == 0) R.warp[warp][k] = w;
  }
  __syncthreads();
  if (threadIdx.x < count) {
    double s = 0.0;
    for (int w = 0; w < kW; ++w) s += R.warp[w][threadIdx.x];
    R.part[R.buf][threadIdx.x] = s;
  }
  cluster_exchange(R, count);
}

// res[j] = sum over the fit's rows of M[i + j*n] * x_i for j < ncols, with x
// given by the owned rows in registers.
// With has_extra, res[ncols] is also the cluster sum of the per-thread value extra.
// With CG the columns are read through L2 only (ld.global.cg): for data of an
// earlier grid read before this grid's dependency wait.
template <bool CG = false>
static __device__ void cluster_dots(ClusterRed& R, const double* __restrict__ M, int n, int ncols, const Rows& rw,
                                    const double (&x)[kLR], bool has_extra = false, double extra = 0.0) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (has_extra) {
    const double w = warp_sum(extra);
    if (lane == 0) R.xw[warp] = w;
  }
  for (int c0 = 0; c0 < ncols; c0 += kDotChunk) {
    const int cn = min(kDotChunk, ncols - c0);
    // kDotCols columns per pass, loads issued together (no data-dependent
    // exit: a column past the end re-reads the last one and is discarded)
    for (int j0 = 0; j0 < cn; j0 += kDotCols) {
      double acc[kDotCols];
#pragma unroll
      for (int jj = 0; jj < kDotCols; ++jj) acc[jj] = 0.0;
#pragma unroll
      for (int jj = 0; jj < kDotCols; ++jj) {
        const int jc = min(j0 + jj, cn - 1);
        const double* col = M + (size_t)(c0 + jc) * n;
#pragma unroll
        for (int k = 0; k < kLR; ++k)
          if (rw.ok(k)) acc[jj] += (CG ? __ldcg(col + rw.row(k)) : col[rw.row(k)]) * x[k];
      }
#pragma unroll
      for (int jj = 0; jj < kDotCols; ++jj) {
        const double w = warp_sum(acc[jj]);
        if (lane == 0 && j0 + jj < cn) R.warp[warp][j0 + jj] = w;
      }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cn; j += kT) {
      double s = 0.0;
      for (int w = 0; w < kW; ++w) s += R.warp[w][j];
      R.part[R.buf][c0 + j] = s;
    }
    if (has_extra && c0 == 0 && threadIdx.x == kT - 1) {
      double v = 0.0;
      for (int w = 0; w < kW; ++w) v += R.xw[w];
      R.part[R.buf][ncols] = v;
    }
    if (c0 + kDotChunk < ncols) __syncthreads();   // before the next chunk reuses warp[][]
  }
  cluster_exchange(R, has_extra ? ncols + 1 : ncols);
}

// The one reduction of a merged launch (m <= kFuseM) as a single 8 x 8 product
// over the fit's rows on the FP64 tensor cores: D = A^T B with the columns
// A = [C_S (m) | c_v] and B = [K C_S (m) | K c_v | k_y], where c_v, K c_v are
// the Gram-Schmidt result of component a - 1 (unnormalised, stored in cvb, kvb
// by this CTA before a block barrier) and k_y the warm start K c_y of component
// a.  Each warp takes 4-row chunks of the CTA's rows (one m8n8k4 per chunk:
// lane l loads column l / 4 of A and of B at row l % 4), the warps' tiles are
// summed in order and then over the cluster: res[8 g + h] = A[:,g] . B[:,h], so
//   res[8 j + k] = C_S[:,j] . K C_S[:,k]   res[8 j + m] = C_S[:,j] . K c_v
//   res[8 j + m + 1] = C_S[:,j] . k_y      res[8 m + k] = c_v . K C_S[:,k]
//   res[8 m + m] = c_v . K c_v             res[8 m + m + 1] = c_v . k_y
static __device__ void fused_dots(ClusterRed& R, const double* CS, const double* KCS, const double* cvb,
                                  const double* kvb, const double* kyb, int n, int m, const Rows& rw) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const double* colA = g < m ? CS + (size_t)g * n : (g == m ? cvb : nullptr);
  const double* colB = g < m ? KCS + (size_t)g * n : (g == m ? kvb : (g == m + 1 ? kyb : nullptr));
  double d0 = 0.0, d1 = 0.0;
  const int nch = (rw.nl + 3) >> 2;
  for (int c0 = warp; c0 < nch; c0 += 4 * kW) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = (c0 + u * kW) * 4 + t;
      const bool ok = r < rw.nl;
      av[u] = (ok && colA) ? colA[rw.r0 + r] : 0.0;
      bv[u] = (ok && colB) ? colB[rw.r0 + r] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) dmma_8x8x4(d0, d1, av[u], bv[u]);
  }
  R.warp[warp][8 * g + 2 * t] = d0;
  R.warp[warp][8 * g + 2 * t + 1] = d1;
  __syncthreads();
  for (int q = threadIdx.x; q < 64; q += kT) {
    double v = 0.0;
    for (int w = 0; w < kW; ++w) v += R.warp[w][q];
    R.part[R.buf][q] = v;
  }
  cluster_exchange(R, 64);
}

// After fused_dots and the normalisation by vn = |v|: fv[j] = S^T v / |v| (the
// deflation coefficients) and fz[zb][..] = the refresh direction after `iters`
// power iterations from the warm start (lanes j < m of warp 0; every thread
// sees the result after the closing block barrier).  Returns zb.
static __device__ int fused_refresh(ClusterRed& R, int m, int iters, double vn) {
  int zb = 0;
  if (threadIdx.x < 32) {
    const int j = threadIdx.x;
    const double vv = R.res[8 * m + m], cky = R.res[8 * m + m + 1] / vn;
    double vj = 0.0;
    if (j < m) {
      vj = R.res[8 * j + m] / vn;
      R.fv[j] = vj;
      R.fz[0][j] = R.res[8 * j + m + 1] - cky * vj;
    }
    __syncwarp();
    const double vvn = vv / (vn * vn);
    for (int it = 1; it < iters; ++it) {
      if (j < m) {
        double t = 0.0;
        for (int k = 0; k < m; ++k) {
          const double vk = R.fv[k];
          const double mjk = R.res[8 * j + k] - vj * vk - vj * (R.res[8 * m + k] / vn) + vj * vk * vvn;
          t += mjk * R.fz[zb][k];
        }
        R.fz[zb ^ 1][j] = t;
      }
      zb ^= 1;
      __syncwarp();
    }
  } else {
    for (int it = 1; it < iters; ++it) zb ^= 1;
  }
  __syncthreads();
  return zb;
}

// Refresh (power iterations of S S^T from the sketch or the warm start),
// Householder normalisation, scores t = X_f r, q = Y^T t, and the loading
// coefficients c_p for the K product.
// In the merged launch (MG) the refresh was already run by dual_b (c_y, K c_y in
// pre_cy, pre_ky) and only the scores part follows.
// The CTA arrives on the closing cluster barrier (arrived = true) once its
// last read of a peer's shared memory is behind it, so that the writes of c_p
// and its digit planes overlap the barrier.
static __device__ bool dual_a(const DualEng& e, int a, ClusterRed& R, const Fixed& P, const Rows& rw, int rank,
                              const double (&pre_cy)[kLR], const double (&pre_ky)[kLR], bool& arrived) {
  __shared__ double wcls[kW][kMaxM + 5];   // per-warp class sums and the reduction's scalars
  const int f = blockIdx.x / kCl;
  const int n = e.n, m = e.m;
  const double* CS = e.CS + (size_t)f * n * m;
  const double* KCS = e.KCS + (size_t)f * n * m;
  double cy[kLR], ky[kLR];
  int steps = e.iters;
  if constexpr (MG) {
#pragma unroll
    for (int k = 0; k < kLR; ++k) {
      cy[k] = pre_cy[k];
      ky[k] = pre_ky[k];
    }
    steps = 0;
  } else if (e.m1) {
#pragma unroll
    for (int k = 0; k < kLR; ++k) {
      cy[k] = rw.ok(k) ? CS[rw.row(k)] : 0.0;
      ky[k] = rw.ok(k) ? KCS[rw.row(k)] : 0.0;
    }
    steps = 0;
  } else {
    // z = S^T (start): the sketch through X Omega at the first component,
    // else the warm start r_{a-1} through its K image.
    const double* src = (a == 0) ? e.XOmega + (size_t)f * n : e.Kcy + (size_t)f * n;
#pragma unroll
    for (int k = 0; k < kLR; ++k) ky[k] = rw.ok(k) ? src[rw.row(k)] : 0.0;
    cluster_dots(R, CS, n, m, rw, ky);
  }
  for (int it = 0; it < steps; ++it) {
    // y = S z: c_y = C_S z, K c_y = (K C_S) z, z in R.res
#pragma unroll
    for (int k = 0; k < kLR; ++k) cy[k] = ky[k] = 0.0;
#pragma unroll 4
    for (int j = 0; j < m; ++j) {
      const double zj = R.res[j];
      const double* cs = CS + (size_t)j * n;
      const double* ks = KCS + (size_t)j * n;
#pragma unroll
      for (int k = 0; k < kLR; ++k)
        if (rw.ok(k)) {
          cy[k] += cs[rw.row(k)] * zj;
          ky[k] += ks[rw.row(k)] * zj;
        }
    }
    if (it + 1 < steps) cluster_dots(R, CS, n, m, rw, ky);
  }
  // One reduction for the refresh result and its scores: ||y||^2 = c_y^T K c_y
  // (all rows), y[0] = Xc[:,0]^T c_y, and over the train rows the class sums,
  // the sum S, the sum of squares Q and the largest magnitude of K c_y (per
  // warp, label-segmented warp sums, warps combined in order).  The scores
  // u = sg K c_y - cmean are then known row by row, and their class sums, sum
  // and norm follow with the exact class counts n_c: sum_c u = sg S_c - cmean n_c,
  // ||u||^2 = sg^2 (Q - S^2 / n_f) when centred (sg^2 Q otherwise).  When the
  // centred sum of squares falls below 1e-6 Q (the train mean dominates the
  // spread) it is taken by a second, exact pass instead.
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* wrow = wcls[warp];
  for (int c = lane; c < m + 5; c += 32) wrow[c] = 0.0;
  __syncwarp();
  double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0, kmax = 0.0;
#pragma unroll
  for (int k = 0; k < kLR; ++k) {
    int lab = -1;
    double kt = 0.0;
    if (rw.ok(k)) {
      const int sl = k * kT + threadIdx.x;
      r0 += cy[k] * ky[k];
      r1 += P.x0[sl] * cy[k];
      if (P.lab[sl] >= 0) {
        kt = ky[k];
        r2 += kt;
        r3 += kt * kt;
        kmax = fmax(kmax, fabs(kt));
        lab = P.lab[sl];
      }
    }
    unsigned pending = __ballot_sync(0xffffffffu, lab >= 0);
    while (pending) {
      const int c = __shfl_sync(0xffffffffu, lab, __ffs(pending) - 1);
      const bool mine = lab == c;
      const double v = warp_sum(mine ? kt : 0.0);
      if (lane == 0) wrow[c] += v;
      pending &= ~__ballot_sync(0xffffffffu, mine);
    }
  }
  r0 = warp_sum(r0);
  r1 = warp_sum(r1);
  r2 = warp_sum(r2);
  r3 = warp_sum(r3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) kmax = fmax(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  if (lane == 0) {
    wrow[m] = r0;
    wrow[m + 1] = r1;
    wrow[m + 2] = r2;
    wrow[m + 3] = r3;
    wrow[m + 4] = kmax;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < m + 5; j += kT) {
    double v = wcls[0][j];
    for (int w = 1; w < kW; ++w) v = (j == m + 4) ? fmax(v, wcls[w][j]) : v + wcls[w][j];
    R.part[R.buf][j] = v;
  }
  cluster_exchange(R, m + 5, m + 4);
  const double nrm = sqrt(R.res[m]);
  const double y0 = R.res[m + 1];
  if (!(nrm > 0.0) || !isfinite(nrm)) {
    if (rank == 0 && threadIdx.x == 0) e.status[f] = 1;
    return false;
  }
  const double sg = ((y0 >= 0.0) ? -1.0 : 1.0) / nrm;
  const double nf = P.nf;
  const double S = R.res[m + 2], Q = R.res[m + 3];
  // U = X r = sg * K c_y; its mean over the train rows centres the scores
  const double cmean = e.center ? sg * S / nf : 0.0;
  const double var = e.center ? Q - S * S / nf : Q;
  const double kmax_all = R.res[m + 4];
  // q = Y^T t: class sums of the centred scores (written now: the exact
  // fallback below reuses the reduction buffer)
  if (rank == 0)
    for (int j = threadIdx.x; j < m; j += kT)
      e.qs[(size_t)f * m + j] = sg * R.res[j] - cmean * P.cnt[j];
#pragma unroll
  for (int k = 0; k < kLR; ++k) ky[k] *= sg;
  double tn2, st;
  if (var > 1e-6 * Q) {
    tn2 = sg * sg * var;
    st = sg * S - (e.center ? nf * cmean : 0.0);
  } else {
    double s2[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < kLR; ++k)
      if (rw.ok(k) && P.lab[k * kT + threadIdx.x] >= 0) {
        const double uc = ky[k] - cmean;
        s2[0] += uc * uc;
        s2[1] += uc;
      }
    cluster_sum(R, s2, 2);
    tn2 = R.res[0];
    st = R.res[1];
  }
  const double tn = sqrt(tn2);
  if (!(tn > 0.0) || !isfinite(tn)) {
    if (rank == 0 && threadIdx.x == 0) e.status[f] = 1;
    return false;
  }
  if constexpr (CL > 1) {
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    arrived = true;
  }
  double* keep = e.Tkeep ? e.Tkeep + ((size_t)f * e.K + a) * n : nullptr;
  // Digit planes of c_p for the INT8 K product: scale 2^ex above the bound
  // (|sg| max |K c_y| + |cmean| + |mean|) / ||t|| of every |c_p[i]|, then the
  // signed 7-bit digits taken exactly (scale by 128, truncate, subtract).
  double inv = 0.0;
  if (e.cpd) {
    const double bound = (fabs(sg) * kmax_all + fabs(cmean) + (e.center ? fabs(st) / nf : 0.0)) / tn *
                         (1.0 + 0x1p-30);
    int ex = 0;
    if (bound > 0.0) frexp(bound, &ex);
    ex = max(-1000, min(1000, ex));
    inv = __longlong_as_double(static_cast<long long>(1023 - ex) << 52);
    if (rank == 0 && threadIdx.x == 0) e.cps[f] = __longlong_as_double(static_cast<long long>(1023 + ex) << 52);
  }
#pragma unroll
  for (int k = 0; k < kLR; ++k) {
    if (!rw.ok(k)) continue;
    const int i = rw.row(k);
    const double uc = ky[k] - cmean;
    if (keep) keep[i] = uc;
    const double c = P.lab[k * kT + threadIdx.x] >= 0 ? (uc - (e.center ? st / nf : 0.0)) / tn : 0.0;
    e.cp[(size_t)f * n + i] = c;
    e.Kcy[(size_t)f * n + i] = ky[k] / tn;
    if (e.cpd) {
      int8_t* d = e.cpd + (size_t)f * e.cpldk + i;
      double x = c * inv;
      for (int sl = 0; sl < e.cpS; ++sl) {
        x *= 128.0;
        const double dg = trunc(x);
        x -= dg;
        d[(size_t)sl * e.cpstride] = static_cast<int8_t>(static_cast<int>(dg));
      }
    }
  }
  if (rank == 0) {
    if (threadIdx.x == 0) {
      e.scal[2 * f] = tn;
      e.scal[2 * f + 1] = st;
    }
  }
  return true;
}

// Gram-Schmidt of the loading against the earlier ones in K-coordinates,
// normalisation, rank-1 deflation of C_S and K C_S, and the component outputs.
// In the merged launch (MG: m <= kFuseM, launches between the first and the
// last) the refresh of component a + 1 rides on this component's reduction:
// the merged dots give z0 = C_S'^T k_y for the deflated C_S' and the m x m matrix
// M' = C_S'^T K C_S' = S'^T S' in closed form (M' = M - v v^T - v e^T / |v|
// + v v^T c_v.Kc_v / |v|^2), the power iterations z <- M' z run on it, and the
// deflation pass accumulates c_y = C_S' z and K c_y = K C_S' z (into fcy, fky)
// as it writes C_S' and K C_S'.  This saves two cluster reductions and one pass
// over C_S and K C_S per launch.
// On entry cv holds c_p of component a (this thread's rows) and, for a > 0,
// R.res[0 .. a) the Gram-Schmidt coefficients C_V^T K c_p (taken by run()
// before the dependency wait).
static __device__ bool dual_b(const DualEng& e, int a, ClusterRed& R, const Rows& rw, int rank,
                              const int (&ks0)[kLR], const int (&ks1)[kLR], double (&cv)[kLR],
                              double (&fcy)[kLR], double (&fky)[kLR]) {
  const int f = blockIdx.x / kCl;
  const int n = e.n, m = e.m, K = e.K;
  double* CV = e.CV + (size_t)f * n * K;
  double* KCV = e.KCV + (size_t)f * n * K;
  double* CS = e.CS + (size_t)f * n * m;
  double* KCS = e.KCS + (size_t)f * n * m;
  double kv[kLR];
#pragma unroll
  for (int k = 0; k < kLR; ++k) {
    kv[k] = 0.0;
    if (!rw.ok(k)) continue;
    const int i = rw.row(k);
    if (e.kpart) {
      // the tile's segments in order, eight loads in flight at a time
      const double* pp = e.kpart + (size_t)(f & 63) * 128 + (i & 127);
      double v = 0.0;
      for (int s0 = ks0[k]; s0 < ks1[k]; s0 += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = s0 + u < ks1[k] ? pp[(size_t)(s0 + u) * 64 * 128] : 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (s0 + u < ks1[k]) v += t[u];
      }
      kv[k] = v;
    } else {
      kv[k] = e.Gp[(size_t)f * n + i];
    }
  }
  if (a > 0) {
#pragma unroll (kColUnroll)
    for (int l = 0; l < a; ++l) {
      const double wl = R.res[l];
      const double* vc = CV + (size_t)l * n;
      const double* vk = KCV + (size_t)l * n;
#pragma unroll
      for (int k = 0; k < kLR; ++k)
        if (rw.ok(k)) {
          cv[k] -= vc[rw.row(k)] * wl;
          kv[k] -= vk[rw.row(k)] * wl;
        }
    }
  }
  if constexpr (MG) {
    // the unnormalised c_v, K c_v go to this component's columns first: the
    // reduction reads them across the CTA's threads
#pragma unroll
    for (int k = 0; k < kLR; ++k)
      if (rw.ok(k)) {
        CV[rw.row(k) + (size_t)a * n] = cv[k];
        KCV[rw.row(k) + (size_t)a * n] = kv[k];
      }
    __syncthreads();
    fused_dots(R, CS, KCS, CV + (size_t)a * n, KCV + (size_t)a * n, e.Kcy + (size_t)f * n, n, m, rw);
    const double vv = R.res[8 * m + m];
    const double vn = sqrt(vv);
    if (!(vn > 0.0) || !isfinite(vn)) {
      if (rank == 0 && threadIdx.x == 0) e.status[f] = 1;
      return false;
    }
#pragma unroll
    for (int k = 0; k < kLR; ++k) {
      cv[k] /= vn;
      kv[k] /= vn;
      if (rw.ok(k)) {
        CV[rw.row(k) + (size_t)a * n] = cv[k];
        KCV[rw.row(k) + (size_t)a * n] = kv[k];
      }
    }
    const int zb = fused_refresh(R, m, e.iters, vn);
#pragma unroll
    for (int k = 0; k < kLR; ++k) fcy[k] = fky[k] = 0.0;
    // (kFC columns per chunk: two in the register-capped 512-thread layout)
    constexpr int kFC = kLR <= 2 ? 2 : 4;
#pragma unroll
    for (int j0 = 0; j0 < kFuseM; j0 += kFC) {
      if (j0 >= m) break;
      double csv[kFC][kLR], ksv[kFC][kLR];
#pragma unroll
      for (int jj = 0; jj < kFC; ++jj) {
        const int j = min(j0 + jj, m - 1);
#pragma unroll
        for (int k = 0; k < kLR; ++k) {
          csv[jj][k] = rw.ok(k) ? CS[(size_t)j * n + rw.row(k)] : 0.0;
          ksv[jj][k] = rw.ok(k) ? KCS[(size_t)j * n + rw.row(k)] : 0.0;
        }
      }
#pragma unroll
      for (int jj = 0; jj < kFC; ++jj) {
        if (j0 + jj >= m || j0 + jj >= kFuseM) break;
        const double vj = R.fv[j0 + jj], zj = R.fz[zb][j0 + jj];
        double* cs = CS + (size_t)(j0 + jj) * n;
        double* ks = KCS + (size_t)(j0 + jj) * n;
#pragma unroll
        for (int k = 0; k < kLR; ++k)
          if (rw.ok(k)) {
            const double cn = csv[jj][k] - cv[k] * vj;
            const double kn = ksv[jj][k] - kv[k] * vj;
            cs[rw.row(k)] = cn;
            ks[rw.row(k)] = kn;
            fcy[k] += cn * zj;
            fky[k] += kn * zj;
          }
      }
    }
  } else {
    // ||v||^2 = c_v^T K c_v and S^T v = C_S^T K c_v in one reduction (the
    // normalisation only rescales the dots)
    double vv = 0.0;
#pragma unroll
    for (int k = 0; k < kLR; ++k) vv += cv[k] * kv[k];
    cluster_dots(R, CS, n, m, rw, kv, true, vv);
    const double vn = sqrt(R.res[m]);
    if (!(vn > 0.0) || !isfinite(vn)) {
      if (rank == 0 && threadIdx.x == 0) e.status[f] = 1;
      return false;
    }
#pragma unroll
    for (int k = 0; k < kLR; ++k) {
      cv[k] /= vn;
      kv[k] /= vn;
      if (rw.ok(k)) {
        CV[rw.row(k) + (size_t)a * n] = cv[k];
        KCV[rw.row(k) + (size_t)a * n] = kv[k];
      }
    }
    // Rank-1 deflation of C_S and K C_S, four columns at a time: every load of
    // a chunk is issued before its stores (the stores could alias later loads,
    // which would otherwise serialise each column's read-modify-write).
    for (int j0 = 0; j0 < m; j0 += 4) {
      double csv[4][kLR], ksv[4][kLR];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int j = min(j0 + jj, m - 1);
#pragma unroll
        for (int k = 0; k < kLR; ++k) {
          csv[jj][k] = rw.ok(k) ? CS[(size_t)j * n + rw.row(k)] : 0.0;
          ksv[jj][k] = rw.ok(k) ? KCS[(size_t)j * n + rw.row(k)] : 0.0;
        }
      }
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        if (j0 + jj >= m) break;
        const double vj = R.res[j0 + jj] / vn;
        double* cs = CS + (size_t)(j0 + jj) * n;
        double* ks = KCS + (size_t)(j0 + jj) * n;
#pragma unroll
        for (int k = 0; k < kLR; ++k)
          if (rw.ok(k)) {
            cs[rw.row(k)] = csv[jj][k] - cv[k] * vj;
            ks[rw.row(k)] = ksv[jj][k] - kv[k] * vj;
          }
      }
    }
  }
  if (rank == 0) {
    const double tn = e.scal[2 * f], st = e.scal[2 * f + 1];
    double* Qcol = e.Q + ((size_t)f * K + a) * m;
    for (int j = threadIdx.x; j < m; j += kT) {
      const double off = e.mY_all[j] + (e.dY ? e.dY[(size_t)f * m + j] : 0.0);
      Qcol[j] = (e.qs[(size_t)f * m + j] - off * st) / tn;
    }
    if (threadIdx.x == 0) {
      e.tnorm[(size_t)f * K + a] = tn;
      e.ncomp_done[f] = a + 1;
    }
  }
  return true;
}

// One launch per component boundary: the Gram-Schmidt / deflation of
// component a - 1 and then the refresh / scores of component a, per fit.
static __device__ void run(const DualEng& e, int a) {
  __shared__ ClusterRed R;
  const int f = blockIdx.x / kCl;
  int rank = 0;
  if constexpr (CL > 1) rank = static_cast<int>(cg::this_cluster().block_rank());
  const int rows_per = (e.n + kCl - 1) / kCl;
  Rows rw;
  rw.r0 = rank * rows_per;
  rw.nl = max(0, min(e.n, rw.r0 + rows_per) - rw.r0);
  // Segment ranges of the K-product partials of this thread's rows: the plan's
  // table was written when the plan was made, so it is read before the wait.
  int ks0[kLR], ks1[kLR];
#pragma unroll
  for (int k = 0; k < kLR; ++k) {
    ks0[k] = ks1[k] = 0;
    if (a > 0 && e.kpart && rw.ok(k)) {
      const int tile = (rw.row(k) >> 7) * e.kntn + (f >> 6);
      ks0[k] = e.kseg[tile];
      ks1[k] = e.kseg[tile + 1];
    }
  }
  __shared__ Fixed P;
#pragma unroll
  for (int k = 0; k < kLR; ++k)
    if (rw.ok(k)) {
      const int i = rw.row(k);
      P.x0[k * kT + threadIdx.x] = e.x0[i];
      P.lab[k * kT + threadIdx.x] = e.mask[(size_t)f * e.n + i] ? static_cast<signed char>(e.labels[i]) : -1;
    }
  for (int j = threadIdx.x; j < e.m; j += kT) P.cnt[j] = e.class_cnt[(size_t)f * e.m + j];
  if (threadIdx.x == 0) P.nf = static_cast<double>(e.ntrain[f]);
  // The product this grid depends on releases it only after its own wait, so
  // the step launch before it has completed: its outputs (c_p, K C_V, the fit
  // status) are read through L2 before this grid's wait, and the Gram-Schmidt
  // coefficients of component a - 1, C_V^T K c_p = (K C_V)^T c_p (K is
  // symmetric), are reduced while the product finishes.
  if (__ldcg(e.status + f)) return;   // set only in earlier launches: uniform over the cluster
  if (threadIdx.x == 0) R.buf = 0;
  __syncthreads();
  double cv[kLR];
#pragma unroll
  for (int k = 0; k < kLR; ++k) cv[k] = 0.0;
  if (a > 0) {
#pragma unroll
    for (int k = 0; k < kLR; ++k) cv[k] = rw.ok(k) ? __ldcg(e.cp + (size_t)f * e.n + rw.row(k)) : 0.0;
    if (a > 1) cluster_dots<true>(R, e.KCV + (size_t)f * e.n * e.K, e.n, a - 1, rw, cv);
  }
  tc::grid_dep_wait();     // the previous product has completed
  tc::grid_dep_launch();
  // Every CTA of the cluster takes the same branches (they follow the
  // cluster-wide sums, identical in all CTAs), and all of them end on the same
  // cluster barrier, which also keeps each CTA's shared memory alive until the
  // last remote read of it.
  // MG (the merged launch) is chosen by the host for 0 < a < K when the fit
  // set allows it (e.merge).
  bool ok = true;
  double fcy[kLR], fky[kLR];
  if (a > 0) ok = dual_b(e, a - 1, R, rw, rank, ks0, ks1, cv, fcy, fky);
  bool arrived = false;
  if (ok && a < e.K) dual_a(e, a, R, P, rw, rank, fcy, fky, arrived);
  if constexpr (CL > 1) {
    if (!arrived) asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
}
};  // struct Step

// 512-thread CTAs are held to 64 registers so that two fit on an SM and the
// 240 CTAs of a 60-fit grid run in one wave.
template <int CL, int T, int LR, bool MG>
__global__ void __launch_bounds__(T, T >= 512 ? 2 : 1) k_dual_step(DualEng e, int a) {
  Step<CL, T, LR, MG>::run(e, a);
}

__global__ void symmetrize_kernel(double* K, int n) {
  const size_t total = (size_t)n * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % n), j = static_cast<int>(t / n);
    if (i < j) {
      const double v = 0.5 * (K[t] + K[j + (size_t)i * n]);
      K[t] = v;
      K[j + (size_t)i * n] = v;
    }
  }
}

}  // namespace

void symmetrize(double* K, int n) {
  Context& ctx = Context::get();
  symmetrize_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(K, n); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

namespace {

template <int CL, int T, int LR, bool MG>
void launch_step_cfg(const DualEng& e, int a, int F, cudaStream_t st) {
  if constexpr (CL == 1) {
    k_dual_step<1, T, LR, MG><<<F, T, 0, st>>>(e, a);
  } else {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(F * CL);
    lc.blockDim = dim3(T);
    lc.dynamicSmemBytes = 0;
    lc.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = tc::pdl_enabled() ? 2 : 1;
    FPLS_CUDA(cudaLaunchKernelEx(&lc, k_dual_step<CL, T, LR, MG>, e, a));
  }
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

// Step layouts (rows of a fit over a 4-CTA cluster): 512 threads with up to 2
// rows each for n <= 4096, 256 threads with up to 8 rows each for n <= 8192.
// On the 3000-row omics grid the 512-thread layout beat one CTA per fit
// (768 threads), 2-CTA clusters, 8-CTA clusters and 1024-thread CTAs: the
// step is bound by the loads each SM keeps in flight, and more CTAs per
// cluster cost more in the cluster reductions than they add.
enum StepLayout { kStepWide = 0, kStepDeep = 1 };

int choose_step_layout(int n) {
  const bool wide_fits = n <= 4 * 512 * 2;
  if (const char* v = std::getenv("FASTPLS_DUAL_STEP"))
    if (std::string(v) == "deep") return kStepDeep;
  if (active_tune().step_layout == 1) return kStepDeep;
  return wide_fits ? kStepWide : kStepDeep;
}

void launch_step(int layout, const DualEng& e, int a, int F, cudaStream_t st) {
  const bool mg = e.merge && a > 0 && a < e.K;
  if (layout == kStepWide) {
    if (mg) launch_step_cfg<4, 512, 2, true>(e, a, F, st);
    else launch_step_cfg<4, 512, 2, false>(e, a, F, st);
  } else {
    if (mg) launch_step_cfg<4, 256, 8, true>(e, a, F, st);
    else launch_step_cfg<4, 256, 8, false>(e, a, F, st);
  }
}

}  // namespace

// FASTPLS_DUAL_MERGE=0 runs the refresh of every component in its own
// reductions (the unmerged launch) instead.
static bool dual_merge_enabled() {
  if (const char* v = std::getenv("FASTPLS_DUAL_MERGE")) return v[0] != '0';
  return active_tune().merge != 0;
}

// FASTPLS_LOOP_GRAPH=0 enqueues the component loop launch by launch instead of
// as one CUDA graph.
static bool loop_graph_enabled() {
  static const int v = [] {
    const char* e = std::getenv("FASTPLS_LOOP_GRAPH");
    return e ? (e[0] != '0' ? 1 : 0) : 1;
  }();
  return v != 0;
}

// The executable graph of the last captured component loop.  Each call
// captures its loop afresh and updates this graph in place when the topology
// matches (same launches, new parameters), else instantiates a new one; an
// update does not touch launches of the graph already in flight.
static cudaGraphExec_t g_loop_exec = nullptr;

template <typename Loop>
static void launch_as_graph(cudaStream_t st, Loop&& loop) {
  FPLS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaGraph_t graph = nullptr;
  try {
    loop();
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  FPLS_CUDA(cudaStreamEndCapture(st, &graph));
  bool updated = false;
  if (g_loop_exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(g_loop_exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(g_loop_exec);
      g_loop_exec = nullptr;
    }
  }
  cudaError_t e = cudaSuccess;
  if (!updated) e = cudaGraphInstantiate(&g_loop_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g_loop_exec = nullptr;
    FPLS_CUDA(e);
  }
  FPLS_CUDA(cudaGraphLaunch(g_loop_exec, st));
}

bool dual_engine_applies(int n, int p, int m, int K) {
  if (const char* e = std::getenv("FASTPLS_DUAL"))
    if (e[0] == '0') return false;
  return n >= 2 && n <= kMaxN && 2 * n <= p && m <= kMaxM && K <= kMaxK;
}

void dual_simpls_run(const DualBatch& b) {
  Context& ctx = Context::get();
  Arena& ar = ctx.arena;
  FPLS_REQUIRE(dual_engine_applies(b.n, 2 * b.n, b.m, b.K), "dual SIMPLS: shape outside its limits");
  DualEng e{};
  e.n = b.n; e.m = b.m; e.F = b.F; e.K = b.K;
  e.iters = b.m1_mode ? 0 : std::max(b.power_iters, 0);
  e.m1 = b.m1_mode ? 1 : 0;
  e.center = b.center ? 1 : 0;
  e.merge = (!e.m1 && e.iters >= 1 && e.m <= kFuseM && dual_merge_enabled()) ? 1 : 0;
  e.x0 = b.x0; e.XOmega = b.XOmega; e.mask = b.mask; e.labels = b.labels; e.mY_all = b.mY_all; e.dY = b.dY;
  e.Q = b.Q; e.tnorm = b.tnorm; e.Tkeep = b.Tkeep; e.ncomp_done = b.ncomp_done; e.status = b.status;
  const size_t F = b.F, n = b.n, m = b.m, K = b.K;
  e.CS = ar.alloc_n<double>(F * n * m);
  e.KCS = ar.alloc_n<double>(F * n * m);
  e.CV = ar.alloc_n<double>(F * n * K);
  e.KCV = ar.alloc_n<double>(F * n * K);
  e.Kcy = ar.alloc_n<double>(F * n);
  e.cp = ar.alloc_n<double>(F * n);
  e.Gp = ar.alloc_n<double>(F * n);
  e.scal = ar.alloc_n<double>(2 * F);
  e.qs = ar.alloc_n<double>(F * m);
  e.ntrain = b.ntrain;
  FPLS_REQUIRE(b.class_cnt != nullptr, "dual SIMPLS: class counts missing");
  e.class_cnt = b.class_cnt;
  OzakiPlanes cpP;
  if (b.kop_int8_slices > 0) {
    cpP = ozaki_alloc(b.F, b.n, b.kop_int8_slices);
    dzero(cpP.data, (size_t)cpP.slices * cpP.rows_pad * cpP.ldk);
    dzero(cpP.scale, (size_t)cpP.rows_pad * sizeof(double));
    e.cpd = cpP.data;
    e.cps = cpP.scale;
    e.cpldk = cpP.ldk;
    e.cpS = cpP.slices;
    e.cpstride = (size_t)cpP.rows_pad * cpP.ldk;
  }
  dzero(b.status, F * sizeof(int));
  dzero(b.ncomp_done, F * sizeof(int));
  dzero(b.Q, F * m * K * sizeof(double));
  dzero(b.tnorm, F * K * sizeof(double));
  cudaStream_t st = ctx.stream;
  const int cfg = choose_step_layout(b.n);
  k_dual_cs0<<<2 * ctx.sm_count, 256, 0, st>>>(e); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  b.Kop->times(e.CS, static_cast<int>(F * m), e.KCS);   // K C_S for every fit
  PhaseTimer pt("dual SIMPLS engine");
  const double nd = static_cast<double>(n), md = static_cast<double>(m), Fd = static_cast<double>(F);
  const double it = static_cast<double>(e.iters);
  // With INT8 K products the component loop is captured as one CUDA graph
  // (not while the kernel-class profiler or the phase trace records events
  // between its launches); the product's plan and kernel attribute are made
  // before the capture, which then holds launches only.
  const bool graph = b.kop_int8_slices > 0 && loop_graph_enabled() && !ctx.profile && !pt.enabled();
  if (graph) ozaki_sym_prepare_partials(*b.Kop, cpP);
  auto loop = [&]() {
  for (int a = 0; a <= b.K; ++a) {
    // algorithmic bytes of one step launch (all fits): the Gram-Schmidt and
    // deflation of component a - 1 and the refresh / scores of component a
    // (merged launch: c_p, K c_p, the 3 (a - 1) Gram-Schmidt columns, c_v and
    // K c_v stored twice, the 8 x 8 product's 2m + 3 columns, the deflation's
    // 4m, and x0, t, c_p, K c_y of the scores part)
    double words = 0.0;
    if (e.merge && a > 0 && a < b.K) {
      words = (13.0 + 3.0 * (a - 1) + 6.0 * md) * nd;
    } else {
      if (a > 0) words += (4.0 + 3.0 * (a - 1) + 5.0 * md) * nd;
      if (a < b.K) words += (5.0 + md + 2.0 * it * md + std::max(it - 1.0, 0.0) * md) * nd;
    }
    const int slot = ctx.prof_begin("dual_step", st);
    launch_step(cfg, e, a, b.F, st);
    ctx.prof_end(slot, st, Fd * (8.0 * words + (a < b.K ? 5.0 * nd : 0.0)), 0.0);
    pt.mark("per-fit steps");
    if (a == b.K) break;
    if (b.kop_int8_slices > 0) {
      // digit planes of K and of the F coefficient columns, the FP64 columns in
      // and out; the S (S + 1) / 2 int8 plane products.  The next step sums
      // the stream-K partials as it reads K c_p.
      const double S = b.kop_int8_slices;
      const int ks = ctx.prof_begin("k_products_int8", st);
      const OzakiPartials pp = ozaki_sym_partials_from_planes(*b.Kop, cpP);
      e.kpart = pp.part;
      e.kseg = pp.tile_seg;
      e.kntn = pp.n_tiles_n;
      ctx.prof_end(ks, st, S * nd * nd + S * nd * Fd + 16.0 * nd * Fd, 0.5 * S * (S + 1.0) * 2.0 * nd * nd * Fd);
    } else {
      const int ks = ctx.prof_begin("k_products_f64", st);
      b.Kop->times(e.cp, b.F, e.Gp);
      ctx.prof_end(ks, st, 8.0 * (nd * nd + 2.0 * nd * Fd), 2.0 * nd * nd * Fd);
    }
    pt.mark("K products");
  }
  };
  if (graph) launch_as_graph(st, loop);
  else loop();
  pt.report();
}

void dual_release_graph() {
  if (g_loop_exec) cudaGraphExecDestroy(g_loop_exec);
  g_loop_exec = nullptr;
}

}  // namespace fpls
