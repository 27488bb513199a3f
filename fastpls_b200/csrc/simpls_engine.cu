#include "blas_f64.cuh"
#include "context.cuh"
#include "simpls_engine.cuh"

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <string>
#include <typeinfo>
#include <vector>

namespace fpls {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct Eng {
  int n, p, m, F, K, cp, cn, szp, szn;
  const double* Yg;
  const int* labels;
  const double* mY_all;
  const uint8_t* mask;
  const double* delta;
  const double* colsum;
  const double* colscale;
  const double* dY;
  double* S;
  const double* omega;
  int m1_mode;
  int iters;
  double* R;
  double* Q;
  double* V;
  double* tnorm;
  double* Tkeep;
  int* ncomp_done;
  int* status;
  // workspace
  double* y;       // F x p
  double* zA;      // F x cp x m
  double* zB;      // F x cp x m
  double* npart;   // F x cp
  double* r;       // F x p (unit r before the t normalisation)
  double* Rhat;    // p x F
  double* cpart;   // F x cp
  double* U;       // n x F
  double* T;       // n x F
  double* tpart;   // F x cn x 2
  double* qpart;   // F x cn x m
  double* P;       // p x F
  double* pv;      // F x p
  double* wpart;   // F x cp x K
  double* v;       // F x p
  double* vpart;   // F x cp
  double* vSpart;  // F x cp x m
};

__device__ __forceinline__ void chunk_range(int chunk, int sz, int total, int& b, int& e) {
  b = chunk * sz;
  e = min(total, b + sz);
}

__device__ __forceinline__ double sum_parts(const double* parts, int count, int stride) {
  double s = 0.0;
  for (int c = 0; c < count; ++c) s += parts[(size_t)c * stride];
  return s;
}

// Block-wide sums of the first `count` entries of a per-thread vector; the
// result is written to out[0..count) by threads 0..count-1.  One pass of warp
// shuffles per entry and a single shared-memory exchange for all entries.
template <int NV>
__device__ __forceinline__ void block_sum_vec(double (&v)[NV], int count, double* out, int out_stride) {
  __shared__ double sm[kWarps][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    if (j < count) {
      const double w = warp_sum(v[j]);
      if (lane == 0) sm[warp][j] = w;
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < count; j += blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s += sm[w][j];
    out[(size_t)j * out_stride] = s;
  }
  __syncthreads();
}

constexpr int NV = 16;      // register block of per-thread partial sums
constexpr int kMaxChunk = 4096;  // rows of a chunk staged in shared memory

// out[j * out_stride] = sum_{r < rows} M[r + j*ld] * xs[r] for j < ncols, with xs
// (the chunk's vector) in shared memory.  Warps take columns; when there are
// fewer columns than warps, several warps split the rows of one column.  Each
// lane streams consecutive rows, so every column read is coalesced.
__device__ void chunk_dots(const double* __restrict__ M, size_t ld, int ncols,
                           const double* xs, int rows, double* out, int out_stride) {
  __shared__ double red[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (ncols >= kWarps) {
    for (int j = warp; j < ncols; j += kWarps) {
      const double* col = M + (size_t)j * ld;
      double a0 = 0.0, a1 = 0.0;
      int r = lane;
      for (; r + 32 < rows; r += 64) {
        a0 += col[r] * xs[r];
        a1 += col[r + 32] * xs[r + 32];
      }
      if (r < rows) a0 += col[r] * xs[r];
      const double acc = warp_sum(a0 + a1);
      if (lane == 0) out[(size_t)j * out_stride] = acc;
    }
    return;
  }
  const int g = kWarps / max(ncols, 1);   // warps per column
  const int j = warp / g, sub = warp % g;
  double acc = 0.0;
  if (j < ncols) {
    const double* col = M + (size_t)j * ld;
    for (int r = sub * 32 + lane; r < rows; r += 32 * g) acc += col[r] * xs[r];
  }
  acc = warp_sum(acc);
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x < ncols) {
    double t = 0.0;
    for (int u = 0; u < g; ++u) t += red[threadIdx.x * g + u];
    out[(size_t)threadIdx.x * out_stride] = t;
  }
  __syncthreads();
}

// Partials of S_f^T y over the chunk (y staged in ys), or the chunk's ||y||^2.
__device__ __forceinline__ void chunk_StY(const Eng& e, int f, int chunk, const double* Sf,
                                          const double* ys, int b, int en, double* zout,
                                          bool norm_only) {
  if (norm_only) {
    __shared__ double scratch[32];
    double s2 = 0.0;
    for (int r = threadIdx.x; r < en - b; r += blockDim.x) s2 += ys[r] * ys[r];
    s2 = block_sum(s2, scratch);
    if (threadIdx.x == 0) e.npart[(size_t)f * e.cp + chunk] = s2;
    return;
  }
  chunk_dots(Sf + b, e.p, e.m, ys, en - b, zout + ((size_t)f * e.cp + chunk) * e.m, 1);
}

// First component's refresh start: y = Omega (or the single column of S).
__global__ void k_refresh_start(Eng e) {
  __shared__ double ys[kMaxChunk];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  const double* Sf = e.S + (size_t)f * e.p * e.m;
  const double* y0 = e.m1_mode ? Sf : e.omega + (size_t)f * e.p;
  double* yf = e.y + (size_t)f * e.p;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    yf[i] = y0[i];
    ys[i - b] = y0[i];
  }
  __syncthreads();
  chunk_StY(e, f, chunk, Sf, ys, b, en, e.zA, e.iters == 0);
}

// y <- S z with z = sum of the partials of S^T y; then the next partials (or ||y||^2).
__global__ void k_refresh_apply(Eng e, const double* zin, double* zout, int last) {
  extern __shared__ double zs[];
  __shared__ double ys[kMaxChunk];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  for (int j = threadIdx.x; j < e.m; j += blockDim.x)
    zs[j] = sum_parts(zin + (size_t)f * e.cp * e.m + j, e.cp, e.m);
  __syncthreads();
  const double* Sf = e.S + (size_t)f * e.p * e.m;
  double* yf = e.y + (size_t)f * e.p;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < e.m; ++j) acc += Sf[i + (size_t)j * e.p] * zs[j];
    yf[i] = acc;
    ys[i - b] = acc;
  }
  __syncthreads();
  chunk_StY(e, f, chunk, Sf, ys, b, en, zout, last != 0);
}

// r = -sign(y0) y / ||y|| (Householder QR of a single column; the 1 x m core
// SVD from gesvd keeps U = 1).  Rhat = colscale * r; cpart = delta . Rhat.
__global__ void k_refresh_finish(Eng e) {
  __shared__ double scratch[32];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  const double nrm = sqrt(sum_parts(e.npart + (size_t)f * e.cp, e.cp, 1));
  if (!(nrm > 0.0) || !isfinite(nrm)) {
    // Degenerate refresh: the reference's refresh returns false and the loop stops.
    if (chunk == 0 && threadIdx.x == 0) e.status[f] = 1;
    return;
  }
  const double* yf = e.y + (size_t)f * e.p;
  const double sgn = (yf[0] >= 0.0) ? -1.0 : 1.0;
  const double* sc = e.colscale ? e.colscale + (size_t)f * e.p : nullptr;
  const double* dl = e.delta ? e.delta + (size_t)f * e.p : nullptr;
  double c = 0.0;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    const double ri = sgn * yf[i] / nrm;
    e.r[(size_t)f * e.p + i] = ri;
    const double rh = sc ? ri * sc[i] : ri;
    e.Rhat[(size_t)f * e.p + i] = rh;
    if (dl) c += dl[i] * rh;
  }
  if (dl) {
    c = block_sum(c, scratch);
    if (threadIdx.x == 0) e.cpart[(size_t)f * e.cp + chunk] = c;
  }
}

// t = mask * (U - delta.rhat); partial sums of t^2, t and q = Y^T t.
__global__ void k_scores(Eng e, int a) {
  extern __shared__ double qs[];
  __shared__ double ts[kMaxChunk];
  __shared__ double scratch[32];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  int b, en;
  chunk_range(chunk, e.szn, e.n, b, en);
  const double c = e.delta ? sum_parts(e.cpart + (size_t)f * e.cp, e.cp, 1) : 0.0;
  const uint8_t* mk = e.mask ? e.mask + (size_t)f * e.n : nullptr;
  const double* Uf = e.U + (size_t)f * e.n;
  double* Tf = e.T + (size_t)f * e.n;
  double* keep = e.Tkeep ? e.Tkeep + ((size_t)f * e.K + a) * e.n : nullptr;
  if (e.labels) {
    for (int j = threadIdx.x; j < e.m; j += blockDim.x) qs[j] = 0.0;
    __syncthreads();
  }
  double s2 = 0.0, s1 = 0.0;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    const double u = Uf[i] - c;
    const double t = (mk && !mk[i]) ? 0.0 : u;
    Tf[i] = t;
    ts[i - b] = t;
    if (keep) keep[i] = u;
    s2 += t * t;
    s1 += t;
    if (e.labels && t != 0.0) atomicAdd(&qs[e.labels[i]], t);
  }
  s2 = block_sum(s2, scratch);
  s1 = block_sum(s1, scratch);
  if (threadIdx.x == 0) {
    e.tpart[((size_t)f * e.cn + chunk) * 2 + 0] = s2;
    e.tpart[((size_t)f * e.cn + chunk) * 2 + 1] = s1;
  }
  double* qp = e.qpart + ((size_t)f * e.cn + chunk) * e.m;
  if (e.labels) {
    for (int j = threadIdx.x; j < e.m; j += blockDim.x) qp[j] = qs[j];
    return;
  }
  chunk_dots(e.Yg + b, e.n, e.m, ts, en - b, qp, 1);
}

__device__ __forceinline__ void t_stats(const Eng& e, int f, double& tn, double& st) {
  double s2 = 0.0, s1 = 0.0;
  const double* tp = e.tpart + (size_t)f * e.cn * 2;
  for (int c = 0; c < e.cn; ++c) {
    s2 += tp[2 * c];
    s1 += tp[2 * c + 1];
  }
  tn = sqrt(s2);
  st = s1;
}

// p = colscale * (P - delta * sum(t)) / ||t||; partial w = V^T p.
__global__ void k_loading(Eng e, int a) {
  __shared__ double ps[kMaxChunk];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  double tn, st;
  t_stats(e, f, tn, st);
  if (!(tn > 0.0) || !isfinite(tn)) {
    if (chunk == 0 && threadIdx.x == 0) e.status[f] = 1;
    return;
  }
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  const double* sc = e.colscale ? e.colscale + (size_t)f * e.p : nullptr;
  const double* dl = e.delta ? e.delta + (size_t)f * e.p : nullptr;
  const double* Pf = e.P + (size_t)f * e.p;
  double* pf = e.pv + (size_t)f * e.p;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    double v = Pf[i];
    if (dl) v -= dl[i] * st;
    if (sc) v *= sc[i];
    v /= tn;
    pf[i] = v;
    ps[i - b] = v;
  }
  __syncthreads();
  if (a > 0)
    chunk_dots(e.V + (size_t)f * e.p * e.K + b, e.p, a, ps, en - b,
               e.wpart + ((size_t)f * e.cp + chunk) * e.K, 1);
}

// v = p - V (V^T p); partials of ||v||^2 and of S^T v.
__global__ void k_orth(Eng e, int a) {
  extern __shared__ double ws[];
  __shared__ double vsh[kMaxChunk];
  __shared__ double scratch[32];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  for (int l = threadIdx.x; l < a; l += blockDim.x)
    ws[l] = sum_parts(e.wpart + (size_t)f * e.cp * e.K + l, e.cp, e.K);
  __syncthreads();
  const double* Vf = e.V + (size_t)f * e.p * e.K;
  const double* pf = e.pv + (size_t)f * e.p;
  double* vf = e.v + (size_t)f * e.p;
  double s2 = 0.0;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    double x = pf[i];
    int l = 0;
    for (; l + 4 <= a; l += 4) {
      const double v0 = Vf[i + (size_t)l * e.p], v1 = Vf[i + (size_t)(l + 1) * e.p];
      const double v2 = Vf[i + (size_t)(l + 2) * e.p], v3 = Vf[i + (size_t)(l + 3) * e.p];
      x -= v0 * ws[l] + v1 * ws[l + 1] + v2 * ws[l + 2] + v3 * ws[l + 3];
    }
    for (; l < a; ++l) x -= Vf[i + (size_t)l * e.p] * ws[l];
    vf[i] = x;
    vsh[i - b] = x;
    s2 += x * x;
  }
  s2 = block_sum(s2, scratch);
  if (threadIdx.x == 0) e.vpart[(size_t)f * e.cp + chunk] = s2;
  // S^T v (unnormalised) for the deflation.
  chunk_dots(e.S + (size_t)f * e.p * e.m + b, e.p, e.m, vsh, en - b,
             e.vSpart + ((size_t)f * e.cp + chunk) * e.m, 1);
}

// v /= ||v||; V[:, a] = v; S -= v (v^T S); R[:, a] = r / ||t||; Q[:, a] = q / ||t||;
// then the next component's refresh start (partials of S^T r_a over the
// deflated S, or ||S[:,0]||^2 when m == 1).
__global__ void k_deflate(Eng e, int a, int next) {
  extern __shared__ double vs[];
  __shared__ double ysh[kMaxChunk];
  const int f = blockIdx.y, chunk = blockIdx.x;
  if (e.status[f]) return;
  const double vn = sqrt(sum_parts(e.vpart + (size_t)f * e.cp, e.cp, 1));
  if (!(vn > 0.0) || !isfinite(vn)) {
    if (chunk == 0 && threadIdx.x == 0) e.status[f] = 1;
    return;
  }
  int b, en;
  chunk_range(chunk, e.szp, e.p, b, en);
  for (int j = threadIdx.x; j < e.m; j += blockDim.x)
    vs[j] = sum_parts(e.vSpart + (size_t)f * e.cp * e.m + j, e.cp, e.m) / vn;
  __syncthreads();
  double tn, st;
  t_stats(e, f, tn, st);
  double* Sf = e.S + (size_t)f * e.p * e.m;
  double* vf = e.v + (size_t)f * e.p;
  double* Vcol = e.V + ((size_t)f * e.K + a) * e.p;
  double* Rcol = e.R + ((size_t)f * e.K + a) * e.p;
  const double* rf = e.r + (size_t)f * e.p;
  double* yf = e.y + (size_t)f * e.p;
  for (int i = b + threadIdx.x; i < en; i += blockDim.x) {
    const double vi = vf[i] / vn;
    vf[i] = vi;
    Vcol[i] = vi;
    for (int j = 0; j < e.m; ++j) Sf[i + (size_t)j * e.p] -= vi * vs[j];
    const double ri = rf[i] / tn;
    Rcol[i] = ri;
    if (next) {
      const double y0 = e.m1_mode ? Sf[i] : ri;
      yf[i] = y0;
      ysh[i - b] = y0;
    }
  }
  if (chunk == 0) {
    double* Qcol = e.Q + ((size_t)f * e.K + a) * e.m;
    for (int j = threadIdx.x; j < e.m; j += blockDim.x) {
      double q = sum_parts(e.qpart + (size_t)f * e.cn * e.m + j, e.cn, e.m);
      double off = 0.0;
      if (e.labels) off += e.mY_all[j];
      if (e.dY) off += e.dY[(size_t)f * e.m + j];
      q -= off * st;
      Qcol[j] = q / tn;
    }
    if (threadIdx.x == 0) {
      e.tnorm[(size_t)f * e.K + a] = tn;
      e.ncomp_done[f] = a + 1;
    }
  }
  if (next) {
    __syncthreads();
    chunk_StY(e, f, chunk, Sf, ysh, b, en, e.zA, e.iters == 0);
  }
}

__global__ void k_masked_response(Eng e, double* M) {
  const size_t total = (size_t)e.n * e.F * e.m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % e.n);
    const size_t col = t / e.n;
    const int f = static_cast<int>(col / e.m), j = static_cast<int>(col % e.m);
    const bool in = !e.mask || e.mask[(size_t)f * e.n + i];
    double v = 0.0;
    if (in) v = e.labels ? (e.labels[i] == j ? 1.0 : 0.0) : e.Yg[i + (size_t)j * e.n];
    M[t] = v;
  }
}

__global__ void k_crosscov_finish(Eng e, const double* P) {
  const size_t total = (size_t)e.F * e.p * e.m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % e.p);
    const size_t col = t / e.p;
    const int f = static_cast<int>(col / e.m), j = static_cast<int>(col % e.m);
    double v = P[i + col * e.p];
    if (e.colsum) {
      double off = 0.0;
      if (e.labels) off += e.mY_all[j];
      if (e.dY) off += e.dY[(size_t)f * e.m + j];
      v -= e.colsum[(size_t)f * e.p + i] * off;
    }
    if (e.colscale) v *= e.colscale[(size_t)f * e.p + i];
    e.S[(size_t)f * e.p * e.m + i + (size_t)j * e.p] = v;
  }
}

// Row-sharded fits: after X^T T, the loading P (p x F), the score sums
// (t^T t, sum t: F x 2) and Y^T t (F x m) are rank-local partial sums.  Pack
// folds the row-chunk partials in chunk order into one buffer [P | t | q];
// after the all-reduce, unpack puts the totals in chunk 0 (the other chunks
// zero), so the kernels that follow read sums over all ranks' rows.
__global__ void k_shard_pack(Eng e, double* __restrict__ red) {
  const size_t np = (size_t)e.F * e.p, nt = (size_t)e.F * 2, nq = (size_t)e.F * e.m;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np + nt + nq;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < np) {
      red[i] = e.P[i];
    } else if (i < np + nt) {
      const size_t k = i - np, f = k / 2, c2 = k % 2;
      double s = 0.0;
      for (int c = 0; c < e.cn; ++c) s += e.tpart[(f * e.cn + c) * 2 + c2];
      red[i] = s;
    } else {
      const size_t k = i - np - nt, f = k / e.m, j = k % e.m;
      double s = 0.0;
      for (int c = 0; c < e.cn; ++c) s += e.qpart[(f * e.cn + c) * e.m + j];
      red[i] = s;
    }
  }
}

__global__ void k_shard_unpack(Eng e, const double* __restrict__ red) {
  const size_t np = (size_t)e.F * e.p, nt = (size_t)e.F * e.cn * 2, nq = (size_t)e.F * e.cn * e.m;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np + nt + nq;
       i += (size_t)gridDim.x * blockDim.x) {
    if (i < np) {
      e.P[i] = red[i];
    } else if (i < np + nt) {
      const size_t k = i - np, f = k / (2 * (size_t)e.cn), c = (k / 2) % e.cn, c2 = k % 2;
      e.tpart[k] = c == 0 ? red[np + f * 2 + c2] : 0.0;
    } else {
      const size_t k = i - np - nt, f = k / ((size_t)e.cn * e.m), c = (k / e.m) % e.cn, j = k % e.m;
      e.qpart[k] = c == 0 ? red[np + (size_t)e.F * 2 + f * e.m + j] : 0.0;
    }
  }
}

Eng make_eng(const SimplsBatch& b) {
  Eng e{};
  e.n = b.n; e.p = b.p; e.m = b.m; e.F = b.F; e.K = b.K;
  const int target = 4 * Context::get().sm_count;
  e.cp = std::max(1, std::min(ceil_div(target, b.F), ceil_div(b.p, 256)));
  e.cp = std::max(e.cp, ceil_div(b.p, kMaxChunk));
  e.szp = ceil_div(b.p, e.cp);
  e.cp = ceil_div(b.p, e.szp);
  e.cn = std::max(1, std::min(ceil_div(target, b.F), ceil_div(b.n, 256)));
  e.cn = std::max(e.cn, ceil_div(b.n, kMaxChunk));
  e.szn = ceil_div(b.n, e.cn);
  e.cn = ceil_div(b.n, e.szn);
  e.Yg = b.Yg; e.labels = b.labels; e.mY_all = b.mY_all; e.mask = b.mask; e.delta = b.delta;
  e.colsum = b.colsum;
  e.colscale = b.colscale; e.dY = b.dY; e.S = b.S; e.omega = b.omega; e.m1_mode = b.m1_mode;
  e.iters = b.m1_mode ? 0 : std::max(b.power_iters, 0);
  e.R = b.R; e.Q = b.Q; e.V = b.V; e.tnorm = b.tnorm; e.Tkeep = b.Tkeep;
  e.ncomp_done = b.ncomp_done; e.status = b.status;
  return e;
}

}  // namespace

void XOperatorF64::times(const double* Rhat, int F, double* U) {
  if (F == 1) gemv(false, n, p, 1.0, Xc, n, Rhat, 0.0, U);
  else gemm(false, false, n, F, p, 1.0, Xc, n, Rhat, p, 0.0, U, n);
}

void XOperatorF64::t_times(const double* T, int F, double* P) {
  if (F == 1) gemv(true, n, p, 1.0, Xc, n, T, 0.0, P);
  else gemm(true, false, p, F, n, 1.0, Xc, n, T, n, 0.0, P, p);
}

void XOperatorF64::gram(double* K) { gram_f64(Xc, n, p, n, K, n); }

void simpls_batch_crosscov(const SimplsBatch& b, const double* /*Xc*/, const int* /*n_train*/) {
  Context& ctx = Context::get();
  Eng e = make_eng(b);
  double* M = ctx.arena.alloc_n<double>((size_t)b.n * b.F * b.m);
  double* P = ctx.arena.alloc_n<double>((size_t)b.p * b.F * b.m);
  k_masked_response<<<2 * ctx.sm_count, kThreads, 0, ctx.stream>>>(e, M); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  b.X->t_times(M, b.F * b.m, P);
  k_crosscov_finish<<<2 * ctx.sm_count, kThreads, 0, ctx.stream>>>(e, P); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

namespace {

// FASTPLS_LOOP_GRAPH=0 enqueues the component loop launch by launch.
bool simpls_graph_enabled() {
  static const int v = [] {
    const char* e = std::getenv("FASTPLS_LOOP_GRAPH");
    return e ? (e[0] != '0' ? 1 : 0) : 1;
  }();
  return v != 0;
}

// Shapes whose component loop has run once launch by launch: its GEMM plans,
// split-K workspace and arena blocks exist, so a later call of the shape enqueues
// launches only and can be captured.
std::set<std::array<long long, 9>>& simpls_seen() {
  static std::set<std::array<long long, 9>> seen;
  return seen;
}

// The executable graph of the last captured component loop; each call captures
// its loop and updates it in place when the topology matches, else
// instantiates a new one (launches already in flight are not affected).
cudaGraphExec_t g_simpls_exec = nullptr;

// Returns false, with nothing enqueued, when the loop could not be captured
// (a host step of the loop that a capture does not allow, such as the first
// allocation of a GEMM plan); the caller then runs the loop launch by launch.
template <typename Loop>
bool simpls_launch_as_graph(cudaStream_t st, Loop&& loop) {
  FPLS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaGraph_t graph = nullptr;
  try {
    loop();
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return false;
  }
  if (cudaStreamEndCapture(st, &graph) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return false;
  }
  bool updated = false;
  if (g_simpls_exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(g_simpls_exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(g_simpls_exec);
      g_simpls_exec = nullptr;
    }
  }
  cudaError_t e = cudaSuccess;
  if (!updated) e = cudaGraphInstantiate(&g_simpls_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    g_simpls_exec = nullptr;
    FPLS_CUDA(e);
  }
  FPLS_CUDA(cudaGraphLaunch(g_simpls_exec, st));
  return true;
}

}  // namespace

void simpls_release_graph() {
  if (g_simpls_exec) cudaGraphExecDestroy(g_simpls_exec);
  g_simpls_exec = nullptr;
  simpls_seen().clear();
}

void simpls_batch_run(const SimplsBatch& b) {
  Context& ctx = Context::get();
  Eng e = make_eng(b);
  Arena& ar = ctx.arena;
  const size_t F = b.F;
  e.y = ar.alloc_n<double>(F * b.p);
  e.zA = ar.alloc_n<double>(F * e.cp * b.m);
  e.zB = ar.alloc_n<double>(F * e.cp * b.m);
  e.npart = ar.alloc_n<double>(F * e.cp);
  e.r = ar.alloc_n<double>(F * b.p);
  e.Rhat = ar.alloc_n<double>(F * b.p);
  e.cpart = ar.alloc_n<double>(F * e.cp);
  e.U = ar.alloc_n<double>(F * b.n);
  e.T = ar.alloc_n<double>(F * b.n);
  e.tpart = ar.alloc_n<double>(F * e.cn * 2);
  e.qpart = ar.alloc_n<double>(F * e.cn * b.m);
  e.P = ar.alloc_n<double>(F * b.p);
  e.pv = ar.alloc_n<double>(F * b.p);
  e.wpart = ar.alloc_n<double>(F * e.cp * std::max(b.K, 1));
  e.v = ar.alloc_n<double>(F * b.p);
  e.vpart = ar.alloc_n<double>(F * e.cp);
  e.vSpart = ar.alloc_n<double>(F * e.cp * b.m);
  dzero(b.status, F * sizeof(int));
  dzero(b.ncomp_done, F * sizeof(int));
  dzero(b.R, F * b.p * b.K * sizeof(double));
  dzero(b.Q, F * b.m * b.K * sizeof(double));
  dzero(b.V, F * b.p * b.K * sizeof(double));
  dzero(b.tnorm, F * b.K * sizeof(double));
  const dim3 gp(e.cp, b.F), gn(e.cn, b.F);
  // all-reduce buffer of a row-sharded fit: [P (F x p) | t^T t, sum t (F x 2) | Y^T t (F x m)]
  const size_t shard_count = sharded() ? F * ((size_t)b.p + 2 + b.m) : 0;
  double* shard_red = shard_count ? ar.alloc_n<double>(shard_count) : nullptr;
  const unsigned shard_grid =
      shard_count ? (unsigned)std::min<size_t>(ceil_div(F * ((size_t)b.p + e.cn * (2 + (size_t)b.m)), kThreads),
                                               (size_t)ctx.sm_count * 8)
                  : 1u;
  const size_t sm_m = std::max<size_t>(b.m, 1) * sizeof(double);
  const size_t sm_k = std::max<size_t>(b.K, 1) * sizeof(double);
  cudaStream_t st = ctx.stream;
  // Optional per-phase device timing (FASTPLS_TRACE=1), printed to stderr.
  const char* trace_env = std::getenv("FASTPLS_TRACE");
  const bool trace = trace_env && trace_env[0] == '1';
  std::vector<std::pair<const char*, cudaEvent_t>> marks;
  auto mark = [&](const char* name) {
    if (!trace) return;
    cudaEvent_t ev;
    FPLS_CUDA(cudaEventCreate(&ev));
    FPLS_CUDA(cudaEventRecord(ev, st));
    marks.emplace_back(name, ev);
  };
  mark("start");
  // The component loop as one CUDA graph once its shape has run (not while a
  // trace or the kernel-class profiler records events, nor for row-sharded
  // fits, whose all-reduce callback is the caller's).
  const std::array<long long, 9> key{b.F, b.n, b.p, b.m, b.K, e.iters, b.labels ? 1 : 0, ctx.precision,
                                     static_cast<long long>(typeid(*b.X).hash_code())};
  const bool eligible = simpls_graph_enabled() && !trace && !ctx.profile && !shard_red;
  const bool graph = eligible && simpls_seen().count(key) > 0;
  auto loop = [&]() {
  k_refresh_start<<<gp, kThreads, 0, st>>>(e); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  for (int a = 0; a < b.K; ++a) {
    // Refresh: y <- S (S^T y) `iters` times from the warm start, then normalise.
    double* zin = e.zA;
    double* zout = e.zB;
    for (int it = 0; it < e.iters; ++it) {
      const int last = (it == e.iters - 1) ? 1 : 0;
      k_refresh_apply<<<gp, kThreads, sm_m, st>>>(e, zin, zout, last); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      std::swap(zin, zout);
    }
    k_refresh_finish<<<gp, kThreads, 0, st>>>(e); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    mark("refresh");
    b.X->times(e.Rhat, b.F, e.U);
    mark("X*R");
    k_scores<<<gn, kThreads, b.labels ? sm_m : 0, st>>>(e, a); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    mark("scores");
    b.X->t_times(e.T, b.F, e.P);
    if (shard_red) {
      k_shard_pack<<<shard_grid, kThreads, 0, st>>>(e, shard_red); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      shard_sum(shard_red, shard_count);
      k_shard_unpack<<<shard_grid, kThreads, 0, st>>>(e, shard_red); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
    mark("X^T*T");
    k_loading<<<gp, kThreads, 0, st>>>(e, a); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    mark("loading");
    k_orth<<<gp, kThreads, sm_k, st>>>(e, a); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    mark("orth");
    k_deflate<<<gp, kThreads, sm_m, st>>>(e, a, a + 1 < b.K ? 1 : 0); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    mark("deflate");
  }
  };
  if (!(graph && simpls_launch_as_graph(st, loop))) {
    loop();
    if (eligible) simpls_seen().insert(key);
  }
  if (trace) {
    FPLS_CUDA(cudaStreamSynchronize(st));
    std::map<std::string, double> acc;
    for (size_t k = 1; k < marks.size(); ++k) {
      float ms = 0.f;
      FPLS_CUDA(cudaEventElapsedTime(&ms, marks[k - 1].second, marks[k].second));
      acc[marks[k].first] += ms;
    }
    double total = 0.0;
    for (auto& kv : acc) total += kv.second;
    std::fprintf(stderr, "[fastpls trace] SIMPLS engine F=%d n=%d p=%d m=%d K=%d: %.3f ms\n", b.F, b.n,
                 b.p, b.m, b.K, total);
    for (auto& kv : acc) std::fprintf(stderr, "  %-10s %8.3f ms\n", kv.first.c_str(), kv.second);
    for (auto& mk : marks) cudaEventDestroy(mk.second);
  }
}

}  // namespace fpls
