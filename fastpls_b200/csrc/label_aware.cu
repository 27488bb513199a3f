// Label-aware PLSSVD on the device: the class-sum cross-covariance
// S = sum_c e_c (x) sum_{i in c} x~_i - (sum_i x~_i) mY^T (mY = counts / n) built
// by a segmented reduction over class-sorted rows (no dense one-hot response),
// its SVD, the latent Gram G = (X~R)^T(X~R) and the per-ncomp coefficients
// C_k = (G_k + 1e-10 mean(diag G_k) I)^{-1} diag(d_k), W_k = C_k Q_k^T.
// Reference: .plssvd_label_aware_stream_model (R/main.R:513-655).
//
// Layout: the centred (scaled) predictor block is kept once, row-major
// (p x n column-major, FP64), so a class-sorted walk over rows reads whole
// contiguous rows, and X~R is a transposed-A GEMM over the same copy.
#include "../../include/fastpls_b200.h"

#include <algorithm>
#include <cmath>
#include <vector>

#include "xop_split.cuh"
#include "blas_f64.cuh"
#include "capi_util.cuh"
#include "cknn.cuh"
#include "context.cuh"
#include "label_aware.cuh"
#include "linalg_small.cuh"
#include "svd.cuh"

namespace fpls {
namespace {

// Column sums (and sums of squares) of the raw predictors, one CTA per column
// (R/main.R:542-551).
template <typename T>
__global__ void col_sums_kernel(const T* __restrict__ X, int n, int p, double* __restrict__ sums,
                                double* __restrict__ sumsq) {
  __shared__ double scratch[32];
  const int j = blockIdx.x;
  const T* col = X + (size_t)j * n;
  double s = 0.0, q = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = static_cast<double>(col[i]);
    s += v;
    q += v * v;
  }
  s = block_sum(s, scratch);
  q = block_sum(q, scratch);
  if (threadIdx.x == 0) {
    sums[j] = s;
    sumsq[j] = q;
  }
}

// mX = sums / n (scaling < 3, else 0); vX = sqrt(max(sumsq - n mX^2, 0) / max(1, n - 1))
// for scaling 2 with zero / non-finite -> 1 (R/main.R:552-558).
__global__ void la_stats_kernel(const double* sums, const double* sumsq, int n, int p, int scaling,
                                double* mX, double* vX) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    const double m = scaling < 3 ? sums[j] / n : 0.0;
    mX[j] = m;
    double v = 1.0;
    if (scaling == 2) {
      const double css = fmax(sumsq[j] - n * m * m, 0.0);
      v = sqrt(css / (double)max(1, n - 1));
      if (!isfinite(v) || v == 0.0) v = 1.0;
    }
    vX[j] = v;
  }
}

// Xt[j + i * p] = (X[i + j * n] - mX[j]) / vX[j]  (column-major n x p -> row-major),
// 32 x 32 tiles through shared memory.
template <typename T>
__global__ void transpose_center_kernel(const T* __restrict__ X, int n, int p, const double* __restrict__ mX,
                                        const double* __restrict__ vX, int scaling, double* __restrict__ Xt) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (i < n && j < p) {
      double v = static_cast<double>(X[i + (size_t)j * n]);
      if (scaling < 3) v -= mX[j];
      if (scaling == 2) v /= vX[j];
      tile[r][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (i < n && j < p) Xt[j + (size_t)i * p] = tile[threadIdx.x][r];
  }
}

__global__ void la_sort_kernel(const int* __restrict__ y, int n, const int* __restrict__ offs, int* cursor,
                               int* __restrict__ perm, int* __restrict__ ysorted) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = y[i] - 1;
    const int d = offs[c] + atomicAdd(cursor + c, 1);
    perm[d] = i;
    ysorted[d] = c;
  }
}

// Class sums over class-sorted rows: each CTA walks `rows` sorted rows (their
// row indices and classes staged in shared memory), each thread owns up to
// kColsPerThread columns and keeps running sums in registers, flushing them
// (atomicAdd into cs, p x m column-major) when the class changes and at the
// end of its range.  Loads of kRowBatch rows are issued before they are
// accumulated, so each thread keeps 32 loads in flight.
constexpr int kColsPerThread = 4;
constexpr int kRowBatch = 8;
__global__ void __launch_bounds__(256) class_sum_kernel(const double* __restrict__ Xt, int p, int n,
                                                        const int* __restrict__ perm,
                                                        const int* __restrict__ ysorted, int col0,
                                                        int rows, double* __restrict__ cs) {
  extern __shared__ int sidx[];  // [rows] row index, [rows] class
  const int s0 = blockIdx.x * rows;
  const int nr = min(n, s0 + rows) - s0;
  for (int t = threadIdx.x; t < nr; t += blockDim.x) {
    sidx[t] = perm[s0 + t];
    sidx[rows + t] = ysorted[s0 + t];
  }
  __syncthreads();
  int jcol[kColsPerThread];
  double acc[kColsPerThread];
#pragma unroll
  for (int u = 0; u < kColsPerThread; ++u) {
    jcol[u] = col0 + threadIdx.x + u * blockDim.x;
    acc[u] = 0.0;
  }
  int cur = sidx[rows];
  for (int base = 0; base < nr; base += kRowBatch) {
    double v[kRowBatch][kColsPerThread];
#pragma unroll
    for (int g = 0; g < kRowBatch; ++g) {
      const int r = base + g;
      const double* row = Xt + (size_t)(r < nr ? sidx[r] : 0) * p;
#pragma unroll
      for (int u = 0; u < kColsPerThread; ++u)
        v[g][u] = (r < nr && jcol[u] < p) ? __ldg(row + jcol[u]) : 0.0;
    }
#pragma unroll
    for (int g = 0; g < kRowBatch; ++g) {
      const int r = base + g;
      if (r >= nr) break;
      const int c = sidx[rows + r];
      if (c != cur) {
#pragma unroll
        for (int u = 0; u < kColsPerThread; ++u) {
          if (jcol[u] < p) atomicAdd(cs + jcol[u] + (size_t)cur * p, acc[u]);
          acc[u] = 0.0;
        }
        cur = c;
      }
#pragma unroll
      for (int u = 0; u < kColsPerThread; ++u) acc[u] += v[g][u];
    }
  }
#pragma unroll
  for (int u = 0; u < kColsPerThread; ++u)
    if (jcol[u] < p) atomicAdd(cs + jcol[u] + (size_t)cur * p, acc[u]);
}

// S = cs - total mY^T with total_j = sum_c cs[j, c] (class order) and
// mY = counts / n (R/main.R:560-592).
__global__ void la_crosscov_kernel(double* cs, int p, int m, const int* counts, int n, double* mY) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int c = 0; c < m; ++c) t += cs[j + (size_t)c * p];
    for (int c = 0; c < m; ++c) cs[j + (size_t)c * p] -= t * ((double)counts[c] / n);
  }
  if (blockIdx.x == 0)
    for (int c = threadIdx.x; c < m; c += blockDim.x) mY[c] = (double)counts[c] / n;
}

// out (n x p, column-major FP64) = (X - mX) / vX as the model's scaling.
template <typename T>
__global__ void center_to_f64_kernel(const T* __restrict__ X, int n, int p, const double* __restrict__ mX,
                                     const double* __restrict__ vX, int scaling, double* __restrict__ out) {
  const size_t total = (size_t)n * p;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int j = static_cast<int>(t / n);
    double v = static_cast<double>(X[t]);
    if (scaling < 3) v -= mX[j];
    if (scaling == 2) v /= vX[j];
    out[t] = v;
  }
}

__global__ void diag_rhs_kernel(const double* d, int k, double* D) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < k * k; t += gridDim.x * blockDim.x)
    D[t] = (t % k == t / k) ? d[t % k] : 0.0;
}

}  // namespace

std::vector<int> cap_plssvd_ncomp(const int* ncomp, int L, int n, int p, int m, int* max_rank) {
  const int mr = std::min(n, std::min(p, m));
  FPLS_REQUIRE(mr >= 1, "plssvd rank is < 1");
  std::vector<int> out(L);
  for (int a = 0; a < L; ++a) out[a] = std::min(std::max(ncomp[a], 1), mr);
  if (max_rank) *max_rank = mr;
  return out;
}

LabelAwareFit label_aware_fit(const void* dX, bool f32, int n, int p, const int* dy, const int* y_host,
                              int m, const std::vector<int>& ncomp, int scaling, int svd_method,
                              int oversample, int power_iters, unsigned int seed) {
  Context& ctx = Context::get();
  FPLS_REQUIRE(n >= 1 && p >= 1 && m >= 2,
               "label-aware PLSSVD requires non-empty X and at least two classes");
  PhaseTimer pt("label-aware PLSSVD");
  LabelAwareFit f;
  f.n = n;
  f.p = p;
  f.m = m;
  f.ncomp = ncomp;
  f.K = *std::max_element(ncomp.begin(), ncomp.end());
  const int K = f.K;
  const int L = static_cast<int>(ncomp.size());

  // predictor statistics and the centred row-major copy
  double* sums = ctx.arena.alloc_n<double>(p);
  double* sumsq = ctx.arena.alloc_n<double>(p);
  f.mX = ctx.arena.alloc_n<double>(p);
  f.vX = ctx.arena.alloc_n<double>(p);
  if (f32) col_sums_kernel<float><<<p, 256, 0, ctx.stream>>>(static_cast<const float*>(dX), n, p, sums, sumsq);
  else col_sums_kernel<double><<<p, 256, 0, ctx.stream>>>(static_cast<const double*>(dX), n, p, sums, sumsq);
  ::fpls::note_launch();
  la_stats_kernel<<<ceil_div(p, 256), 256, 0, ctx.stream>>>(sums, sumsq, n, p, scaling, f.mX, f.vX); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  f.Xt = ctx.arena.alloc_n<double>((size_t)n * p);
  {
    dim3 grid(ceil_div(n, 32), ceil_div(p, 32));
    if (f32)
      transpose_center_kernel<float><<<grid, dim3(32, 8), 0, ctx.stream>>>(static_cast<const float*>(dX), n, p,
                                                                          f.mX, f.vX, scaling, f.Xt);
    else
      transpose_center_kernel<double><<<grid, dim3(32, 8), 0, ctx.stream>>>(static_cast<const double*>(dX), n, p,
                                                                           f.mX, f.vX, scaling, f.Xt);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  pt.mark("stats + centred copy");

  // class-sorted row order (counting sort of the labels)
  std::vector<int> counts_h(m, 0);
  for (int i = 0; i < n; ++i) counts_h[y_host[i] - 1]++;
  std::vector<int> offs(m + 1, 0);
  for (int c = 0; c < m; ++c) offs[c + 1] = offs[c] + counts_h[c];
  int* counts = ctx.arena.alloc_n<int>(m);
  int* d_offs = ctx.arena.alloc_n<int>(m + 1);
  int* cursor = ctx.arena.alloc_n<int>(m);
  int* perm = ctx.arena.alloc_n<int>(n);
  int* ysorted = ctx.arena.alloc_n<int>(n);
  h2d(counts, counts_h.data(), m * sizeof(int));
  h2d(d_offs, offs.data(), (m + 1) * sizeof(int));
  FPLS_CUDA(cudaMemsetAsync(cursor, 0, m * sizeof(int), ctx.stream));
  const int g = std::max(1, std::min(ceil_div(n, 256), 8 * ctx.sm_count));
  la_sort_kernel<<<g, 256, 0, ctx.stream>>>(dy, n, d_offs, cursor, perm, ysorted); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  pt.mark("class sort");

  // class sums -> S (p x m)
  f.S = ctx.arena.alloc_n<double>((size_t)p * m);
  fill(f.S, (size_t)p * m, 0.0);
  const int rows = std::min(4096, std::max(256, ceil_div(ceil_div(n, 4 * ctx.sm_count), 8) * 8));
  for (int col0 = 0; col0 < p; col0 += 256 * kColsPerThread) {
    class_sum_kernel<<<ceil_div(n, rows), 256, 2 * rows * sizeof(int), ctx.stream>>>(f.Xt, p, n, perm, ysorted,
                                                                                    col0, rows, f.S); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  f.mY = ctx.arena.alloc_n<double>(m);
  la_crosscov_kernel<<<ceil_div(p, 128), 128, 0, ctx.stream>>>(f.S, p, m, counts, n, f.mY); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  pt.mark("class sums");

  // SVD of S: R = U[:, :K], Q = V[:, :K], d
  f.R = ctx.arena.alloc_n<double>((size_t)p * K);
  f.Q = ctx.arena.alloc_n<double>((size_t)m * K);
  f.d = ctx.arena.alloc_n<double>(K);
  fill(f.R, (size_t)p * K, 0.0);
  fill(f.Q, (size_t)m * K, 0.0);
  fill(f.d, K, 0.0);
  const bool exact = svd_method == kSvdExact;
  SvdResult sr = truncated_svd_device(f.S, p, m, p, K, exact ? kSvdExact : svd_method, oversample,
                                      power_iters, seed, false, exact, f.R, p, f.d, f.Q, m);
  f.rank = sr.rank;
  pt.mark("svd");

  // T = X~ R (n x K), G = T^T T
  f.T = ctx.arena.alloc_n<double>((size_t)n * K);
  xgemm(true, n, K, p, f.Xt, p, f.R, p, f.T, n);
  f.G = ctx.arena.alloc_n<double>((size_t)K * K);
  gemm(true, false, K, K, n, 1.0, f.T, n, f.T, n, 0.0, f.G, K);
  pt.mark("scores + gram");

  // per-ncomp coefficients
  f.C = ctx.arena.alloc_n<double>((size_t)K * K * L);
  f.W = ctx.arena.alloc_n<double>((size_t)K * m * L);
  fill(f.C, (size_t)K * K * L, 0.0);
  fill(f.W, (size_t)K * m * L, 0.0);
  double* D = ctx.arena.alloc_n<double>((size_t)K * K);
  int* flag = ctx.d_status + 9;
  FPLS_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), ctx.stream));
  for (int a = 0; a < L; ++a) {
    const int k = ncomp[a];
    diag_rhs_kernel<<<ceil_div(k * k, 256), 256, 0, ctx.stream>>>(f.d, k, D); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    double* Ca = f.C + (size_t)a * K * K;
    spd_solve(k, f.G, K, k, D, k, Ca, K, flag, 1e-10);
    gemm(false, true, k, m, k, 1.0, Ca, K, f.Q, m, 0.0, f.W + (size_t)a * K * m, K);
  }
  int bad = 0;
  d2h(&bad, flag, sizeof(int));
  ctx.sync();
  pt.mark("coefficients");
  pt.report();
  if (bad) throw Error(kErrNumerical, "label-aware PLSSVD: latent Gram system is singular");
  return f;
}


// Label-aware PLSSVD fit, candidate-kNN fit in the PLSSVD prediction-latent
// score space (T C_k, row-normalised; R/main.R:700-730, 795-873) and
// candidate-kNN prediction of the test rows (R/main.R:875-950), all on
// device buffers.  d_ti / d_ts: ntest x max(1, min(top_k, m)).
void label_aware_cknn_device(const void* dX, const void* dXtest, bool f32, int n, int ntest, int p,
                             const int* dy, const int* y_host, int m, int ncomp, int scaling, int svd_method,
                             int oversample, int power_iters, unsigned int seed, int knn_k, double tau,
                             double alpha, int top_m, int top_k, int* d_ti, double* d_ts,
                             capi::SideUpload* xtest_copy) {
  Context& ctx = Context::get();
  const std::vector<int> nc = cap_plssvd_ncomp(&ncomp, 1, n, p, m, nullptr);
  LabelAwareFit f = label_aware_fit(dX, f32, n, p, dy, y_host, m, nc, scaling, svd_method, oversample,
                                    power_iters, seed);
  PhaseTimer pt("candidate-kNN on label-aware scores");
  const int K = f.K;
  double* Tn = ctx.arena.alloc_n<double>((size_t)n * K);
  candidate_scores_device(f.T, n, K, f.C, Tn);
  double* cent = ctx.arena.alloc_n<double>((size_t)m * K);
  candidate_centroids_device(Tn, n, K, dy, m, cent);
  pt.mark("train scores + centroids");
  double* Xc = ctx.arena.alloc_n<double>((size_t)ntest * p);
  if (xtest_copy) xtest_copy->wait();
  const int g = std::max(1, std::min(ceil_div((long long)ntest * p, 256), 8 * ctx.sm_count));
  if (f32)
    center_to_f64_kernel<float><<<g, 256, 0, ctx.stream>>>(static_cast<const float*>(dXtest), ntest, p, f.mX,
                                                          f.vX, scaling, Xc);
  else
    center_to_f64_kernel<double><<<g, 256, 0, ctx.stream>>>(static_cast<const double*>(dXtest), ntest, p, f.mX,
                                                           f.vX, scaling, Xc);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  double* Tt = ctx.arena.alloc_n<double>((size_t)ntest * K);
  gemm(false, false, ntest, K, p, 1.0, Xc, ntest, f.R, p, 0.0, Tt, ntest);
  double* Ttn = ctx.arena.alloc_n<double>((size_t)ntest * K);
  candidate_scores_device(Tt, ntest, K, f.C, Ttn);
  pt.mark("test scores");
  candidate_knn_predict_device(Ttn, ntest, Tn, n, K, dy, cent, m, nullptr, top_k, top_m, knn_k, tau, alpha,
                               d_ti, d_ts);
  pt.mark("candidate-kNN predict");
  pt.report();
}

}  // namespace fpls

using namespace fpls;
using capi::upload;

extern "C" {

int fpls_plssvd_label_aware(const void* X, int x_is_float32, int n, int p, const int* y_codes, int m,
                            const int* ncomp, int L, int scaling, int svd_method, int oversample,
                            int power_iters, int seed, int* ncomp_out, double* C_latent,
                            double* W_latent, double* Q, double* R, double* mX, double* vX,
                            double* mY, double* s, double* Ttrain, int* max_rank, char* err,
                            size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(X && y_codes && ncomp && L >= 1, "label-aware PLSSVD: missing inputs");
    FPLS_REQUIRE(n >= 1 && p >= 1 && m >= 2,
                 "label-aware PLSSVD requires non-empty X and at least two classes");
    FPLS_REQUIRE(scaling >= 1 && scaling <= 3, "scaling must be 1, 2 or 3");
    FPLS_REQUIRE(svd_method == kSvdExact || svd_method == kSvdCpuRsvd || svd_method == kSvdCudaRsvd,
                 "label-aware PLSSVD: svd_method must be exact (3) or rsvd (4 / 5)");
    for (int i = 0; i < n; ++i)
      FPLS_REQUIRE(y_codes[i] >= 1 && y_codes[i] <= m, "label-aware PLSSVD: class code outside 1..m");
    Context& ctx = Context::get();
    ctx.begin_call();
    std::vector<int> nc = cap_plssvd_ncomp(ncomp, L, n, p, m, nullptr);
    const size_t xbytes = (size_t)n * p * (x_is_float32 ? sizeof(float) : sizeof(double));
    void* dX = ctx.arena.alloc_n<char>(xbytes);
    h2d(dX, X, xbytes);
    const int* dy = upload(y_codes, n);
    LabelAwareFit f = label_aware_fit(dX, x_is_float32 != 0, n, p, dy, y_codes, m, nc, scaling,
                                      svd_method, oversample, power_iters,
                                      static_cast<unsigned int>(seed));
    const int K = f.K;
    for (int a = 0; a < L; ++a) ncomp_out[a] = nc[a];
    if (max_rank) *max_rank = K;
    d2h(C_latent, f.C, (size_t)K * K * L * sizeof(double));
    d2h(W_latent, f.W, (size_t)K * m * L * sizeof(double));
    d2h(Q, f.Q, (size_t)m * K * sizeof(double));
    d2h(R, f.R, (size_t)p * K * sizeof(double));
    d2h(mX, f.mX, p * sizeof(double));
    d2h(vX, f.vX, p * sizeof(double));
    d2h(mY, f.mY, m * sizeof(double));
    if (s) d2h(s, f.d, K * sizeof(double));
    if (Ttrain) d2h(Ttrain, f.T, (size_t)n * K * sizeof(double));
    ctx.sync();
  });
}

int fpls_label_aware_cknn(const void* Xtrain, int x_is_float32, int n, int p, const int* y_codes, int m,
                          const void* Xtest, int ntest, int ncomp, int scaling, int svd_method,
                          int oversample, int power_iters, int seed, int knn_k, double tau,
                          double alpha, int top_m, int top_k, int* top_index, double* top_score,
                          char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(Xtrain && Xtest && y_codes && top_index && top_score, "label-aware cKNN: missing inputs");
    FPLS_REQUIRE(n >= 1 && p >= 1 && m >= 2 && ntest >= 1,
                 "label-aware PLSSVD requires non-empty X and at least two classes");
    FPLS_REQUIRE(scaling >= 1 && scaling <= 3, "scaling must be 1, 2 or 3");
    FPLS_REQUIRE(svd_method == kSvdExact || svd_method == kSvdCpuRsvd || svd_method == kSvdCudaRsvd,
                 "label-aware PLSSVD: svd_method must be exact (3) or rsvd (4 / 5)");
    FPLS_REQUIRE(std::isfinite(tau) && tau > 0.0, "candidate_tau must be positive");
    FPLS_REQUIRE(std::isfinite(alpha), "candidate_alpha must be finite");
    for (int i = 0; i < n; ++i)
      FPLS_REQUIRE(y_codes[i] >= 1 && y_codes[i] <= m, "label-aware PLSSVD: class code outside 1..m");
    Context& ctx = Context::get();
    ctx.begin_call();
    const size_t es = x_is_float32 ? sizeof(float) : sizeof(double);
    void* dX = ctx.arena.alloc_n<char>((size_t)n * p * es);
    h2d(dX, Xtrain, (size_t)n * p * es);
    const int* dy = upload(y_codes, n);
    // the test rows cross the link while the fit runs
    capi::SideUpload xt(Xtest, (size_t)ntest * p * es);
    const int tk = std::max(1, std::min(top_k, m));
    int* d_ti = ctx.arena.alloc_n<int>((size_t)ntest * tk);
    double* d_ts = ctx.arena.alloc_n<double>((size_t)ntest * tk);
    label_aware_cknn_device(dX, xt.dst, x_is_float32 != 0, n, ntest, p, dy, y_codes, m, ncomp, scaling,
                            svd_method, oversample, power_iters, static_cast<unsigned int>(seed), knn_k,
                            tau, alpha, top_m, top_k, d_ti, d_ts, &xt);
    d2h(top_index, d_ti, (size_t)ntest * tk * sizeof(int));
    d2h(top_score, d_ts, (size_t)ntest * tk * sizeof(double));
    ctx.sync();
  });
}

int fpls_label_aware_cknn_resident(int xtrain_handle, const int* y_codes, int m, int xtest_handle,
                                   int ncomp, int scaling, int svd_method, int oversample,
                                   int power_iters, int seed, int knn_k, double tau, double alpha,
                                   int top_m, int top_k, int* top_index, double* top_score, char* err,
                                   size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    const int nres = static_cast<int>(ctx.resident.size());
    FPLS_REQUIRE(xtrain_handle >= 0 && xtrain_handle < nres && ctx.resident[xtrain_handle].ptr,
                 "label-aware cKNN: unknown training handle");
    FPLS_REQUIRE(xtest_handle >= 0 && xtest_handle < nres && ctx.resident[xtest_handle].ptr,
                 "label-aware cKNN: unknown test handle");
    const ResidentX tr = ctx.resident[xtrain_handle];
    const ResidentX te = ctx.resident[xtest_handle];
    FPLS_REQUIRE(tr.p == te.p && tr.f32 == te.f32, "label-aware cKNN: train / test matrices differ in p or type");
    FPLS_REQUIRE(m >= 2, "label-aware PLSSVD requires non-empty X and at least two classes");
    FPLS_REQUIRE(scaling >= 1 && scaling <= 3, "scaling must be 1, 2 or 3");
    FPLS_REQUIRE(svd_method == kSvdExact || svd_method == kSvdCpuRsvd || svd_method == kSvdCudaRsvd,
                 "label-aware PLSSVD: svd_method must be exact (3) or rsvd (4 / 5)");
    FPLS_REQUIRE(std::isfinite(tau) && tau > 0.0, "candidate_tau must be positive");
    FPLS_REQUIRE(std::isfinite(alpha), "candidate_alpha must be finite");
    for (int i = 0; i < tr.n; ++i)
      FPLS_REQUIRE(y_codes[i] >= 1 && y_codes[i] <= m, "label-aware PLSSVD: class code outside 1..m");
    ctx.begin_call();
    const int* dy = upload(y_codes, tr.n);
    const int tk = std::max(1, std::min(top_k, m));
    int* d_ti = ctx.arena.alloc_n<int>((size_t)te.n * tk);
    double* d_ts = ctx.arena.alloc_n<double>((size_t)te.n * tk);
    label_aware_cknn_device(tr.ptr, te.ptr, tr.f32, tr.n, te.n, tr.p, dy, y_codes, m, ncomp, scaling,
                            svd_method, oversample, power_iters, static_cast<unsigned int>(seed), knn_k,
                            tau, alpha, top_m, top_k, d_ti, d_ts, nullptr);
    d2h(top_index, d_ti, (size_t)te.n * tk * sizeof(int));
    d2h(top_score, d_ts, (size_t)te.n * tk * sizeof(double));
    ctx.sync();
  });
}

}  // extern "C"
