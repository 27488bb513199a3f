// extern "C" entry points of libfastpls_b200.so (declared in include/fastpls_b200.h).
#include "../../include/fastpls_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <sstream>
#include <vector>

#include "autotune.cuh"
#include "dual_engine.cuh"
#include "gaussian.cuh"
#include "blas_f64.cuh"
#include "capi_util.cuh"
#include "context.cuh"
#include "cv_driver.cuh"
#include "fits.cuh"
#include "heads.cuh"
#include "kernel_pls.cuh"
#include "ozaki_gemm.cuh"
#include "simpls_engine.cuh"
#include "svd.cuh"
#include "xop_split.cuh"
#include "xprod.cuh"

using namespace fpls;

namespace {

using capi::guarded;
using capi::upload;
using capi::download;

int max_of(const int* v, int L) {
  int m = 0;
  for (int i = 0; i < L; ++i) m = std::max(m, v[i]);
  return m;
}

__global__ void transpose_small(const double* A, int rows, int cols, double* B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * cols) return;
  const int i = t % rows, j = t / rows;
  B[j + (size_t)i * cols] = A[t];
}

__global__ void scale_column_kernel(const double* src, int n, double inv, double* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] * inv;
}

__global__ void center_copy_kernel(const double* X, int w, int p, const double* mX,
                                   const double* vX, double* out) {
  const size_t total = (size_t)w * p;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int j = static_cast<int>(t / w);
    out[t] = (X[t] - mX[j]) / vX[j];
  }
}

double* centered_test_copy(const double* Xh, int w, int p, const double* mX_d, const double* vX_d) {
  Context& ctx = Context::get();
  double* X = upload(Xh, (size_t)w * p);
  center_copy_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(X, w, p, mX_d, vX_d, X); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  return X;
}

// Block results (rb x top_k, ld rb) into the full outputs (w x top_k, ld w) at row r0.
__global__ void place_rows_kernel(const int* __restrict__ bi, const double* __restrict__ bs, int rb, int top_k, int w,
                                  int r0, int* __restrict__ di, double* __restrict__ ds) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)rb * top_k) return;
  const int i = static_cast<int>(t % rb), j = static_cast<int>(t / rb);
  di[r0 + i + (size_t)j * w] = bi[t];
  if (ds) ds[r0 + i + (size_t)j * w] = bs[t];
}

// Test rows per block of a class prediction: all of them while the scores of
// every slice, the latent scores and the centred rows fit in 1 GiB, else
// blocks that do (at least 128 rows); FASTPLS_PREDICT_BLOCK_ROWS sets it.
int predict_block_rows(int w, int p, int kmax, int m, int L) {
  if (const char* e = std::getenv("FASTPLS_PREDICT_BLOCK_ROWS")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v >= 1) return static_cast<int>(std::min<long>(v, w));
  }
  const double per_row = 8.0 * (static_cast<double>(p) + kmax + static_cast<double>(m) * L + 2.0 * p);
  const double budget = 1024.0 * 1024.0 * 1024.0;
  if (per_row * w <= budget) return w;
  return std::max(128, static_cast<int>(budget / per_row));
}

// outer_pred[i] = prediction of the refit of i's outer fold at the chosen slice
// (or the single-class fallback).
__global__ void gather_outer_pred_kernel(const int* __restrict__ pred, const int* __restrict__ outer,
                                         const int* __restrict__ best_slice, const int* __restrict__ fb,
                                         int Ko, int L, int n, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = outer[i];
  if (o < 0 || o >= Ko) { out[i] = 0; return; }
  out[i] = fb[o] ? fb[o] : pred[((size_t)Ko * L + best_slice[o]) * n + i];
}

// Class scores behind the outer predictions: row i of outer slot o takes the
// refit's scores at the chosen slice (zeros for a fallback fold).
__global__ void gather_outer_score_kernel(const double* __restrict__ score, const int* __restrict__ outer,
                                          const int* __restrict__ best_slice, const int* __restrict__ fb,
                                          int Ko, int L, int n, int m, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = outer[i];
  const bool take = o >= 0 && o < Ko && !fb[o];
  const double* src = take ? score + (((size_t)Ko * L + best_slice[o]) * n + i) * m : nullptr;
  for (int j = 0; j < m; ++j) out[(size_t)i * m + j] = take ? src[j] : 0.0;
}

// Slot s of a double CV (outer fold ids[s]): the inner accuracy of every ncomp
// slice from the prediction counts (NaN when no row was predicted), the first
// slice of maximal finite accuracy (.cv_best_index) and the chosen ncomp (the
// smallest one for a single-class fold, fb[s] != 0, whose rows get the
// fallback class).
__global__ void select_ncomp_kernel(const long long* __restrict__ counts, int S, int L, const int* __restrict__ ids,
                                    int Ko, const int* __restrict__ nc, const int* __restrict__ fb, int nc_min,
                                    double* __restrict__ acc_out, int* __restrict__ best_slice,
                                    int* __restrict__ best_comp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int o = ids[s];
  int bi = 0;
  double bv = -1.0;
  bool any = false;
  for (int l = 0; l < L; ++l) {
    const long long ok = counts[2 * ((size_t)s * L + l)], tot = counts[2 * ((size_t)s * L + l) + 1];
    const double acc = tot ? static_cast<double>(ok) / static_cast<double>(tot) : nan("");
    acc_out[o + (size_t)l * Ko] = acc;
    if (isfinite(acc) && (!any || acc > bv)) {
      bv = acc;
      bi = l;
      any = true;
    }
  }
  best_slice[s] = bi;
  best_comp[o] = fb[s] ? nc_min : nc[bi];
}

void lda_outputs_to_host(const LdaModelsDev& d, int C, int kmax, int L, double* means,
                         double* linear, double* constants, double* priors) {
  download(means, d.means, (size_t)C * kmax * L);
  download(linear, d.linear, (size_t)C * kmax * L);
  download(constants, d.constants, (size_t)C * L);
  download(priors, d.priors, (size_t)C);
}

}  // namespace

extern "C" {

const char* fpls_version(void) { return "fastpls_b200 0.1 (sm_100a)"; }

int fpls_has_cuda(void) {
  try {
    Context::get();
    return 1;
  } catch (...) {
    return 0;
  }
}

int fpls_reset_workspace(char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context::get().sync();
    split_gemm_release_cache();
    dual_release_graph();
    simpls_release_graph();
    ozaki_release_cache();
    Context::get().release();
  });
}

int fpls_matrix_multiply(const double* A, int a_rows, int a_cols, const double* B, int b_cols,
                         double* C, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(a_rows >= 0 && a_cols >= 0 && b_cols >= 0, "matrix dimensions must be >= 0");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dA = upload(A, (size_t)a_rows * a_cols);
    const double* dB = upload(B, (size_t)a_cols * b_cols);
    double* dC = ctx.arena.alloc_n<double>((size_t)a_rows * b_cols + 1);
    gemm(false, false, a_rows, b_cols, a_cols, 1.0, dA, a_rows, dB, a_cols, 0.0, dC, a_rows);
    download(C, dC, (size_t)a_rows * b_cols);
    ctx.sync();
  });
}

int fpls_truncated_svd(const double* A, int rows, int cols, int k, int svd_method, int oversample,
                       int power_iters, double svds_tol, int seed, int left_only, double* U,
                       double* s, double* Vt, int* rank_out, char* err, size_t errlen) {
  (void)svds_tol;
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(rows > 0 && cols > 0, "truncated_svd requires a non-empty matrix");
    FPLS_REQUIRE(k >= 1, "truncated_svd: k must be >= 1");
    Context& ctx = Context::get();
    ctx.begin_call();
    const int kcap = std::min(std::min(rows, cols), std::max(k, 1));
    const double* dA = upload(A, (size_t)rows * cols);
    double* dU = ctx.arena.alloc_n<double>((size_t)rows * kcap);
    double* ds = ctx.arena.alloc_n<double>(kcap);
    double* dV = ctx.arena.alloc_n<double>((size_t)cols * kcap);
    dzero(dU, (size_t)rows * kcap * sizeof(double));
    dzero(ds, kcap * sizeof(double));
    dzero(dV, (size_t)cols * kcap * sizeof(double));
    SvdResult r = truncated_svd_device(dA, rows, cols, rows, k, svd_method, oversample,
                                       power_iters, static_cast<unsigned int>(seed), left_only != 0,
                                       false, dU, rows, ds, left_only ? nullptr : dV, cols);
    download(U, dU, (size_t)rows * kcap);
    download(s, ds, kcap);
    if (!left_only && Vt) {
      double* dVt = ctx.arena.alloc_n<double>((size_t)cols * kcap);
      transpose_small<<<ceil_div((long long)cols * kcap, 256), 256, 0, ctx.stream>>>(dV, cols, kcap, dVt); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      download(Vt, dVt, (size_t)cols * kcap);
    }
    ctx.sync();
    if (rank_out) *rank_out = r.rank;
  });
}

}  // extern "C"

namespace {

int pls_model1_impl(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                    int scaling, int fit, int svd_method, int oversample, int power_iters,
                    double svds_tol, int seed, bool xprod, int* ncomp_out, double* C_latent,
                    double* W_latent, double* Q, double* Ttrain, double* R, double* mX, double* vX,
                    double* mY, double* B, double* Yfit, double* R2Y, double* s, int* k_eff, char* err,
                    size_t errlen, fpls_allreduce_fn allreduce = nullptr, void* user = nullptr) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model1 requires non-empty X and Y");
    FPLS_REQUIRE(L >= 1 && ncomp, "ncomp must contain at least one value");
    FPLS_REQUIRE(!(fit && !Yfit), "fit = 1 requires a Yfit buffer");
    FPLS_REQUIRE(!(allreduce && xprod), "row-sharded fits form S = X^T Y (no matrix-free operator)");
    Context& ctx = Context::get();
    ctx.begin_call();
    std::unique_ptr<RowShardScope> shards;
    if (allreduce) shards.reset(new RowShardScope(ctx, allreduce, user, n));
    const int max_rank = static_cast<int>(std::min<long long>(shard_rows(n), std::min(p, m)));
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, std::min(c, max_rank));
    const int K0 = std::min(max_of(nc.data(), L), max_rank);
    double* dX = upload(X, (size_t)n * p);
    double* dY = upload(Y, (size_t)n * m);
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    double* dmY = ctx.arena.alloc_n<double>(m);
    center_scale_xy(dX, n, p, dY, m, scaling, dmX, dvX, dmY);
    FitOptions opt;
    opt.scaling = scaling;
    opt.fit = fit != 0;
    opt.svd_method = svd_method;
    opt.oversample = oversample;
    opt.power_iters = power_iters;
    opt.svds_tol = svds_tol;
    opt.seed = static_cast<unsigned int>(seed);
    opt.xprod = xprod;
    PlssvdOut o;
    o.C_latent = ctx.arena.alloc_n<double>((size_t)K0 * K0 * L);
    o.W_latent = ctx.arena.alloc_n<double>((size_t)K0 * m * L);
    o.R = ctx.arena.alloc_n<double>((size_t)p * K0);
    o.Q = ctx.arena.alloc_n<double>((size_t)m * K0);
    o.T = ctx.arena.alloc_n<double>((size_t)n * K0);
    o.s = ctx.arena.alloc_n<double>(K0);
    o.B = B ? ctx.arena.alloc_n<double>((size_t)p * m * L) : nullptr;
    o.Yfit = fit ? ctx.arena.alloc_n<double>((size_t)n * m * L) : nullptr;
    std::vector<double> r2(L, 0.0);
    o.R2Y = r2.data();
    const int keff = plssvd_fit_centered(dX, n, p, dY, m, nc.data(), L, K0, opt, dmY, o);
    download(C_latent, o.C_latent, (size_t)K0 * K0 * L);
    download(W_latent, o.W_latent, (size_t)K0 * m * L);
    download(Q, o.Q, (size_t)m * K0);
    download(Ttrain, o.T, (size_t)n * K0);
    download(R, o.R, (size_t)p * K0);
    download(mX, dmX, p);
    download(vX, dvX, p);
    download(mY, dmY, m);
    if (B) download(B, o.B, (size_t)p * m * L);
    if (fit) download(Yfit, o.Yfit, (size_t)n * m * L);
    download(s, o.s, K0);
    ctx.sync();
    if (R2Y) std::copy(r2.begin(), r2.end(), R2Y);
    if (ncomp_out) std::copy(nc.begin(), nc.end(), ncomp_out);
    if (k_eff) *k_eff = keff;
  });
}

}  // namespace

extern "C" {

int fpls_pls_model1(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                    int scaling, int fit, int svd_method, int oversample, int power_iters,
                    double svds_tol, int seed, int* ncomp_out, double* C_latent, double* W_latent,
                    double* Q, double* Ttrain, double* R, double* mX, double* vX, double* mY,
                    double* B, double* Yfit, double* R2Y, double* s, int* k_eff, char* err,
                    size_t errlen) {
  return pls_model1_impl(X, n, p, Y, m, ncomp, L, scaling, fit, svd_method, oversample, power_iters,
                         svds_tol, seed, false, ncomp_out, C_latent, W_latent, Q, Ttrain, R, mX, vX,
                         mY, B, Yfit, R2Y, s, k_eff, err, errlen);
}

int fpls_pls_model1_xprod(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                          int L, int scaling, int fit, int oversample, int power_iters,
                          double svds_tol, int seed, int xprod_precision, int* ncomp_out,
                          double* C_latent, double* W_latent, double* Q, double* Ttrain, double* R,
                          double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                          double* s, int* k_eff, char* err, size_t errlen) {
  if (xprod_precision != 3) {
    capi::set_err(err, errlen, xprod_precision == 5
                                   ? "xprod_precision 5 (IRLBA operator) is a CPU-only path in fastPLS"
                                   : "xprod_precision values 1, 2, and 4 have been removed from fastPLS.");
    return FPLS_ERR_ARGUMENT;
  }
  return pls_model1_impl(X, n, p, Y, m, ncomp, L, scaling, fit, kSvdCpuRsvd, oversample, power_iters,
                         svds_tol, seed, true, ncomp_out, C_latent, W_latent, Q, Ttrain, R, mX, vX, mY,
                         B, Yfit, R2Y, s, k_eff, err, errlen);
}

int fpls_pls_model2_fast_xprod(const double* X, int n, int p, const double* Y, int m,
                               const int* ncomp, int L, int scaling, int fit, int seed,
                               int xprod_precision, double* R, double* Q, double* mX, double* vX,
                               double* mY, double* B, double* Yfit, double* R2Y, int* n_components,
                               char* err, size_t errlen) {
  if (xprod_precision != 3) {
    capi::set_err(err, errlen, xprod_precision == 5
                                   ? "xprod_precision 5 (IRLBA operator) is a CPU-only path in fastPLS"
                                   : "xprod_precision values 1, 2, and 4 have been removed from fastPLS.");
    return FPLS_ERR_ARGUMENT;
  }
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model2_fast requires non-empty X and Y");
    FPLS_REQUIRE(L >= 1 && ncomp, "ncomp must contain at least one value");
    FPLS_REQUIRE(!(fit && !Yfit), "fit = 1 requires a Yfit buffer");
    Context& ctx = Context::get();
    ctx.begin_call();
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, c);
    const int K = max_of(nc.data(), L);
    double* dX = upload(X, (size_t)n * p);
    double* dY = upload(Y, (size_t)n * m);
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    double* dmY = ctx.arena.alloc_n<double>(m);
    center_scale_xy(dX, n, p, dY, m, scaling, dmX, dvX, dmY);
    double* dR = ctx.arena.alloc_n<double>((size_t)p * K);
    double* dQ = ctx.arena.alloc_n<double>((size_t)m * K);
    double* dB = B ? ctx.arena.alloc_n<double>((size_t)p * m * L) : nullptr;
    double* dYf = fit ? ctx.arena.alloc_n<double>((size_t)n * m * L) : nullptr;
    std::vector<double> r2(L, 0.0);
    const int done = simpls_xprod_fit(dX, n, p, dY, m, nc.data(), L, fit != 0,
                                      static_cast<unsigned int>(seed), dmY, dR, dQ, dB, dYf, r2.data());
    download(R, dR, (size_t)p * K);
    download(Q, dQ, (size_t)m * K);
    download(mX, dmX, p);
    download(vX, dvX, p);
    download(mY, dmY, m);
    if (B) download(B, dB, (size_t)p * m * L);
    if (fit) download(Yfit, dYf, (size_t)n * m * L);
    ctx.sync();
    if (R2Y) std::copy(r2.begin(), r2.end(), R2Y);
    if (n_components) *n_components = done;
  });
}

// Fast SIMPLS (pls_model2_fast) on device copies of X (n x p) and Y (n x m),
// both centred / scaled in place; host outputs as fpls_pls_model2_fast.
static void simpls_fast_on_device(double* dX, int n, int p, double* dYc, int m, const int* ncomp, int L,
                                  int scaling, int fit, int seed, double* R, double* Q, double* mX, double* vX,
                                  double* mY, double* B, double* Yfit, double* R2Y, int* n_components) {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model2_fast requires non-empty X and Y");
    FPLS_REQUIRE(L >= 1 && ncomp, "ncomp must contain at least one value");
    FPLS_REQUIRE(!(fit && !Yfit), "fit = 1 requires a Yfit buffer");
    FPLS_REQUIRE(p > 5 || m == 1,
                 "pls_model2_fast with <= 5 predictors and several responses is not supported on "
                 "the GPU path");
    Context& ctx = Context::get();
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, c);
    const int K = max_of(nc.data(), L);
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    double* dmY = ctx.arena.alloc_n<double>(m);
    center_scale_xy(dX, n, p, dYc, m, scaling, dmX, dvX, dmY);
    // Single fit on all rows: S = Xc^T Yc as the reference (fastPLS.cpp:2499);
    // the two predictor passes per component run FP64 or, in the mixed
    // session precision, as BF16x3 tensor-core products.
    std::unique_ptr<XOperator> xop;
    if (ctx.precision >= 1) xop = make_split_operator(dX, n, p, true, ctx.precision == 2 ? 3 : 2);
    else xop.reset(new XOperatorF64(dX, n, p));
    SimplsBatch b;
    b.n = n; b.p = p; b.m = m; b.F = 1; b.K = K;
    int iters = 2;
    if (const char* e = std::getenv("FASTPLS_FAST_INC_ITERS")) {
      char* endp = nullptr;
      long v = std::strtol(e, &endp, 10);
      if (endp != e) iters = static_cast<int>(std::min(6L, std::max(1L, v)));
    }
    b.power_iters = iters;
    b.X = xop.get();
    b.Yg = dYc;
    b.S = ctx.arena.alloc_n<double>((size_t)p * m);
    xgemm(true, p, m, n, dX, n, dYc, n, b.S, p);
    shard_sum(b.S, (size_t)p * m);
    double* om = ctx.arena.alloc_n<double>(p);
    device_gaussian(om, p, static_cast<unsigned int>(seed));
    b.omega = om;
    b.m1_mode = (m == 1);
    b.R = ctx.arena.alloc_n<double>((size_t)p * K);
    b.Q = ctx.arena.alloc_n<double>((size_t)m * K);
    b.V = ctx.arena.alloc_n<double>((size_t)p * K);
    b.tnorm = ctx.arena.alloc_n<double>(K);
    b.Tkeep = fit ? ctx.arena.alloc_n<double>((size_t)n * K) : nullptr;
    b.ncomp_done = ctx.arena.alloc_n<int>(1);
    b.status = ctx.arena.alloc_n<int>(1);
    simpls_batch_run(b);
    int done = 0;
    d2h(&done, b.ncomp_done, sizeof(int));
    std::vector<double> tn(K);
    d2h(tn.data(), b.tnorm, K * sizeof(double));
    ctx.sync();
    // Slices exactly as the reference's while loop assigns them (fastPLS.cpp:2648-2661).
    double* dB = B ? ctx.arena.alloc_n<double>((size_t)p * m * L) : nullptr;
    if (dB) dzero(dB, (size_t)p * m * L * sizeof(double));
    double* dYf = fit ? ctx.arena.alloc_n<double>((size_t)n * m * L) : nullptr;
    double* cur = fit ? ctx.arena.alloc_n<double>((size_t)n * m) : nullptr;
    double* tcol = fit ? ctx.arena.alloc_n<double>(n) : nullptr;
    double* rq = fit ? ctx.arena.alloc_n<double>(2 * L) : nullptr;
    if (fit) {
      dzero(rq, 2 * (size_t)L * sizeof(double));
      dzero(dYf, (size_t)n * m * L * sizeof(double));
      dzero(cur, (size_t)n * m * sizeof(double));
    }
    std::vector<int> filled(L, 0);
    const double* rq_mu = fit ? shard_rq_means(dYc, n, m) : nullptr;
    int i_out = 0;
    for (int a = 0; a < done; ++a) {
      while (i_out < L && a == nc[i_out] - 1) {
        if (dB) gemm(false, true, p, m, a + 1, 1.0, b.R, p, b.Q, m, 0.0, dB + (size_t)i_out * p * m, p);
        if (fit) {
          scale_column_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(b.Tkeep + (size_t)a * n, n, 1.0 / tn[a], tcol); ::fpls::note_launch();
          FPLS_CHECK_LAUNCH();
          gemm(false, true, n, m, 1, 1.0, tcol, n, b.Q + (size_t)a * m, m, 1.0, cur, n);
          rq_sums(dYc, cur, n, m, rq + 2 * i_out, rq_mu);
          double* sl = dYf + (size_t)i_out * n * m;
          d2d(sl, cur, (size_t)n * m * sizeof(double));
          add_row_vector(sl, n, m, n, dmY);
        }
        filled[i_out] = 1;
        ++i_out;
      }
    }
    download(R, b.R, (size_t)p * K);
    download(Q, b.Q, (size_t)m * K);
    download(mX, dmX, p);
    download(vX, dvX, p);
    download(mY, dmY, m);
    if (B) download(B, dB, (size_t)p * m * L);
    std::vector<double> hrq(2 * L, 0.0);
    if (fit) {
      shard_sum(rq, 2 * (size_t)L);
      download(Yfit, dYf, (size_t)n * m * L);
      download(hrq.data(), rq, 2 * (size_t)L);
    }
    ctx.sync();
    if (R2Y) {
      for (int i = 0; i < L; ++i)
        R2Y[i] = (fit && filled[i]) ? 1.0 - hrq[2 * i] / hrq[2 * i + 1] : 0.0;
    }
    if (n_components) *n_components = done;
}

int fpls_pls_model2_fast(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                         int L, int scaling, int fit, int seed, double* R, double* Q, double* mX,
                         double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                         int* n_components, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model2_fast requires non-empty X and Y");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dX = upload(X, (size_t)n * p);
    double* dYc = upload(Y, (size_t)n * m);
    simpls_fast_on_device(dX, n, p, dYc, m, ncomp, L, scaling, fit, seed, R, Q, mX, vX, mY, B, Yfit, R2Y,
                          n_components);
  });
}

int fpls_pls_model2_fast_rows(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                              int L, int scaling, int fit, int seed, fpls_allreduce_fn allreduce, void* user,
                              double* R, double* Q, double* mX, double* vX, double* mY, double* B,
                              double* Yfit, double* R2Y, int* n_components, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model2_fast requires non-empty X and Y");
    FPLS_REQUIRE(allreduce != nullptr, "pls_model2_fast_rows: the all-reduce callback is null");
    Context& ctx = Context::get();
    ctx.begin_call();
    RowShardScope shards(ctx, allreduce, user, n);
    double* dX = upload(X, (size_t)n * p);
    double* dYc = upload(Y, (size_t)n * m);
    simpls_fast_on_device(dX, n, p, dYc, m, ncomp, L, scaling, fit, seed, R, Q, mX, vX, mY, B, Yfit, R2Y,
                          n_components);
  });
}

int fpls_pls_model1_rows(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                         int scaling, int fit, int svd_method, int oversample, int power_iters,
                         double svds_tol, int seed, fpls_allreduce_fn allreduce, void* user, int* ncomp_out,
                         double* C_latent, double* W_latent, double* Q, double* Ttrain, double* R, double* mX,
                         double* vX, double* mY, double* B, double* Yfit, double* R2Y, double* s, int* k_eff,
                         char* err, size_t errlen) {
  if (!allreduce) {
    capi::set_err(err, errlen, "pls_model1_rows: the all-reduce callback is null");
    return FPLS_ERR_ARGUMENT;
  }
  return pls_model1_impl(X, n, p, Y, m, ncomp, L, scaling, fit, svd_method, oversample, power_iters,
                         svds_tol, seed, false, ncomp_out, C_latent, W_latent, Q, Ttrain, R, mX, vX,
                         mY, B, Yfit, R2Y, s, k_eff, err, errlen, allreduce, user);
}

int fpls_kernel_matrix(const double* X1, int n1, const double* X2, int n2, int p, int kernel, double gamma,
                       int degree, double coef0, double* K, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n1 > 0 && n2 > 0 && p > 0, "X1 and X2 must be non-empty");
    FPLS_REQUIRE(kernel >= 1 && kernel <= 3, "Unknown kernel id");
    FPLS_REQUIRE(kernel == 1 || (std::isfinite(gamma) && gamma > 0.0), "gamma must be a finite positive number");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* d1 = upload(X1, (size_t)n1 * p);
    const double* d2 = (X2 == X1 && n2 == n1) ? d1 : upload(X2, (size_t)n2 * p);
    double* dK = ctx.arena.alloc_n<double>((size_t)n1 * n2);
    kernel_matrix_device(d1, n1, d2, n2, p, kernel, gamma, degree, coef0, dK);
    download(K, dK, (size_t)n1 * n2);
    ctx.sync();
  });
}

int fpls_center_kernel_train(const double* K, int n, double* Kc, double* col_means, double* grand_mean, char* err,
                             size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0, "K must be non-empty");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dK = upload(K, (size_t)n * n);
    double* dcm = ctx.arena.alloc_n<double>(n);
    double* dg = ctx.arena.alloc_n<double>(1);
    center_kernel_train_device(dK, n, dcm, dg);
    download(Kc, dK, (size_t)n * n);
    download(col_means, dcm, n);
    download(grand_mean, dg, 1);
    ctx.sync();
  });
}

int fpls_center_kernel_test(const double* Ktest, int nt, int n, const double* col_means, double grand_mean,
                            double* Kc, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(nt > 0 && n > 0, "Ktest must be non-empty");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dK = upload(Ktest, (size_t)nt * n);
    const double* dcm = upload(col_means, n);
    const double* dg = upload(&grand_mean, 1);
    center_kernel_test_device(dK, nt, n, dcm, dg);
    download(Kc, dK, (size_t)nt * n);
    ctx.sync();
  });
}

int fpls_kernel_pls_model2_fast(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                                int scaling, int kernel, double gamma, int degree, double coef0, int fit,
                                int seed, double* R, double* Q, double* mK, double* vK, double* mY, double* B,
                                double* Yfit, double* R2Y, int* n_components, double* mX, double* vX,
                                double* col_means, double* grand_mean, double* gamma_used, char* err,
                                size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "kernel PLS requires non-empty X and Y");
    FPLS_REQUIRE(kernel >= 1 && kernel <= 3, "Unknown kernel id");
    FPLS_REQUIRE(scaling >= 1 && scaling <= 3, "scaling must be 1, 2 or 3");
    const double g = gamma > 0.0 ? gamma : 1.0 / std::max(1, p);   // .kernel_pls_gamma: NULL -> 1 / p
    FPLS_REQUIRE(std::isfinite(g), "gamma must be a finite positive number");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dX = upload(X, (size_t)n * p);
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    preprocess_kernel_x_device(dX, n, p, scaling, dmX, dvX);
    double* dK = ctx.arena.alloc_n<double>((size_t)n * n);
    kernel_matrix_device(dX, n, dX, n, p, kernel, g, degree, coef0, dK);
    double* dcm = ctx.arena.alloc_n<double>(n);
    double* dg = ctx.arena.alloc_n<double>(1);
    center_kernel_train_device(dK, n, dcm, dg);
    download(mX, dmX, p);
    download(vX, dvX, p);
    download(col_means, dcm, n);
    download(grand_mean, dg, 1);
    if (gamma_used) *gamma_used = g;
    double* dY = upload(Y, (size_t)n * m);
    // The inner fit runs on the centred kernel with scaling "none" (R/main.R:2875-2891).
    simpls_fast_on_device(dK, n, n, dY, m, ncomp, L, 3, fit, seed, R, Q, mK, vK, mY, B, Yfit, R2Y, n_components);
  });
}

int fpls_pls_model2(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                    int L, int scaling, int fit, int svd_method, int oversample, int power_iters,
                    double svds_tol, int seed, double* R, double* Q, double* P, double* Ttrain,
                    double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                    int* n_components, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0, "pls_model2 requires non-empty X and Y");
    FPLS_REQUIRE(L >= 1 && ncomp, "ncomp must contain at least one value");
    FPLS_REQUIRE(!(fit && !Yfit), "fit = 1 requires a Yfit buffer");
    Context& ctx = Context::get();
    ctx.begin_call();
    const int K = max_of(ncomp, L);
    FPLS_REQUIRE(K >= 1, "ncomp must be >= 1");
    double* dX = upload(X, (size_t)n * p);
    double* dYraw = upload(Y, (size_t)n * m);
    double* dY = ctx.arena.alloc_n<double>((size_t)n * m);
    d2d(dY, dYraw, (size_t)n * m * sizeof(double));
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    double* dmY = ctx.arena.alloc_n<double>(m);
    center_scale_xy(dX, n, p, dY, m, scaling, dmX, dvX, dmY);
    FitOptions opt;
    opt.scaling = scaling;
    opt.fit = fit != 0;
    opt.svd_method = svd_method;
    opt.oversample = oversample;
    opt.power_iters = power_iters;
    opt.svds_tol = svds_tol;
    opt.seed = static_cast<unsigned int>(seed);
    SimplsOut o;
    o.R = ctx.arena.alloc_n<double>((size_t)p * K);
    o.Q = ctx.arena.alloc_n<double>((size_t)m * K);
    o.P = ctx.arena.alloc_n<double>((size_t)p * K);
    o.T = ctx.arena.alloc_n<double>((size_t)n * K);
    o.B = B ? ctx.arena.alloc_n<double>((size_t)p * m * L) : nullptr;
    if (o.B) dzero(o.B, (size_t)p * m * L * sizeof(double));
    o.Yfit = fit ? ctx.arena.alloc_n<double>((size_t)n * m * L) : nullptr;
    if (o.Yfit) dzero(o.Yfit, (size_t)n * m * L * sizeof(double));
    std::vector<double> r2(L, 0.0);
    o.R2Y = r2.data();
    const int done = simpls_classic_fit(dX, n, p, dY, m, dYraw, ncomp, L, opt, dmY, o);
    download(R, o.R, (size_t)p * K);
    download(Q, o.Q, (size_t)m * K);
    download(P, o.P, (size_t)p * K);
    download(Ttrain, o.T, (size_t)n * K);
    download(mX, dmX, p);
    download(vX, dvX, p);
    download(mY, dmY, m);
    if (B) download(B, o.B, (size_t)p * m * L);
    if (fit) download(Yfit, o.Yfit, (size_t)n * m * L);
    ctx.sync();
    if (R2Y) std::copy(r2.begin(), r2.end(), R2Y);
    if (n_components) *n_components = done;
  });
}

int fpls_predict_lowrank(const double* Xtest, int w, int p, const double* mX, const double* vX,
                         const double* mY, int m, const double* R, int kmax, const double* W,
                         const int* ncomp, int L, double* Ypred, double* Ttest, char* err,
                         size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && p > 0 && m > 0 && kmax > 0 && L > 0, "predict: empty input");
    for (int a = 0; a < L; ++a)
      FPLS_REQUIRE(ncomp[a] >= 1 && ncomp[a] <= kmax, "ncomp exceeds latent rank for prediction");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dmX = upload(mX, p);
    const double* dvX = upload(vX, p);
    const double* dmY = upload(mY, m);
    const double* dR = upload(R, (size_t)p * kmax);
    const double* dW = upload(W, (size_t)kmax * m * L);
    double* dX = centered_test_copy(Xtest, w, p, dmX, dvX);
    double* dT = ctx.arena.alloc_n<double>((size_t)w * kmax);
    double* dYp = ctx.arena.alloc_n<double>((size_t)w * m * L);
    lowrank_predict(dX, w, p, dR, kmax, dW, m, ncomp, L, dmY, dT, dYp);
    download(Ypred, dYp, (size_t)w * m * L);
    if (Ttest) download(Ttest, dT, (size_t)w * kmax);
    ctx.sync();
  });
}

int fpls_predict_classes(const double* Xtest, int w, int p, const double* mX, const double* vX,
                         const double* mY, int m, const double* R, int kmax, const double* W,
                         const int* ncomp, int L, const double* class_bias, int top_k,
                         int* top_index, double* top_score, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && p > 0 && m > 0 && kmax > 0 && L > 0, "predict: empty input");
    FPLS_REQUIRE(top_k >= 1 && top_k <= std::min(m, 32), "top_k must be in 1..min(m, 32)");
    for (int a = 0; a < L; ++a)
      FPLS_REQUIRE(ncomp[a] >= 1 && ncomp[a] <= kmax, "ncomp exceeds latent rank for prediction");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dmX = upload(mX, p);
    const double* dvX = upload(vX, p);
    const double* dmY = upload(mY, m);
    const double* dR = upload(R, (size_t)p * kmax);
    const double* dW = upload(W, (size_t)kmax * m * L);
    const double* dbias = class_bias ? upload(class_bias, m) : nullptr;
    int* didx = ctx.arena.alloc_n<int>((size_t)w * top_k * L);
    double* dsc = ctx.arena.alloc_n<double>((size_t)w * top_k * L);
    const int B = predict_block_rows(w, p, kmax, m, L);
    if (B >= w) {
      double* dX = centered_test_copy(Xtest, w, p, dmX, dvX);
      double* dT = ctx.arena.alloc_n<double>((size_t)w * kmax);
      double* dYp = ctx.arena.alloc_n<double>((size_t)w * m * L);
      lowrank_predict(dX, w, p, dR, kmax, dW, m, ncomp, L, dmY, dT, dYp);
      for (int a = 0; a < L; ++a) {
        const double* Ya = dYp + (size_t)a * w * m;
        if (top_k == 1 && !top_score) {
          row_argmax(Ya, w, m, dbias, didx + (size_t)a * w);
        } else {
          row_topk(Ya, w, m, dbias, top_k, didx + (size_t)a * w * top_k, dsc + (size_t)a * w * top_k);
        }
      }
    } else {
      // Streamed: row blocks of B test rows, the next block's copy (copy
      // stream, double-buffered) in flight while this one is scored; device
      // memory O(B (p + kmax + m L)) whatever the number of test rows.
      double* xb[2] = {ctx.arena.alloc_n<double>((size_t)B * p), ctx.arena.alloc_n<double>((size_t)B * p)};
      double* dT = ctx.arena.alloc_n<double>((size_t)B * kmax);
      double* dYp = ctx.arena.alloc_n<double>((size_t)B * m * L);
      int* bidx = ctx.arena.alloc_n<int>((size_t)B * top_k);
      double* bsc = ctx.arena.alloc_n<double>((size_t)B * top_k);
      FPLS_CUDA(cudaEventRecord(ctx.copy_event(4), ctx.stream));   // the buffers are this call's
      FPLS_CUDA(cudaStreamWaitEvent(ctx.copy, ctx.copy_event(4), 0));
      const int nblk = ceil_div(w, B);
      auto issue_copy = [&](int blk) {
        const int r0 = blk * B, rb = std::min(B, w - r0), b = blk & 1;
        if (blk >= 2) FPLS_CUDA(cudaStreamWaitEvent(ctx.copy, ctx.copy_event(2 + b), 0));   // xb[b] is free
        FPLS_CUDA(cudaMemcpy2DAsync(xb[b], (size_t)rb * sizeof(double), Xtest + r0, (size_t)w * sizeof(double),
                                    (size_t)rb * sizeof(double), p, cudaMemcpyDefault, ctx.copy));
        FPLS_CUDA(cudaEventRecord(ctx.copy_event(b), ctx.copy));
      };
      issue_copy(0);
      for (int blk = 0; blk < nblk; ++blk) {
        const int r0 = blk * B, rb = std::min(B, w - r0), b = blk & 1;
        if (blk + 1 < nblk) issue_copy(blk + 1);
        FPLS_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.copy_event(b), 0));
        center_copy_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(xb[b], rb, p, dmX, dvX, xb[b]);
        ::fpls::note_launch();
        FPLS_CHECK_LAUNCH();
        lowrank_predict(xb[b], rb, p, dR, kmax, dW, m, ncomp, L, dmY, dT, dYp);
        FPLS_CUDA(cudaEventRecord(ctx.copy_event(2 + b), ctx.stream));   // xb[b] read by now
        for (int a = 0; a < L; ++a) {
          const double* Ya = dYp + (size_t)a * rb * m;
          if (top_k == 1 && !top_score) row_argmax(Ya, rb, m, dbias, bidx);
          else row_topk(Ya, rb, m, dbias, top_k, bidx, bsc);
          place_rows_kernel<<<ceil_div((long long)rb * top_k, 256), 256, 0, ctx.stream>>>(
              bidx, top_score ? bsc : nullptr, rb, top_k, w, r0, didx + (size_t)a * w * top_k,
              top_score ? dsc + (size_t)a * w * top_k : nullptr);
          ::fpls::note_launch();
          FPLS_CHECK_LAUNCH();
        }
      }
    }
    download(top_index, didx, (size_t)w * top_k * L);
    if (top_score) download(top_score, dsc, (size_t)w * top_k * L);
    ctx.sync();
  });
}

int fpls_lda_train_prefix(const double* T, int n, int kmax, const int* y, int n_classes,
                          const int* ncomp, int L, double ridge, double* means, double* linear,
                          double* constants, double* priors, double* lambda, char* err,
                          size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && kmax > 0, "lda_train_prefix requires a non-empty score matrix");
    FPLS_REQUIRE(L >= 1, "lda_train_prefix requires at least one component count");
    const int km = max_of(ncomp, L);
    for (int a = 0; a < L; ++a)
      FPLS_REQUIRE(ncomp[a] >= 1 && ncomp[a] <= kmax,
                   "lda_train_prefix component counts must be in 1..ncol(Ttrain)");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dT = upload(T, (size_t)n * kmax);
    LdaModelsDev d;
    d.means = ctx.arena.alloc_n<double>((size_t)n_classes * km * L);
    d.linear = ctx.arena.alloc_n<double>((size_t)n_classes * km * L);
    d.constants = ctx.arena.alloc_n<double>((size_t)n_classes * L);
    d.priors = ctx.arena.alloc_n<double>(n_classes);
    std::vector<double> lam(L);
    d.lambda = lam.data();
    lda_train_prefix(dT, n, km, y, n_classes, ncomp, L, ridge, d);
    lda_outputs_to_host(d, n_classes, km, L, means, linear, constants, priors);
    ctx.sync();
    if (lambda) std::copy(lam.begin(), lam.end(), lambda);
  });
}

int fpls_lda_project_train_prefix(const double* X, int n, int p, const double* R, int k,
                                  const double* offset, const int* y, int n_classes,
                                  const int* ncomp, int L, double ridge, double* means,
                                  double* linear, double* constants, double* priors,
                                  double* lambda, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0, "lda_project_train_prefix requires a non-empty predictor matrix");
    FPLS_REQUIRE(k > 0, "lda_project_train_prefix projection matrix has incompatible dimensions");
    const int km = max_of(ncomp, L);
    for (int a = 0; a < L; ++a)
      FPLS_REQUIRE(ncomp[a] >= 1 && ncomp[a] <= k, "component counts must be in 1..ncol(R)");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dX = upload(X, (size_t)n * p);
    const double* dR = upload(R, (size_t)p * k);
    double* dT = ctx.arena.alloc_n<double>((size_t)n * k);
    xgemm(false, n, k, p, dX, n, dR, p, dT, n);
    if (offset) {
      double* doff = upload(offset, k);
      scale_vec(doff, k, -1.0);
      add_row_vector(dT, n, k, n, doff);
    }
    LdaModelsDev d;
    d.means = ctx.arena.alloc_n<double>((size_t)n_classes * km * L);
    d.linear = ctx.arena.alloc_n<double>((size_t)n_classes * km * L);
    d.constants = ctx.arena.alloc_n<double>((size_t)n_classes * L);
    d.priors = ctx.arena.alloc_n<double>(n_classes);
    std::vector<double> lam(L);
    d.lambda = lam.data();
    lda_train_prefix(dT, n, km, y, n_classes, ncomp, L, ridge, d);
    lda_outputs_to_host(d, n_classes, km, L, means, linear, constants, priors);
    ctx.sync();
    if (lambda) std::copy(lam.begin(), lam.end(), lambda);
  });
}

int fpls_lda_predict(const double* T, int w, int k, const double* linear,
                     const double* constants, int n_classes, int* labels, double* scores,
                     char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && k > 0 && n_classes > 0, "lda_predict requires a non-empty score matrix");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dT = upload(T, (size_t)w * k);
    const double* dL = upload(linear, (size_t)n_classes * k);
    const double* dc = upload(constants, n_classes);
    double* dS = ctx.arena.alloc_n<double>((size_t)w * n_classes);
    gemm(false, true, w, n_classes, k, 1.0, dT, w, dL, n_classes, 0.0, dS, w);
    int* dlab = ctx.arena.alloc_n<int>(w);
    row_argmax(dS, w, n_classes, dc, dlab);
    download(labels, dlab, w);
    if (scores) {
      add_row_vector(dS, w, n_classes, w, dc);
      download(scores, dS, (size_t)w * n_classes);
    }
    ctx.sync();
  });
}

}  // extern "C"

namespace {

// LDA scores of raw rows X (w x p, device) through the projection R (p x k, ld
// ldr) and offset: S = (X R - offset) linear^T + constants, by the direct or
// the latent route as lda_project_predict_labels_cpp chooses
// (fastPLS.cpp:2100-2147, CPU rule with the 0.5 factor); labels (device, w) and,
// when scores is set, the full score matrix (device, w x C).  dc is modified.
void lda_project_scores_device(const double* dX, int w, int p, const double* dR, int ldr, int k,
                               const double* doff, const double* dL, int ldl, double* dc, int C, int* dlab,
                               double* dS_out) {
  Context& ctx = Context::get();
  double* dS = dS_out ? dS_out : ctx.arena.alloc_n<double>((size_t)w * C);
  // constants_adj = constants - offset linear^T
  if (doff) gemv(false, C, k, -1.0, dL, ldl, doff, 1.0, dc);
  const double nn = w, pp = p, kk = k, cc = C;
  const double latent_ops = nn * kk * (pp + cc);
  const double direct_ops = nn * pp * cc;
  if (direct_ops < 0.5 * latent_ops) {
    double* dW = ctx.arena.alloc_n<double>((size_t)p * C);
    gemm(false, true, p, C, k, 1.0, dR, ldr, dL, ldl, 0.0, dW, p);
    xgemm(false, w, C, p, dX, w, dW, p, dS, w);
  } else {
    double* dT = ctx.arena.alloc_n<double>((size_t)w * k);
    gemm(false, false, w, k, p, 1.0, dX, w, dR, ldr, 0.0, dT, w);
    gemm(false, true, w, C, k, 1.0, dT, w, dL, ldl, 0.0, dS, w);
  }
  row_argmax(dS, w, C, dc, dlab);
  if (dS_out) add_row_vector(dS, w, C, w, dc);
}

__global__ void widen_f32_kernel(const float* __restrict__ src, size_t total, double* __restrict__ dst) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
    dst[t] = static_cast<double>(src[t]);
}

// An FP32 device matrix widened exactly into a fresh FP64 copy.
double* widen_on_device(const float* d32, size_t count) {
  Context& ctx = Context::get();
  double* d = ctx.arena.alloc_n<double>(count ? count : 1);
  if (count) {
    widen_f32_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(d32, count, d);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  return d;
}

// A caller's matrix (FP64, or FP32 widened exactly) as a fresh FP64 device copy.
double* upload_widened(const void* X, bool f32, size_t count) {
  if (!f32) return upload(static_cast<const double*>(X), count);
  return widen_on_device(upload(static_cast<const float*>(X), count), count);
}


}  // namespace

extern "C" {

int fpls_pls_lda(const void* Xtrain, int x_is_float32, int n, int p, const double* Ytrain, int m,
                 const int* y, const void* Xtest, int ntest, const int* ncomp, int L, int n_classes,
                 int method, int scaling, int xprod, int fit, int oversample, int power_iters,
                 double svds_tol, int seed, double lda_ridge, int* ncomp_out, double* R, double* Q,
                 double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y, int* n_unique,
                 int* unique_ncomp, double* lda_means, double* lda_linear, double* lda_constants,
                 double* lda_priors, double* lda_lambda, double* R_predict, double* R_offset,
                 int* pred_codes, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && m > 0 && Xtrain && Ytrain && y,
                 "pls_lda requires compatible non-empty Xtrain and Ytrain");
    FPLS_REQUIRE(n_classes >= 2, "pls_lda requires at least two classes");
    FPLS_REQUIRE(L >= 1 && ncomp, "pls_lda requires at least one component count");
    FPLS_REQUIRE(method == 1 || method == 3, "pls_lda supports method 1 (plssvd) or 3 (simpls)");
    FPLS_REQUIRE(ntest == 0 || (Xtest && pred_codes), "pls_lda: Xtest rows need pred_codes");
    FPLS_REQUIRE(!(fit && !Yfit), "fit = 1 requires a Yfit buffer");
    const bool f32 = x_is_float32 != 0;
    Context& ctx = Context::get();
    ctx.begin_call();
    PhaseTimer pt("PLS + LDA call");
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, c);
    // one upload of each matrix for the whole pipeline
    double* dX = upload_widened(Xtrain, f32, (size_t)n * p);
    double* dY = upload(Ytrain, (size_t)n * m);
    // the test rows cross the link while the fit runs
    capi::SideUpload xt_up(Xtest, ntest > 0 ? (size_t)ntest * p * (f32 ? sizeof(float) : sizeof(double)) : 0);
    pt.mark("X, Y to FP64");
    int K0 = 0;
    double* dR = nullptr;
    double* dT = nullptr;   // training scores (X - mX) / vX R, n x K0
    std::vector<double> hR, hmX(p), hvX(p);
    if (method == 1) {
      const int max_rank = std::min(n, std::min(p, m));
      for (int& c : nc) c = std::min(c, max_rank);
      K0 = std::min(max_of(nc.data(), L), max_rank);
      double* dmX = ctx.arena.alloc_n<double>(p);
      double* dvX = ctx.arena.alloc_n<double>(p);
      double* dmY = ctx.arena.alloc_n<double>(m);
      center_scale_xy(dX, n, p, dY, m, scaling, dmX, dvX, dmY);
      pt.mark("centre / scale");
      FitOptions opt;
      opt.scaling = scaling;
      opt.fit = fit != 0;
      opt.svd_method = kSvdCpuRsvd;
      opt.oversample = std::max(oversample, 0);
      opt.power_iters = std::max(power_iters, 0);
      opt.svds_tol = std::max(svds_tol, 0.0);
      opt.seed = static_cast<unsigned int>(seed);
      opt.xprod = xprod != 0;
      PlssvdOut o;
      o.C_latent = ctx.arena.alloc_n<double>((size_t)K0 * K0 * L);
      o.W_latent = ctx.arena.alloc_n<double>((size_t)K0 * m * L);
      o.R = dR = ctx.arena.alloc_n<double>((size_t)p * K0);
      o.Q = ctx.arena.alloc_n<double>((size_t)m * K0);
      o.T = dT = ctx.arena.alloc_n<double>((size_t)n * K0);
      o.s = ctx.arena.alloc_n<double>(K0);
      o.B = B ? ctx.arena.alloc_n<double>((size_t)p * m * L) : nullptr;
      o.Yfit = fit ? ctx.arena.alloc_n<double>((size_t)n * m * L) : nullptr;
      std::vector<double> r2(L, 0.0);
      o.R2Y = r2.data();
      plssvd_fit_centered(dX, n, p, dY, m, nc.data(), L, K0, opt, dmY, o);
      pt.mark("PLSSVD fit");
      download(Q, o.Q, (size_t)m * K0);
      download(mY, dmY, m);
      if (B) download(B, o.B, (size_t)p * m * L);
      if (fit) download(Yfit, o.Yfit, (size_t)n * m * L);
      hR.resize((size_t)p * K0);
      download(hR.data(), dR, (size_t)p * K0);
      download(hmX.data(), dmX, p);
      download(hvX.data(), dvX, p);
      ctx.sync();
      pt.mark("fit outputs to host");
      if (R2Y) std::copy(r2.begin(), r2.end(), R2Y);
    } else {
      K0 = max_of(nc.data(), L);
      hR.resize((size_t)p * K0);
      std::vector<double> hQ((size_t)m * K0), hmY(m);
      int done = 0;
      // centres / scales dX in place (the fit's own copy) and fits on it
      simpls_fast_on_device(dX, n, p, dY, m, nc.data(), L, scaling, fit, seed, hR.data(), hQ.data(), hmX.data(),
                            hvX.data(), hmY.data(), B, Yfit, R2Y, &done);
      if (done < K0) throw Error(FPLS_ERR_NUMERICAL, "pls_lda has invalid effective component count");
      if (Q) std::copy(hQ.begin(), hQ.end(), Q);
      if (mY) std::copy(hmY.begin(), hmY.end(), mY);
      dR = upload(hR.data(), (size_t)p * K0);
      dT = ctx.arena.alloc_n<double>((size_t)n * K0);
      xgemm(false, n, K0, p, dX, n, dR, p, dT, n);
    }
    if (R) std::copy(hR.begin(), hR.end(), R);
    if (mX) std::copy(hmX.begin(), hmX.end(), mX);
    if (vX) std::copy(hvX.begin(), hvX.end(), vX);
    if (ncomp_out) std::copy(nc.begin(), nc.end(), ncomp_out);
    // R_predict = R / vX (rows; a zero or non-finite scale counts as 1) and
    // offset = mX R_predict (fastPLS.cpp:6321-6335)
    std::vector<double> hRp((size_t)p * K0), hoff(K0, 0.0);
    for (int a = 0; a < K0; ++a)
      for (int j = 0; j < p; ++j) {
        double sc = hvX[j];
        if (!std::isfinite(sc) || sc == 0.0) sc = 1.0;
        const double v = hR[j + (size_t)a * p] / sc;
        hRp[j + (size_t)a * p] = v;
        hoff[a] += hmX[j] * v;
      }
    if (R_predict) std::copy(hRp.begin(), hRp.end(), R_predict);
    if (R_offset) std::copy(hoff.begin(), hoff.end(), R_offset);
    // LDA on the fit's training scores, one model per distinct ncomp in
    // increasing order (arma::unique)
    std::vector<int> uq(nc);
    std::sort(uq.begin(), uq.end());
    uq.erase(std::unique(uq.begin(), uq.end()), uq.end());
    const int U = static_cast<int>(uq.size());
    LdaModelsDev d;
    d.means = ctx.arena.alloc_n<double>((size_t)n_classes * K0 * U);
    d.linear = ctx.arena.alloc_n<double>((size_t)n_classes * K0 * U);
    d.constants = ctx.arena.alloc_n<double>((size_t)n_classes * U);
    d.priors = ctx.arena.alloc_n<double>(n_classes);
    std::vector<double> lam(U);
    d.lambda = lam.data();
    pt.mark("prediction weights (host)");
    lda_train_prefix(dT, n, K0, y, n_classes, uq.data(), U, lda_ridge, d);
    pt.mark("LDA train");
    lda_outputs_to_host(d, n_classes, K0, U, lda_means, lda_linear, lda_constants, lda_priors);
    pt.mark("LDA outputs to host");
    if (ntest > 0) {
      xt_up.wait();
      const double* dXt = f32 ? widen_on_device(static_cast<const float*>(xt_up.dst), (size_t)ntest * p)
                              : static_cast<const double*>(xt_up.dst);
      const double* dRp = upload(hRp.data(), (size_t)p * K0);
      const double* doff = upload(hoff.data(), K0);
      int* dpred = ctx.arena.alloc_n<int>((size_t)ntest * L);
      double* dc = ctx.arena.alloc_n<double>(n_classes);
      for (int i = 0; i < L; ++i) {
        const int u = static_cast<int>(std::lower_bound(uq.begin(), uq.end(), nc[i]) - uq.begin());
        d2d(dc, d.constants + (size_t)u * n_classes, n_classes * sizeof(double));
        lda_project_scores_device(dXt, ntest, p, dRp, p, nc[i], doff, d.linear + (size_t)u * n_classes * K0,
                                  n_classes, dc, n_classes, dpred + (size_t)i * ntest, nullptr);
      }
      download(pred_codes, dpred, (size_t)ntest * L);
      pt.mark("test prediction");
    }
    ctx.sync();
    pt.report();
    if (lda_lambda) std::copy(lam.begin(), lam.end(), lda_lambda);
    if (n_unique) *n_unique = U;
    if (unique_ncomp) std::copy(uq.begin(), uq.end(), unique_ncomp);
  });
}

int fpls_lda_project_predict(const double* X, int w, int p, const double* R, int k,
                             const double* offset, const double* linear,
                             const double* constants, int n_classes, int* labels,
                             double* scores, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && p > 0 && k > 0 && n_classes > 0,
                 "lda_project_predict requires non-empty X and projection matrices");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dX = upload(X, (size_t)w * p);
    const double* dR = upload(R, (size_t)p * k);
    const double* dL = upload(linear, (size_t)n_classes * k);
    double* dc = upload(constants, n_classes);
    const double* doff = offset ? upload(offset, k) : nullptr;
    double* dS = scores ? ctx.arena.alloc_n<double>((size_t)w * n_classes) : nullptr;
    int* dlab = ctx.arena.alloc_n<int>(w);
    lda_project_scores_device(dX, w, p, dR, p, k, doff, dL, n_classes, dc, n_classes, dlab, dS);
    download(labels, dlab, w);
    if (scores) download(scores, dS, (size_t)w * n_classes);
    ctx.sync();
  });
}

int fpls_bf16x3_gemm(const double* A, int M, int K, const double* B, int N, double* C, char* err,
                     size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(M > 0 && N > 0 && K > 0, "bf16x3_gemm: dimensions must be positive");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dA = upload(A, (size_t)M * K);
    const double* dB = upload(B, (size_t)K * N);
    double* dC = ctx.arena.alloc_n<double>((size_t)M * N);
    dzero(ctx.d_status + 16, sizeof(int));
    split_gemm_test(dA, dB, M, N, K, dC);
    download(C, dC, (size_t)M * N);
    int e = 0;
    d2h(&e, ctx.d_status + 16, sizeof(int));
    ctx.sync();
    if (e) throw Error(FPLS_ERR_CUDA, "tensor-core pipeline wait timed out");
  });
}

int fpls_int8_gram(const void* X, int x_is_float32, int n, int p, const double* mean, int slices, double* K,
                   char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && X && K, "int8_gram: empty matrix");
    Context& ctx = Context::get();
    ctx.begin_call();
    const size_t np = (size_t)n * p;
    const double* d64 = x_is_float32 ? nullptr : upload(static_cast<const double*>(X), np);
    const float* d32 = x_is_float32 ? upload(static_cast<const float*>(X), np) : nullptr;
    const double* dm = mean ? upload(mean, p) : nullptr;
    double* dK = ctx.arena.alloc_n<double>((size_t)n * n);
    dzero(ctx.d_status + 16, sizeof(int));
    OzakiPlanes pl = ozaki_split_rows(d64, d32, n, p, dm, slices);
    ozaki_gram(pl, dK, n);
    download(K, dK, (size_t)n * n);
    int e = 0;
    d2h(&e, ctx.d_status + 16, sizeof(int));
    ctx.sync();
    if (e) throw Error(FPLS_ERR_CUDA, "tensor-core pipeline wait timed out");
  });
}

int fpls_int8_emulated_gemm(const double* A, int M, int K, const double* B, int N, int slices, double* C,
                            char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(M > 0 && N > 0 && K > 0, "int8_emulated_gemm: dimensions must be positive");
    Context& ctx = Context::get();
    ctx.begin_call();
    // Rows of A are K-contiguous in A^T (K x M, column-major).
    std::vector<double> At((size_t)K * M);
    for (int k = 0; k < K; ++k)
      for (int m = 0; m < M; ++m) At[k + (size_t)m * K] = A[m + (size_t)k * M];
    const double* dAt = upload(At.data(), At.size());
    const double* dB = upload(B, (size_t)K * N);
    double* dC = ctx.arena.alloc_n<double>((size_t)M * N);
    dzero(ctx.d_status + 16, sizeof(int));
    OzakiPlanes pa = ozaki_alloc(M, K, slices);
    OzakiPlanes pb = ozaki_alloc(N, K, slices);
    ozaki_split(dAt, K, pa);
    ozaki_split(dB, K, pb);
    ozaki_gemm(pa, pb, dC, M);
    download(C, dC, (size_t)M * N);
    int e = 0;
    d2h(&e, ctx.d_status + 16, sizeof(int));
    ctx.sync();
    if (e) throw Error(FPLS_ERR_CUDA, "tensor-core pipeline wait timed out");
  });
}

// X of a CV call on the device: the caller's matrix when resident, else an
// arena buffer that the driver fills from the host matrix.
struct CvX {
  const double* x64 = nullptr;
  const float* x32 = nullptr;
  const void* host = nullptr;
};

static CvX cv_x(const void* X, int x_is_float32, bool x_on_device, int n, int p) {
  Context& ctx = Context::get();
  CvX c;
  const size_t np = (size_t)n * p;
  c.host = x_on_device ? nullptr : X;
  if (x_is_float32) c.x32 = x_on_device ? static_cast<const float*>(X) : ctx.arena.alloc_n<float>(np);
  else c.x64 = x_on_device ? static_cast<const double*>(X) : ctx.arena.alloc_n<double>(np);
  return c;
}

static CvGridOptions cv_options(int scaling, int precision, int batched) {
  FPLS_REQUIRE(precision == FPLS_PREC_FP64 || precision == FPLS_PREC_BF16X3 || precision == FPLS_PREC_BF16X6 ||
                   precision == FPLS_PREC_INT8,
               "unknown precision");
  CvGridOptions opt;
  opt.scaling = scaling;
  opt.precision = precision;
  opt.batched = batched != 0;
  if (const char* e = std::getenv("FASTPLS_FAST_INC_ITERS")) {
    char* endp = nullptr;
    long v = std::strtol(e, &endp, 10);
    if (endp != e) opt.power_iters = static_cast<int>(std::min(6L, std::max(1L, v)));
  }
  return opt;
}

// prep: the X-side work already enqueued by the caller (batched grids), or null.
static void run_cv_grid(const CvFitSet& fs, const CvX& x, const int* y, const int* ncomp, int L,
                        const CvGridOptions& opt, CvGridResult& res, CvPreparedX* prep = nullptr) {
  Context& ctx = Context::get();
  // (the error flag of the tensor-core kernels was cleared by begin_call; a
  // flag raised by the X-side work enqueued before this point must survive)
  cv_grid_classify(fs, x.x64, x.x32, y, ncomp, L, opt, res, prep ? nullptr : x.host, prep);
  int e = 0;
  d2h(&e, ctx.d_status + 16, sizeof(int));
  ctx.sync();
  if (e) throw Error(FPLS_ERR_CUDA, "tensor-core pipeline wait timed out");
}

static void cv_predict_impl(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                            const int* fold, int kfold, const int* ncomp, int L, int method, int scaling,
                            int seed, int precision, int batched, int* class_pred, int* status,
                            double* class_score) {
  {
    FPLS_REQUIRE(n >= 2 && p > 0, "Xdata must contain at least two samples");
    FPLS_REQUIRE(n_classes >= 1, "n_classes must be >= 1");
    FPLS_REQUIRE(method == 3 || method == 2, "the GPU CV grid runs method 3 (simpls_fast)");
    FPLS_REQUIRE(kfold >= 1 && L >= 1, "kfold and ncomp must be >= 1");
    Context& ctx = Context::get();
    ctx.begin_call();
    CvFitSet fs;
    fs.n = n; fs.p = p; fs.m = n_classes; fs.F = kfold; fs.G = 1;
    fs.train.assign((size_t)kfold * n, 0);
    fs.test.assign((size_t)kfold * n, 0);
    fs.group.assign(kfold, 0);
    fs.seeds.resize(kfold);
    for (int f = 0; f < kfold; ++f) {
      fs.seeds[f] = static_cast<unsigned>(seed + f);
      for (int i = 0; i < n; ++i) {
        FPLS_REQUIRE(fold[i] >= 0 && fold[i] < kfold, "fold ids must be in 0..kfold-1");
        (fold[i] == f ? fs.test : fs.train)[(size_t)f * n + i] = 1;
      }
    }
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, c);
    CvGridResult res;
    CvGridOptions opt = cv_options(scaling, precision, batched);
    opt.want_scores = class_score != nullptr;
    run_cv_grid(fs, cv_x(X, x_is_float32, false, n, p), y, nc.data(), L, opt, res);
    download(class_pred, res.d_pred, (size_t)n * L);
    if (class_score) download(class_score, res.d_score, (size_t)n * L * n_classes);
    ctx.sync();
    if (status) std::copy(res.status.begin(), res.status.end(), status);
  }
}

int fpls_cv_predict(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                    const int* fold, int kfold, const int* ncomp, int L, int method, int scaling,
                    int seed, int precision, int batched, int* class_pred, int* status,
                    char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    cv_predict_impl(X, x_is_float32, n, p, y, n_classes, fold, kfold, ncomp, L, method, scaling, seed, precision,
                    batched, class_pred, status, nullptr);
  });
}

int fpls_cv_predict_scores(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                           const int* fold, int kfold, const int* ncomp, int L, int method, int scaling,
                           int seed, int precision, int batched, int* class_pred, int* status,
                           double* class_score, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(class_score != nullptr, "class_score must be set");
    cv_predict_impl(X, x_is_float32, n, p, y, n_classes, fold, kfold, ncomp, L, method, scaling, seed, precision,
                    batched, class_pred, status, class_score);
  });
}

// One double CV over the outer folds in outer_ids (all of them, in order, when
// outer_ids is null).  Slot s of the batched grid runs outer fold ids[s]: its
// inner fits are s*Ki .. s*Ki + Ki-1, its refit S*Ki + s, and every output is
// written at the outer fold's own index, so the outputs of disjoint fold lists
// are disjoint and the union of their calls equals one call over all folds.
static void double_cv_impl(const void* X, int x_is_float32, bool x_on_device, int n, int p,
                           const int* y, int n_classes, const int* outer_fold, int kfold_outer,
                           const int* inner_fold, int kfold_inner, const int* outer_ids, int n_ids,
                           const int* ncomp, int L, int scaling, int seed, int run, int precision,
                           int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                           int* inner_pred, int* fit_status, double* inner_score = nullptr,
                           double* outer_score = nullptr) {
  {
    FPLS_REQUIRE(n >= 2 && p > 0, "Xdata must contain at least two samples");
    FPLS_REQUIRE(kfold_outer >= 1 && kfold_inner >= 1 && L >= 1, "fold counts and ncomp must be >= 1");
    const int Ko = kfold_outer, Ki = kfold_inner;
    std::vector<int> ids;
    if (outer_ids) {
      FPLS_REQUIRE(n_ids >= 1 && n_ids <= Ko, "outer fold list must hold 1..kfold_outer ids");
      std::vector<uint8_t> seen(Ko, 0);
      for (int s = 0; s < n_ids; ++s) {
        const int o = outer_ids[s];
        FPLS_REQUIRE(o >= 0 && o < Ko, "outer fold ids must be in 0..kfold_outer-1");
        FPLS_REQUIRE(!seen[o], "outer fold list holds a fold twice");
        seen[o] = 1;
        ids.push_back(o);
      }
    } else {
      for (int o = 0; o < Ko; ++o) ids.push_back(o);
    }
    const int S = static_cast<int>(ids.size());
    Context& ctx = Context::get();
    ctx.begin_call();
    PhaseTimer pt("double CV call");
    std::vector<int> nc(ncomp, ncomp + L);
    for (int& c : nc) c = std::max(1, c);
    CvFitSet fs;
    fs.n = n; fs.p = p; fs.m = n_classes; fs.F = S * Ki + S; fs.G = S + 1;
    std::vector<int> outer_classes(S, 0), fallback(S, 1);
    const int m = n_classes;
    FPLS_REQUIRE(m >= 1, "n_classes must be >= 1");
    for (int i = 0; i < n; ++i)
      FPLS_REQUIRE(y[i] >= 1 && y[i] <= m, "labels must be in 1..n_classes");
    // The X-side work of the grid (upload, column means, BF16 planes, row Gram)
    // does not depend on the folds: enqueued first, it runs on the GPU while
    // the fold set-up below runs on the host.
    CvGridOptions opt = cv_options(scaling, precision, batched);
    opt.want_scores = inner_score != nullptr || outer_score != nullptr;
    const CvX cx = cv_x(X, x_is_float32, x_on_device, n, p);
    std::unique_ptr<CvPreparedX> prep;
    if (opt.batched && opt.scaling != 2 && fs.p > 5)
      prep = cv_prepare_x(cx.x64, cx.x32, n, p, m, *std::max_element(nc.begin(), nc.end()), opt, cx.host);
    pt.mark("X preparation (enqueue)");
    fs.train.assign((size_t)fs.F * n, 0);
    fs.test.assign((size_t)fs.F * n, 0);
    fs.group.assign(fs.F, 0);
    fs.seeds.resize(fs.F);
    // Slot of every row: s when the row belongs to outer fold ids[s], else -1.
    std::vector<int> slot_of_fold(Ko, -1), row_slot(n, -1);
    for (int s = 0; s < S; ++s) slot_of_fold[ids[s]] = s;
    for (int i = 0; i < n; ++i)
      if (outer_fold[i] >= 0 && outer_fold[i] < Ko) row_slot[i] = slot_of_fold[outer_fold[i]];
    // Fold masks and training-row class counts from per-fold histograms: the
    // rows outside outer fold o, split by inner fold id and class, give every
    // inner fit's counts by subtraction (no pass per fit over the masks).
    fs.train_class_counts.assign((size_t)fs.F * m, 0);
    fs.n_train.assign(fs.F, 0);
    fs.n_test.assign(fs.F, 0);
    std::vector<uint8_t> keep(n);
    std::vector<int> outer_cnt(m), inner_cnt((size_t)Ki * m);
    for (int s = 0; s < S; ++s) {
      const int o = ids[s];
      const int* inner_o = inner_fold + (size_t)o * n;
      std::fill(outer_cnt.begin(), outer_cnt.end(), 0);
      std::fill(inner_cnt.begin(), inner_cnt.end(), 0);
      for (int i = 0; i < n; ++i) {
        keep[i] = outer_fold[i] != o;
        if (keep[i]) {
          ++outer_cnt[y[i] - 1];
          const int fi = inner_o[i];
          if (fi >= 0 && fi < Ki) ++inner_cnt[(size_t)fi * m + (y[i] - 1)];
        }
      }
      int best = 0;
      for (int c = 0; c < m; ++c) {
        if (outer_cnt[c] > 0) outer_classes[s]++;
        if (outer_cnt[c] > outer_cnt[best]) best = c;
      }
      fallback[s] = best + 1;
      const bool skip = outer_classes[s] < 2;  // pls.double.cv's single-class fallback
      for (int i0 = 0; i0 < Ki; ++i0) {
        const int f = s * Ki + i0;
        fs.group[f] = s;
        fs.seeds[f] = static_cast<unsigned>(seed + 1000 * run + (o + 1) + i0);
        if (skip) continue;
        uint8_t* tr = fs.train.data() + (size_t)f * n;
        uint8_t* te = fs.test.data() + (size_t)f * n;
        for (int i = 0; i < n; ++i) {
          const uint8_t in = inner_o[i] == i0;
          tr[i] = keep[i] & static_cast<uint8_t>(!in);
          te[i] = keep[i] & in;
        }
        int ntr = 0, nte = 0;
        for (int c = 0; c < m; ++c) {
          const int t = inner_cnt[(size_t)i0 * m + c];
          fs.train_class_counts[(size_t)f * m + c] = outer_cnt[c] - t;
          ntr += outer_cnt[c] - t;
          nte += t;
        }
        fs.n_train[f] = ntr;
        fs.n_test[f] = nte;
      }
      const int f = S * Ki + s;
      fs.group[f] = S;
      fs.seeds[f] = static_cast<unsigned>(seed + 2000 * run + (o + 1));
      if (skip) continue;
      uint8_t* tr = fs.train.data() + (size_t)f * n;
      uint8_t* te = fs.test.data() + (size_t)f * n;
      int ntr = 0;
      for (int i = 0; i < n; ++i) {
        tr[i] = keep[i];
        te[i] = !keep[i];
        ntr += keep[i];
      }
      for (int c = 0; c < m; ++c) fs.train_class_counts[(size_t)f * m + c] = outer_cnt[c];
      fs.n_train[f] = ntr;
      fs.n_test[f] = n - ntr;
    }
    CvGridResult res;
    pt.mark("folds (host)");
    run_cv_grid(fs, cx, y, nc.data(), L, opt, res, prep.get());
    pt.mark("grid");
    // Inner accuracy per (outer fold, ncomp) on the device; the chosen ncomp is the
    // first maximum (.cv_best_index); only counts and the outer predictions return.
    const int* d_y = upload(y, n);
    const int* d_slot = upload(row_slot.data(), n);
    // Accuracies, the chosen ncomp and the outer predictions on the device;
    // one download and one synchronisation at the end.
    const long long* d_cnt = cv_prediction_counts_device(res.d_pred, S, L, n, d_y, d_slot);
    std::vector<int> fb(S, 0);
    for (int s = 0; s < S; ++s) fb[s] = outer_classes[s] < 2 ? fallback[s] : 0;
    int* d_fb = upload(fb.data(), S);
    const int* d_ids = upload(ids.data(), S);
    const int* d_nc = upload(nc.data(), L);
    double* d_acc = ctx.arena.alloc_n<double>((size_t)Ko * L);
    int* d_best = ctx.arena.alloc_n<int>(S);
    int* d_bcomp = ctx.arena.alloc_n<int>(Ko);
    select_ncomp_kernel<<<ceil_div(S, 128), 128, 0, ctx.stream>>>(d_cnt, S, L, d_ids, Ko, d_nc, d_fb,
                                                                  *std::min_element(nc.begin(), nc.end()), d_acc,
                                                                  d_best, d_bcomp);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    int* d_out = ctx.arena.alloc_n<int>(n);
    gather_outer_pred_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(res.d_pred, d_slot, d_best, d_fb, S, L, n, d_out); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    // the accuracies, chosen ncomp and outer predictions through page-locked
    // staging: asynchronous copies, one synchronisation below
    const size_t b_acc = (size_t)Ko * L * sizeof(double), b_bc = (size_t)Ko * sizeof(int), b_out = (size_t)n * sizeof(int);
    char* stg = ctx.host_staging(b_acc + b_bc + b_out);
    d2h(stg, d_acc, b_acc);
    d2h(stg + b_acc, d_bcomp, b_bc);
    d2h(stg + b_acc + b_bc, d_out, b_out);
    double* d_oscore = nullptr;
    if (outer_score) {
      d_oscore = ctx.arena.alloc_n<double>((size_t)n * m);
      gather_outer_score_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(res.d_score, d_slot, d_best, d_fb, S, L,
                                                                          n, m, d_oscore);
      ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
    std::vector<double> oscore_all;
    if (outer_score && outer_ids) {
      oscore_all.resize((size_t)n * m);
      download(oscore_all.data(), d_oscore, (size_t)n * m);
    } else if (outer_score) {
      download(outer_score, d_oscore, (size_t)n * m);
    }
    if (inner_score)
      for (int s = 0; s < S; ++s)
        download(inner_score + (size_t)ids[s] * L * n * m, res.d_score + (size_t)s * L * n * m, (size_t)L * n * m);
    std::vector<int> pred_all;
    if (outer_ids) {
      if (inner_pred)
        for (int s = 0; s < S; ++s)
          download(inner_pred + (size_t)ids[s] * L * n, res.d_pred + (size_t)s * L * n, (size_t)L * n);
    } else {
      if (inner_pred) download(inner_pred, res.d_pred, (size_t)Ko * L * n);
    }
    pt.mark("ncomp + outer");
    ctx.sync();
    std::vector<double> acc_all((size_t)Ko * L);
    std::vector<int> bcomp_all(Ko);
    std::memcpy(acc_all.data(), stg, b_acc);
    std::memcpy(bcomp_all.data(), stg + b_acc, b_bc);
    if (outer_ids) {
      pred_all.resize(n);
      std::memcpy(pred_all.data(), stg + b_acc + b_bc, b_out);
    } else if (outer_pred) {
      std::memcpy(outer_pred, stg + b_acc + b_bc, b_out);
    }
    for (int s = 0; s < S; ++s) {
      const int o = ids[s];
      if (best_comp) best_comp[o] = bcomp_all[o];
      if (inner_accuracy)
        for (int l = 0; l < L; ++l) inner_accuracy[o + (size_t)l * Ko] = acc_all[o + (size_t)l * Ko];
    }
    if (outer_ids)
      for (int i = 0; i < n; ++i)
        if (row_slot[i] >= 0) {
          outer_pred[i] = pred_all[i];
          if (outer_score)
            for (int j = 0; j < m; ++j) outer_score[(size_t)i * m + j] = oscore_all[(size_t)i * m + j];
        }
    if (fit_status)
      for (int s = 0; s < S; ++s) {
        for (int i0 = 0; i0 < Ki; ++i0) fit_status[(size_t)ids[s] * Ki + i0] = res.status[(size_t)s * Ki + i0];
        fit_status[(size_t)Ko * Ki + ids[s]] = res.status[(size_t)S * Ki + s];
      }
    }
}

}  // extern "C"

namespace {

// One double CV with the tuned configuration of its shape in force.  When
// autotuning is on and the shape (device, n, p, fits, ncomp slices, largest
// ncomp, classes, precision, scaling) has not been tuned, the candidates are
// timed first on this call's own inputs: every candidate runs the whole grid
// once to warm up and twice timed (the faster counts), and only candidates
// whose chosen ncomp, outer predictions and inner accuracies equal the
// default configuration's are eligible.  Only the batched row-space path has
// knobs; other grids run as they are.
template <typename Run>
void run_double_cv_tuned(int n, int p, int n_classes, int kfold_outer, int kfold_inner, const int* ncomp, int L,
                         int scaling, int precision, int batched, Run run) {
  Context& ctx = Context::get();
  const int K = std::max(1, max_of(ncomp, L));
  const bool eligible = batched && scaling != 2 && p > 5 && dual_engine_applies(n, p, n_classes, K);
  TuneKey key{ctx.device, n, p, kfold_outer * (kfold_inner + 1), L, K, n_classes, precision, scaling};
  if (eligible && autotune_enabled() && !tuned_lookup(key)) {
    struct Out {
      std::vector<int> best, pred;
      std::vector<double> acc;
      double ms = 0.0;
    };
    auto measure = [&](const TuneConfig& c, Out& o) {
      TuneScope scope(c);
      o.best.assign(kfold_outer, 0);
      o.pred.assign(n, 0);
      o.acc.assign((size_t)kfold_outer * L, 0.0);
      double best_ms = 1e300;
      for (int r = 0; r < 3; ++r) {
        run(o.best.data(), o.acc.data(), o.pred.data());
        ctx.end_call();
        if (r > 0) best_ms = std::min(best_ms, ctx.last_call_ms);
      }
      o.ms = best_ms;
    };
    std::vector<TuneConfig> cands{TuneConfig{}};   // the default first: the equality gate's reference
    const std::vector<int> tiles = precision == 1 ? std::vector<int>{128, 64} : std::vector<int>{0};
    const std::vector<int> layouts = n <= 4096 ? std::vector<int>{0, 1} : std::vector<int>{1};
    const std::vector<int> merges = n_classes <= 6 ? std::vector<int>{1, 0} : std::vector<int>{1};
    // The digit-slice count of the K products sets their accuracy, so it stays
    // the precision mode's own and is not tuned: with the INT8 grid at 5
    // instead of 6 slices the labels still matched (the gate) while the class
    // scores moved from 6.2e-7 to 6.3e-5 of the FP64 grid's.
    const std::vector<int> slices{0};
    for (int t : tiles)
      for (int l : layouts)
        for (int mg : merges)
          for (int sl : slices) {
            TuneConfig c;
            c.gram_tile = t;
            c.step_layout = l;
            c.merge = mg;
            c.ozaki_slices = sl;
            cands.push_back(c);
          }
    Out ref;
    measure(cands[0], ref);   // the default configuration, the reference of the equality gate
    TuneConfig chosen = cands[0];
    double chosen_ms = ref.ms;
    std::ostringstream rep;
    rep << "[{\"config\": " << cands[0].str() << ", \"ms\": " << ref.ms << ", \"same_results\": true}";
    for (size_t i = 1; i < cands.size(); ++i) {
      Out o;
      measure(cands[i], o);
      const bool same = o.best == ref.best && o.pred == ref.pred && o.acc == ref.acc;
      rep << ", {\"config\": " << cands[i].str() << ", \"ms\": " << o.ms << ", \"same_results\": "
          << (same ? "true" : "false") << "}";
      if (same && o.ms < chosen_ms) {
        chosen = cands[i];
        chosen_ms = o.ms;
      }
    }
    rep << "]";
    tuned_store(key, chosen, rep.str());
  }
  const TuneConfig* t = autotune_enabled() ? tuned_lookup(key) : nullptr;
  TuneScope scope(t ? *t : TuneConfig{});
  run(nullptr, nullptr, nullptr);
}

}  // namespace

extern "C" {

int fpls_set_autotune(int on, char* err, size_t errlen) {
  return guarded(err, errlen, [&] { set_autotune(on != 0); });
}

int fpls_autotune_report(char* buf, size_t len, size_t* needed, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    const std::string r = tune_report();
    if (needed) *needed = r.size() + 1;
    if (buf && len) {
      const size_t k = std::min(len - 1, r.size());
      std::memcpy(buf, r.data(), k);
      buf[k] = '\0';
    }
  });
}

int fpls_double_cv(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                   const int* outer_fold, int kfold_outer, const int* inner_fold, int kfold_inner,
                   const int* ncomp, int L, int scaling, int seed, int run, int precision,
                   int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                   int* inner_pred, int* fit_status, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    run_double_cv_tuned(n, p, n_classes, kfold_outer, kfold_inner, ncomp, L, scaling, precision, batched,
                        [&](int* tb, double* ta, int* tp) {
                          const bool probe = tb != nullptr;
                          double_cv_impl(X, x_is_float32, false, n, p, y, n_classes, outer_fold, kfold_outer,
                                         inner_fold, kfold_inner, nullptr, 0, ncomp, L, scaling, seed, run,
                                         precision, batched, probe ? tb : best_comp, probe ? ta : inner_accuracy,
                                         probe ? tp : outer_pred, probe ? nullptr : inner_pred,
                                         probe ? nullptr : fit_status);
                        });
  });
}

int fpls_double_cv_scores(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                          const int* outer_fold, int kfold_outer, const int* inner_fold, int kfold_inner,
                          const int* ncomp, int L, int scaling, int seed, int run, int precision,
                          int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                          int* inner_pred, int* fit_status, double* inner_score, double* outer_score,
                          char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(inner_score || outer_score, "double_cv_scores: no score output requested");
    // the configuration tuned for this shape, if any (no tuning from here)
    Context& ctx = Context::get();
    const TuneKey key{ctx.device, n, p, kfold_outer * (kfold_inner + 1), L, std::max(1, max_of(ncomp, L)),
                      n_classes, precision, scaling};
    const TuneConfig* t = autotune_enabled() ? tuned_lookup(key) : nullptr;
    TuneScope scope(t ? *t : TuneConfig{});
    double_cv_impl(X, x_is_float32, false, n, p, y, n_classes, outer_fold, kfold_outer, inner_fold,
                   kfold_inner, nullptr, 0, ncomp, L, scaling, seed, run, precision, batched, best_comp,
                   inner_accuracy, outer_pred, inner_pred, fit_status, inner_score, outer_score);
  });
}

int fpls_double_cv_outer_subset(const void* X, int x_is_float32, int n, int p, const int* y,
                                int n_classes, const int* outer_fold, int kfold_outer,
                                const int* inner_fold, int kfold_inner, const int* outer_ids,
                                int n_outer_ids, const int* ncomp, int L, int scaling, int seed, int run,
                                int precision, int batched, int* best_comp, double* inner_accuracy,
                                int* outer_pred, int* inner_pred, int* fit_status, char* err,
                                size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(outer_ids, "outer fold list is null");
    double_cv_impl(X, x_is_float32, false, n, p, y, n_classes, outer_fold, kfold_outer, inner_fold,
                   kfold_inner, outer_ids, n_outer_ids, ncomp, L, scaling, seed, run, precision, batched,
                   best_comp, inner_accuracy, outer_pred, inner_pred, fit_status);
  });
}

}  // extern "C"

namespace {

// A new resident matrix (n x p, FP32 or FP64), filled from X when X is set.
int register_resident(const void* X, int x_is_float32, int n, int p) {
  Context& ctx = Context::get();
  ResidentX r;
  r.n = n;
  r.p = p;
  r.f32 = x_is_float32 != 0;
  const size_t bytes = (size_t)n * p * (r.f32 ? sizeof(float) : sizeof(double));
  FPLS_CUDA(cudaMalloc(&r.ptr, bytes));
  if (X) FPLS_CUDA(cudaMemcpyAsync(r.ptr, X, bytes, cudaMemcpyDefault, ctx.stream));
  else FPLS_CUDA(cudaMemsetAsync(r.ptr, 0, bytes, ctx.stream));
  ctx.sync();
  int h = -1;
  for (size_t i = 0; i < ctx.resident.size(); ++i)
    if (!ctx.resident[i].ptr) { h = static_cast<int>(i); break; }
  if (h < 0) { h = static_cast<int>(ctx.resident.size()); ctx.resident.push_back(r); }
  else ctx.resident[h] = r;
  return h;
}

}  // namespace

extern "C" {

int fpls_x_upload(const void* X, int x_is_float32, int n, int p, int* handle, char* err,
                  size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && X && handle, "x_upload: empty matrix");
    Context::get().begin_call();
    *handle = register_resident(X, x_is_float32, n, p);
  });
}

int fpls_x_alloc(int n, int p, int x_is_float32, int* handle, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && handle, "x_alloc: empty matrix");
    Context::get().begin_call();
    *handle = register_resident(nullptr, x_is_float32, n, p);
  });
}

int fpls_x_device_pointer(int handle, void** ptr, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    FPLS_REQUIRE(ptr && handle >= 0 && handle < static_cast<int>(ctx.resident.size()) && ctx.resident[handle].ptr,
                 "x_device_pointer: unknown handle");
    *ptr = ctx.resident[handle].ptr;
  });
}

int fpls_x_download(int handle, void* out, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    FPLS_REQUIRE(out && handle >= 0 && handle < static_cast<int>(ctx.resident.size()) && ctx.resident[handle].ptr,
                 "x_download: unknown handle");
    const ResidentX& r = ctx.resident[handle];
    const size_t bytes = (size_t)r.n * r.p * (r.f32 ? sizeof(float) : sizeof(double));
    FPLS_CUDA(cudaMemcpyAsync(out, r.ptr, bytes, cudaMemcpyDefault, ctx.stream));
    ctx.sync();
  });
}

int fpls_x_free(int handle, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    FPLS_REQUIRE(handle >= 0 && handle < static_cast<int>(ctx.resident.size()) &&
                     ctx.resident[handle].ptr, "x_free: unknown handle");
    FPLS_CUDA(cudaFree(ctx.resident[handle].ptr));
    ctx.resident[handle] = ResidentX();
  });
}

int fpls_set_precision(int precision, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(precision == FPLS_PREC_FP64 || precision == FPLS_PREC_BF16X3 ||
                     precision == FPLS_PREC_BF16X6,
                 "precision must be FPLS_PREC_FP64 (0), FPLS_PREC_BF16X3 (1) or FPLS_PREC_BF16X6 (2)");
    Context::get().precision = precision;
  });
}

int fpls_get_precision(void) { return Context::get().precision; }

int fpls_host_register(void* ptr, size_t bytes, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(ptr && bytes > 0, "host_register: empty buffer");
    Context::get();
    FPLS_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  });
}

int fpls_host_unregister(void* ptr, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(ptr, "host_unregister: null buffer");
    Context::get();
    FPLS_CUDA(cudaHostUnregister(ptr));
  });
}

int fpls_double_cv_resident(int handle, const int* y, int n_classes, const int* outer_fold,
                            int kfold_outer, const int* inner_fold, int kfold_inner,
                            const int* ncomp, int L, int scaling, int seed, int run, int precision,
                            int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                            int* inner_pred, int* fit_status, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    FPLS_REQUIRE(handle >= 0 && handle < static_cast<int>(ctx.resident.size()) &&
                     ctx.resident[handle].ptr, "double_cv_resident: unknown handle");
    const ResidentX r = ctx.resident[handle];
    run_double_cv_tuned(r.n, r.p, n_classes, kfold_outer, kfold_inner, ncomp, L, scaling, precision, batched,
                        [&](int* tb, double* ta, int* tp) {
                          const bool probe = tb != nullptr;
                          double_cv_impl(r.ptr, r.f32 ? 1 : 0, true, r.n, r.p, y, n_classes, outer_fold,
                                         kfold_outer, inner_fold, kfold_inner, nullptr, 0, ncomp, L, scaling, seed,
                                         run, precision, batched, probe ? tb : best_comp,
                                         probe ? ta : inner_accuracy, probe ? tp : outer_pred,
                                         probe ? nullptr : inner_pred, probe ? nullptr : fit_status);
                        });
  });
}

int fpls_double_cv_resident_outer_subset(int handle, const int* y, int n_classes, const int* outer_fold,
                                         int kfold_outer, const int* inner_fold, int kfold_inner,
                                         const int* outer_ids, int n_outer_ids, const int* ncomp, int L,
                                         int scaling, int seed, int run, int precision, int batched,
                                         int* best_comp, double* inner_accuracy, int* outer_pred,
                                         int* inner_pred, int* fit_status, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    FPLS_REQUIRE(outer_ids, "outer fold list is null");
    Context& ctx = Context::get();
    FPLS_REQUIRE(handle >= 0 && handle < static_cast<int>(ctx.resident.size()) &&
                     ctx.resident[handle].ptr, "double_cv_resident: unknown handle");
    const ResidentX r = ctx.resident[handle];
    double_cv_impl(r.ptr, r.f32 ? 1 : 0, true, r.n, r.p, y, n_classes, outer_fold, kfold_outer,
                   inner_fold, kfold_inner, outer_ids, n_outer_ids, ncomp, L, scaling, seed, run,
                   precision, batched, best_comp, inner_accuracy, outer_pred, inner_pred, fit_status);
  });
}

long long fpls_launch_count(void) { return launch_count(); }

double fpls_last_call_ms(void) {
  try {
    return Context::get().last_call_ms;
  } catch (...) {
    return 0.0;
  }
}

int fpls_profile(int enable, double* gemm_ms, long long* gemm_launches, double* gemm_bytes,
                 char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    if (enable) {
      for (auto& c : ctx.prof_classes)
        for (cudaEvent_t e : c.events) cudaEventDestroy(e);
      ctx.prof_classes.clear();
      ctx.profile = true;
      return;
    }
    ctx.profile = false;
    ctx.sync();
    double total = 0.0, bytes = 0.0;
    long long launches = 0;
    for (auto& c : ctx.prof_classes) {
      if (c.name.rfind("split_gemm", 0) != 0 && c.name.rfind("gram_bf16x3", 0) != 0) continue;
      for (size_t i = 0; i + 1 < c.events.size(); i += 2) {
        float ms = 0.f;
        FPLS_CUDA(cudaEventElapsedTime(&ms, c.events[i], c.events[i + 1]));
        total += ms;
      }
      launches += static_cast<long long>(c.events.size() / 2);
      bytes += c.bytes;
    }
    if (gemm_ms) *gemm_ms = total;
    if (gemm_launches) *gemm_launches = launches;
    if (gemm_bytes) *gemm_bytes = bytes;
  });
}

int fpls_profile_class(int index, char* name, size_t namelen, double* ms, long long* launches,
                       double* bytes, double* flops, char* err, size_t errlen) {
  return guarded(err, errlen, [&] {
    Context& ctx = Context::get();
    FPLS_REQUIRE(index >= 0 && index < static_cast<int>(ctx.prof_classes.size()),
                 "profile_class: no kernel class with this index");
    const auto& c = ctx.prof_classes[index];
    double total = 0.0;
    for (size_t i = 0; i + 1 < c.events.size(); i += 2) {
      float t = 0.f;
      FPLS_CUDA(cudaEventElapsedTime(&t, c.events[i], c.events[i + 1]));
      total += t;
    }
    if (name && namelen) {
      std::strncpy(name, c.name.c_str(), namelen - 1);
      name[namelen - 1] = '\0';
    }
    if (ms) *ms = total;
    if (launches) *launches = static_cast<long long>(c.events.size() / 2);
    if (bytes) *bytes = c.bytes;
    if (flops) *flops = c.flops;
  });
}

}  // extern "C"
