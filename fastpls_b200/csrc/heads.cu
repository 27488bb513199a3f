#include "xop_split.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "heads.cuh"
#include "linalg_small.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace fpls {
namespace {

__global__ void argmax_kernel(const double* __restrict__ S, int w, int C, const double* bias,
                              int* labels) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  int best = 0;
  double bv = S[i] + (bias ? bias[0] : 0.0);
  for (int c = 1; c < C; ++c) {
    const double v = S[i + (size_t)c * w] + (bias ? bias[c] : 0.0);
    if (v > bv) { bv = v; best = c; }
  }
  labels[i] = best + 1;
}

// Insertion into a descending top list: strict '>' keeps the earlier class on
// ties (candidate_insert_top, src/fastPLS.cpp:1249-1267).
__global__ void topk_kernel(const double* __restrict__ S, int w, int C, const double* bias,
                            int top_k, int* idx, double* score) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  double vals[32];
  int ids[32];
  const int k = min(top_k, 32);
  for (int j = 0; j < k; ++j) { vals[j] = -INFINITY; ids[j] = 0; }
  for (int c = 0; c < C; ++c) {
    const double v = S[i + (size_t)c * w] + (bias ? bias[c] : 0.0);
    for (int j = 0; j < k; ++j) {
      if (v > vals[j]) {
        for (int h = k - 1; h > j; --h) { vals[h] = vals[h - 1]; ids[h] = ids[h - 1]; }
        vals[j] = v;
        ids[j] = c + 1;
        break;
      }
    }
  }
  for (int j = 0; j < k; ++j) {
    idx[i + (size_t)j * w] = ids[j];
    score[i + (size_t)j * w] = vals[j];
  }
}

// Class sums of the score columns (T n x kmax into sums C x kmax) in a fixed
// order: warp w takes (class c, column j) = (w % C, w / C) and walks that
// class's rows in class-sorted order perm[off[c] .. off[c+1]) lane-strided,
// then a fixed shuffle tree -- the same rounding on every run (no atomics).
__global__ void class_sums_sorted_kernel(const double* __restrict__ T, int n, int kmax,
                                         const int* __restrict__ perm, const int* __restrict__ off, int C,
                                         double* __restrict__ sums) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= (long long)C * kmax) return;  // whole warps leave together
  const int c = static_cast<int>(w % C), j = static_cast<int>(w / C);
  const double* tc = T + (size_t)j * n;
  double acc = 0.0;
  for (int i = off[c] + lane; i < off[c + 1]; i += 32) acc += tc[perm[i]];
  acc = warp_sum(acc);
  if (lane == 0) sums[c + (size_t)j * C] = acc;
}

__global__ void means_from_sums_kernel(double* M, int C, int k, const double* counts,
                                       double* Mw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C * k) return;
  const int c = t % C;
  const double m = M[t] / counts[c];
  M[t] = m;
  Mw[t] = m * counts[c];
}

// pooled = symmatu(P) / df   (upper triangle mirrored)
__global__ void symm_upper_scale_kernel(double* P, int k, double inv_df) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k * k) return;
  const int i = t % k, j = t / k;
  if (i <= j) {
    const double v = P[i + (size_t)j * k] * inv_df;
    P[i + (size_t)j * k] = v;
    if (i != j) P[j + (size_t)i * k] = v;
  }
}

// Leading kk x kk block plus lambda I; lambda = ridge * trace/kk (reference ridge rule).
__global__ void ridge_block_kernel(const double* P, int kmax, int kk, double ridge, double* out,
                                   double* lambda_out) {
  __shared__ double scratch[32];
  __shared__ double lam;
  double tr = 0.0;
  for (int i = threadIdx.x; i < kk; i += blockDim.x) tr += P[i + (size_t)i * kmax];
  tr = block_sum(tr, scratch);
  if (threadIdx.x == 0) {
    double scale = tr / static_cast<double>(kk > 0 ? kk : 1);
    if (!isfinite(scale) || scale <= 0.0) scale = 1.0;
    double l = ridge;
    if (!isfinite(l) || l < 0.0) l = 1e-8;
    lam = l * scale;
    *lambda_out = lam;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x) {
    const int i = t % kk, j = t / kk;
    out[t] = P[i + (size_t)j * kmax] + (i == j ? lam : 0.0);
  }
}

__global__ void transpose_block_kernel(const double* A, int rows, int cols, int lda, double* B,
                                       int ldb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * cols) return;
  const int i = t % rows, j = t / rows;
  B[j + (size_t)i * ldb] = A[i + (size_t)j * lda];
}

// constants[c] = -0.5 * means_c . linear_c + log(max(prior_c, DBL_MIN))
__global__ void lda_constants_kernel(const double* M, const double* Lin, int C, int kk, int ldm,
                                     const double* counts, int n, double* constants,
                                     double* priors) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  double d = 0.0;
  for (int j = 0; j < kk; ++j) d += M[c + (size_t)j * ldm] * Lin[c + (size_t)j * ldm];
  const double prior = counts[c] / static_cast<double>(n);
  constants[c] = -0.5 * d + log(fmax(prior, DBL_MIN));
  if (priors) priors[c] = prior;
}

}  // namespace

void lowrank_predict(const double* Xs, int w, int p, const double* R, int kmax, const double* W,
                     int m, const int* ncomp_host, int L, const double* mY, double* T,
                     double* Ypred) {
  xgemm(false, w, kmax, p, Xs, w, R, p, T, w);
  for (int a = 0; a < L; ++a) {
    const int mc = ncomp_host[a];
    double* Ya = Ypred + (size_t)a * w * m;
    gemm(false, false, w, m, mc, 1.0, T, w, W + (size_t)a * kmax * m, kmax, 0.0, Ya, w);
    add_row_vector(Ya, w, m, w, mY);
  }
}

void row_argmax(const double* S, int w, int C, const double* bias, int* labels) {
  if (w <= 0) return;
  argmax_kernel<<<ceil_div(w, 256), 256, 0, Context::get().stream>>>(S, w, C, bias, labels); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void row_topk(const double* S, int w, int C, const double* bias, int top_k, int* idx,
              double* score) {
  FPLS_REQUIRE(top_k >= 1 && top_k <= 32, "top-k supports 1..32 classes per row");
  if (w <= 0) return;
  topk_kernel<<<ceil_div(w, 128), 128, 0, Context::get().stream>>>(S, w, C, bias, top_k, idx, score); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void lda_train_prefix(const double* T, int n, int kmax, const int* y_host, int C,
                      const int* ncomp_host, int L, double ridge, LdaModelsDev out) {
  Context& ctx = Context::get();
  FPLS_REQUIRE(n > 0 && kmax > 0, "lda_train_prefix requires a non-empty score matrix");
  FPLS_REQUIRE(C >= 2, "lda_train_prefix requires at least two classes");
  // class counts and a stable class-sorted row order (host, O(n))
  std::vector<int> off(C + 1, 0), perm(n);
  for (int i = 0; i < n; ++i) {
    const int cls = y_host[i] - 1;
    if (cls < 0 || cls >= C) throw Error(kErrArgument, "lda_train_prefix labels must be encoded as 1..n_classes");
    ++off[cls + 1];
  }
  std::vector<double> hc(C);
  for (int c = 0; c < C; ++c) {
    if (off[c + 1] <= 0) throw Error(kErrArgument, "lda_train_prefix received an empty class");
    hc[c] = off[c + 1];
    off[c + 1] += off[c];
  }
  {
    std::vector<int> cur(off.begin(), off.end() - 1);
    for (int i = 0; i < n; ++i) perm[cur[y_host[i] - 1]++] = i;
  }
  double* M = ctx.arena.alloc_n<double>((size_t)C * kmax);
  double* Mw = ctx.arena.alloc_n<double>((size_t)C * kmax);
  double* counts = ctx.arena.alloc_n<double>(C);
  int* d_perm = ctx.arena.alloc_n<int>(n);
  int* d_off = ctx.arena.alloc_n<int>(C + 1);
  h2d(counts, hc.data(), C * sizeof(double));
  h2d(d_perm, perm.data(), n * sizeof(int));
  h2d(d_off, off.data(), (C + 1) * sizeof(int));
  const long long warps = (long long)C * kmax;
  class_sums_sorted_kernel<<<static_cast<unsigned>((warps + 7) / 8), 256, 0, ctx.stream>>>(T, n, kmax, d_perm,
                                                                                        d_off, C, M);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  means_from_sums_kernel<<<ceil_div(C * kmax, 256), 256, 0, ctx.stream>>>(M, C, kmax, counts, Mw); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  double* P = ctx.arena.alloc_n<double>((size_t)kmax * kmax);
  gemm(true, false, kmax, kmax, n, 1.0, T, n, T, n, 0.0, P, kmax);
  gemm(true, false, kmax, kmax, C, -1.0, M, C, Mw, C, 1.0, P, kmax);
  const double df = std::max(1.0, static_cast<double>(n) - static_cast<double>(C));
  symm_upper_scale_kernel<<<ceil_div(kmax * kmax, 256), 256, 0, ctx.stream>>>(P, kmax, 1.0 / df); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  double* Pk = ctx.arena.alloc_n<double>((size_t)kmax * kmax);
  double* Mt = ctx.arena.alloc_n<double>((size_t)kmax * C);
  double* Xs = ctx.arena.alloc_n<double>((size_t)kmax * C);
  double* lam = ctx.arena.alloc_n<double>(L);
  for (int a = 0; a < L; ++a) {
    const int kk = ncomp_host[a];
    ridge_block_kernel<<<1, 256, 0, ctx.stream>>>(P, kmax, kk, ridge, Pk, lam + a); ::fpls::note_launch();
    transpose_block_kernel<<<ceil_div(C * kk, 256), 256, 0, ctx.stream>>>(M, C, kk, C, Mt, kk); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    spd_solve(kk, Pk, kk, C, Mt, kk, Xs, kk, ctx.d_status + 5);
    double* Ma = out.means + (size_t)a * C * kmax;
    double* La = out.linear + (size_t)a * C * kmax;
    dzero(Ma, (size_t)C * kmax * sizeof(double));
    dzero(La, (size_t)C * kmax * sizeof(double));
    copy_matrix(Ma, C, M, C, C, kk);
    transpose_block_kernel<<<ceil_div(C * kk, 256), 256, 0, ctx.stream>>>(Xs, kk, C, kk, La, C); ::fpls::note_launch();
    lda_constants_kernel<<<ceil_div(C, 128), 128, 0, ctx.stream>>>(
        Ma, La, C, kk, C, counts, n, out.constants + (size_t)a * C, a == 0 ? out.priors : nullptr); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  std::vector<double> hl(L);
  d2h(hl.data(), lam, L * sizeof(double));
  int singular = 0;
  d2h(&singular, ctx.d_status + 5, sizeof(int));
  ctx.sync();
  if (singular) throw Error(kErrNumerical, "LDA pooled covariance is singular");
  for (int a = 0; a < L; ++a) out.lambda[a] = hl[a];
}

}  // namespace fpls
