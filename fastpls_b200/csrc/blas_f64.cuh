// FP64 dense kernels on B200: DMMA (mma.sync m8n8k4 f64) tiled GEMM and
// bandwidth-bound GEMV / column statistics.  All matrices are column-major
// (R / Armadillo layout); pointers are device pointers; work is issued on the
// context stream.  tcgen05 has no f64 kind, so FP64 contractions run on the
// FP64 tensor path (DMMA) or on DFMA.
#pragma once

#include "common.cuh"

namespace fpls {

// C = alpha * op(A) * op(B) + beta * C, op(A): M x K, op(B): K x N.
void gemm(bool transA, bool transB, int M, int N, int K, double alpha,
          const double* A, int lda, const double* B, int ldb, double beta,
          double* C, int ldc);

// K (n x n) = X X^T for X n x p: the upper-triangle tiles by FP64 tensor-core
// MMA, the lower triangle mirrored (K exactly symmetric).
void gram_f64(const double* X, int n, int p, int ldx, double* K, int ldk);

// G (q x q) = S^T S for S p x q (lds): the same upper-tile product, mirrored.
void gram_t_f64(const double* S, int p, int q, int lds, double* G, int ldg);

// y = alpha * op(A) * x + beta * y.  A is rows x cols (lda).
void gemv(bool trans, int rows, int cols, double alpha, const double* A, int lda,
          const double* x, double beta, double* y);

// Column means of X (n x p).  out[p].
void col_mean(const double* X, int n, int p, int ldx, double* out);
void col_mean(const float* X, int n, int p, int ldx, double* out);
// Column standard deviation (n-1) of an already centred X.
void col_sd_centered(const double* X, int n, int p, int ldx, double* out);
// Column sums; sums of squared deviations from mu; out = in / d (sqrt(in / d)
// with root).  The pieces of col_mean / col_sd_centered for row-sharded fits.
void col_sum(const double* X, int n, int p, int ldx, double* out);
void col_sqdev(const double* X, int n, int p, int ldx, const double* mu, double* out);
void div_vec(const double* in, size_t count, double d, bool root, double* out);
// X[:, j] = (X[:, j] - mean[j]) / scale[j]   (mean or scale may be null).
void center_scale(double* X, int n, int p, int ldx, const double* mean, const double* scale);
// dst (n x p, ldd) = src (n x p, lds)
void copy_matrix(double* dst, int ldd, const double* src, int lds, int n, int p);
// X[i, j] += v[j] for all i (row broadcast)
void add_row_vector(double* X, int n, int p, int ldx, const double* v);
// Frobenius-type sums for R2: out[0] = sum((Y - Yp)^2), out[1] = sum((Y - colmean(Y))^2)
void rq_sums(const double* Y, const double* Yp, int n, int m, double* out2, const double* mus = nullptr);
// Row-sharded fits: the column means of Y over all ranks' rows, the TSS
// centre of rq_sums (null when the fit is not sharded).
const double* shard_rq_means(const double* Y, int n, int m);
void fill(double* x, size_t n, double v);
void scale_vec(double* x, size_t n, double a);

}  // namespace fpls
