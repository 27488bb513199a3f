// Small dense FP64 linear algebra on the device (k x k systems, tall-skinny QR,
// symmetric eigen and thin SVD) replacing the LAPACK / cuSOLVER calls of the
// reference (potrf/potrs, geqrf/orgqr, syevd, gesdd).  Column-major, device
// pointers, context stream.  Failures set d_flag (never trap or spin).
#pragma once

#include "common.cuh"

namespace fpls {

// X = G^{-1} B for symmetric G (k x k): Cholesky, falling back to partial
// pivoting LU when G is not numerically positive definite (as arma::solve with
// solve_opts::likely_sympd).  Sets *d_flag = 1 when G is singular.
// If ridge_rel > 0 the system solved is (G + ridge_rel*mean(diag(G)) I).
void spd_solve(int k, const double* G, int ldg, int nrhs, const double* B, int ldb,
               double* X, int ldx, int* d_flag, double ridge_rel = 0.0);

// Thin QR orthonormalisation of Y (rows x cols, rows >= cols) into Q.
// CholeskyQR2 (FP64 Gram + Cholesky); if the Gram is not positive definite it
// falls back to classical Gram-Schmidt with re-orthogonalisation.  The span of
// Q equals that of Householder QR; column signs follow R_jj > 0.
void qr_orthonormalize(int rows, int cols, const double* Y, int ldy, double* Q, int ldq);

// Symmetric eigen-decomposition (cyclic Jacobi), eigenvalues in descending
// order.  G (l x l) is read only; evals[l], V (l x l).
void eig_sym_desc(int l, const double* G, int ldg, double* evals, double* V, int ldv);

// Eigen-decomposition of a symmetric positive semi-definite G (l x l),
// eigenvalues descending: the single-CTA Jacobi for small l, else the
// whole-GPU one-sided Jacobi SVD of G (singular values = eigenvalues).
void eig_psd_desc(int l, const double* G, int ldg, double* evals, double* V, int ldv);

// Thin SVD A = U diag(s) V^T of a rows x cols matrix by one-sided Jacobi,
// singular values descending, U rows x r, V cols x r with r = min(rows, cols).
// Null directions are completed to an orthonormal set.
void svd_thin(int rows, int cols, const double* A, int lda, double* U, int ldu, double* s,
              double* V, int ldv);

// Same contract as svd_thin, computed by a cooperative one-sided Jacobi over
// the whole GPU (one CTA per column pair, grid barrier per round); for
// min(rows, cols) in the hundreds and above.
void svd_jacobi_coop(int rows, int cols, const double* A, int lda, double* U, int ldu, double* s,
                     double* V, int ldv);

}  // namespace fpls
