// Matrix-free cross-covariance operators for PLSSVD and SIMPLS.
#pragma once

#include "common.cuh"
#include "svd.cuh"

namespace fpls {

// Rank-k SVD of A = X^T Y (X n x p, Y n x m, centred, device) without forming
// A: Gaussian sketch (m x l), power iterations, QR, B = (X Q)^T Y and
// svd_econ(B).  Falls back to the exact SVD of the formed A when
// use_full_svd or l >= min(p, m), as the reference does.  U p x k, s k,
// V m x k (may be null).
SvdResult truncated_rsvd_crossprod_device(const double* X, int n, int p, const double* Y, int m, int k,
                                          int oversample, int power_iters, unsigned int seed,
                                          bool use_full_svd, double* U, int ldu, double* s, double* V,
                                          int ldv);

// Fast SIMPLS with the implicit deflated cross-covariance P_V X^T Y (no p x m
// matrix is kept).  R (p x K), Q (m x K) device outputs; B (p x m x L) and
// Yfit (n x m x L) device outputs or null; R2Y host (L).  Returns the number
// of components built.
int simpls_xprod_fit(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                     bool fit, unsigned int seed, const double* mY, double* R, double* Q, double* B,
                     double* Yfit, double* R2Y);

}  // namespace fpls
