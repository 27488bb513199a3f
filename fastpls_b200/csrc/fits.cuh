// Single-fit drivers (host orchestration of device kernels) for the PLS
// engines of src/fastPLS.cpp.  All pointers are device pointers.
#pragma once

#include "common.cuh"

namespace fpls {

struct FitOptions {
  int scaling = 1;        // 1 centre, 2 autoscale, 3 none (R/main.R:5890)
  bool fit = false;       // return fitted values and R2Y
  int svd_method = 4;     // 3 exact, 4/5 rsvd
  int oversample = 10;
  int power_iters = 1;
  double svds_tol = 0.0;
  unsigned int seed = 1;
  bool store_B = true;    // should_store_coefficients() decided by the caller
  bool xprod = false;     // PLSSVD: matrix-free X^T Y (src/fastPLS.cpp:5518-5690)
};

// Centres / scales X (n x p) and Y (n x m) in place, writing mX, vX (p) and mY (m).
void center_scale_xy(double* X, int n, int p, double* Y, int m, int scaling, double* mX,
                     double* vX, double* mY);

struct PlssvdOut {
  double* C_latent;  // K0 x K0 x L (zeroed by the callee)
  double* W_latent;  // K0 x m x L
  double* R;         // p x K0
  double* Q;         // m x K0
  double* T;         // n x K0
  double* s;         // K0
  double* B;         // p x m x L or null
  double* Yfit;      // n x m x L or null
  double* R2Y;       // L (host)
};

// PLSSVD (src/fastPLS.cpp:4780-4986) on already centred X, Y.  ncomp (host)
// is capped to [1, min(n,p,m)] by the caller.  Returns the effective rank.
int plssvd_fit_centered(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                        int L, int K0, const FitOptions& opt, const double* mY, PlssvdOut out);

struct SimplsOut {
  double* R;      // p x K
  double* Q;      // m x K
  double* T;      // n x K (classic only; may be null)
  double* P;      // p x K (classic only; may be null)
  double* B;      // p x m x L or null
  double* Yfit;   // n x m x L or null
  double* R2Y;    // L (host)
};

// Classic SIMPLS with a fresh leading left singular vector of the deflated
// cross-covariance per component (src/fastPLS.cpp:2260-2451).  Exact mode
// (svd_method 3) or the power-iteration leading vector (rsvd ids).
int simpls_classic_fit(const double* X, int n, int p, const double* Y, int m, const double* Yraw,
                       const int* ncomp, int L, const FitOptions& opt, const double* mY,
                       SimplsOut out);

}  // namespace fpls
