// Batched fast-SIMPLS engine (src/fastPLS.cpp:2454-2778 with the default
// option set) over F fits that share one resident predictor matrix.
//
// Fit f sees the rows where mask_f = 1 ("train" rows); its predictors are the
// resident centred matrix Xc shifted by the fold offset delta_f (the fold's
// column means of Xc) and divided by its column scales.  Per component every
// fit runs the warm-started 1-column refresh (two power iterations, QR sign
// convention of LAPACK), t = X r, p = X^T t, q = Y^T t, the Gram-Schmidt of p
// against earlier loadings and the rank-1 deflation of its cross-covariance,
// exactly as the reference; the two passes over X are batched across fits into
// skinny GEMMs (FP64 DMMA, or the BF16 split tcgen05 path).  No host
// synchronisation happens inside the component loop: a fit whose component is
// degenerate (zero norm) is stopped on the device, as the reference's loop
// breaks.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace fpls {

// Operator applying the two predictor passes for all fits:
//   U (n x F)  = Xc * Rhat      (Rhat p x F)
//   P (p x F)  = Xc^T * T       (T n x F)
struct XOperator {
  virtual ~XOperator() {}
  virtual void times(const double* Rhat, int F, double* U) = 0;
  virtual void t_times(const double* T, int F, double* P) = 0;
  // K (n x n) = Xc Xc^T, the row Gram of the predictors.
  virtual void gram(double* K) = 0;
  int n = 0, p = 0;
};

// FP64 operator over a device matrix Xc (n x p, ld n).
struct XOperatorF64 : public XOperator {
  const double* Xc = nullptr;
  XOperatorF64(const double* X, int n_, int p_) : Xc(X) { n = n_; p = p_; }
  void times(const double* Rhat, int F, double* U) override;
  void t_times(const double* T, int F, double* P) override;
  void gram(double* K) override;
};

struct SimplsBatch {
  int n = 0, p = 0, m = 0, F = 0, K = 0;     // K = max components
  int power_iters = 2;                       // FASTPLS_FAST_INC_ITERS
  XOperator* X = nullptr;
  // Responses: dense centred Yg (n x m) or 0-based labels (one-hot implied,
  // centred by mY_all).  Exactly one is non-null.
  const double* Yg = nullptr;
  const int* labels = nullptr;
  const double* mY_all = nullptr;            // m (labels mode)
  const uint8_t* mask = nullptr;             // F x n train masks, null = all rows
  const double* delta = nullptr;             // F x p fold offsets, null = zero
  const double* colsum = nullptr;            // F x p fold column sums X^T D_f 1 (response centring)
  const double* colscale = nullptr;          // F x p (1/vX), null = ones
  const double* dY = nullptr;                // F x m response offsets, null = zero
  double* S = nullptr;                       // F x p x m cross-covariances (deflated in place)
  const double* omega = nullptr;             // F x p first-component sketch
  bool m1_mode = false;                      // m == 1: exact left vector of S
  // Outputs
  double* R = nullptr;                       // F x p x K
  double* Q = nullptr;                       // F x m x K
  double* V = nullptr;                       // F x p x K (loadings basis)
  double* tnorm = nullptr;                   // F x K
  double* Tkeep = nullptr;                   // optional F x n x K unnormalised scores (all rows)
  int* ncomp_done = nullptr;                 // F
  int* status = nullptr;                     // F (0 active, 1 stopped)
};

// Runs K components for all fits.  Device pointers throughout; launches only.
void simpls_batch_run(const SimplsBatch& b);

// Frees the executable graph of the component loop (fpls_reset_workspace).
void simpls_release_graph();

// S_f = diag(colscale_f) [ Xc^T D_f Y - colsum_f off_f^T ] for all fits (the
// masked cross-covariances with the fold-centred response, off_f the fold's
// response means), via one GEMM Xc^T [D_1 Y ... D_F Y].
void simpls_batch_crosscov(const SimplsBatch& b, const double* Xc, const int* n_train);

}  // namespace fpls
