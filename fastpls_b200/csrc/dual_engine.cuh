// Batched fast SIMPLS in the row space of the predictors ("dual" form), for
// short, wide predictor blocks (n rows << p columns).
//
// Every p-dimensional vector the fast SIMPLS loop builds after its first
// refresh step lies in the row space of the centred predictors Xc: the
// cross-covariance S_f = Xc^T C_S (C_S = D_f (Y - 1 mY_f^T), masked and
// centred within the fold), the refresh vector y = S z, the weight r, the
// loading p = X_f^T t and the orthonormal loading basis V.  Writing each as
// Xc^T c with an n-vector c, every inner product becomes c1^T K c2 with the
// row Gram K = Xc Xc^T, and X_f r becomes the within-fold centring of K c_r.
// The loop then runs on n-vectors: per component one batched K-product (the
// Gram-Schmidt image K c_p); K C_S and K V are carried along and updated by
// the same rank-1 deflations as C_S and V.  The first refresh step applies
// S^T to the p-dimensional sketch through Xc Omega (one pass over X).
//
// The arithmetic is the reference's loop (src/fastPLS.cpp:2454-2778 with the
// default options: refresh block 1, two power iterations from the warm start,
// Householder sign, classical Gram-Schmidt, rank-1 deflation) restated in
// these coordinates, so the per-fit scores, loadings' images, Q and the
// prediction scores agree with the p-space engine to rounding.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "simpls_engine.cuh"

namespace fpls {

struct DualBatch {
  int n = 0, m = 0, F = 0, K = 0;
  int power_iters = 2;
  bool m1_mode = false;
  bool center = true;                // fold centring of the predictors (scaling < 3)
  XOperator* Kop = nullptr;          // K = Xc Xc^T (n x n), times() only
  int kop_int8_slices = 0;           // > 0: Kop is the INT8 digit-plane product with these slices
  const double* x0 = nullptr;        // n: first column of Xc (Householder sign)
  const double* XOmega = nullptr;    // n x F: Xc Omega_f (first refresh step)
  const uint8_t* mask = nullptr;     // F x n train masks
  const int* labels = nullptr;       // n, 0-based classes
  const double* mY_all = nullptr;    // m
  const double* dY = nullptr;        // F x m fold offsets of the class proportions
  const int* ntrain = nullptr;       // F train-row counts
  const double* class_cnt = nullptr; // F x m train rows per class (exact integers)
  // Outputs (as SimplsBatch)
  double* Q = nullptr;               // F x m x K
  double* tnorm = nullptr;           // F x K
  double* Tkeep = nullptr;           // F x n x K unnormalised scores (all rows)
  int* ncomp_done = nullptr;         // F
  int* status = nullptr;             // F
};

// Runs K components for all fits; launches only (no host synchronisation).
void dual_simpls_run(const DualBatch& b);

// Frees the executable graph of the component loop (fpls_reset_workspace).
void dual_release_graph();

// True when the dual form applies to this shape (and fits its staging limits).
bool dual_engine_applies(int n, int p, int m, int K);

// K = (K + K^T) / 2 in place (n x n).
void symmetrize(double* K, int n);

}  // namespace fpls
