// Prediction heads: low-rank regression predict, class argmax / top-k, LDA
// train (prefix models) and predict.  Device pointers, context stream.
#pragma once

#include "common.cuh"

namespace fpls {

// Ypred[:, :, a] = Xs R[:, :mc] W[:mc, :, a] + mY for each slice a, where Xs is
// the already centred / scaled test matrix (w x p).  T (w x kmax) is written.
void lowrank_predict(const double* Xs, int w, int p, const double* R, int kmax, const double* W,
                     int m, const int* ncomp_host, int L, const double* mY, double* T,
                     double* Ypred);

// labels[i] = 1 + first argmax_c (S[i, c] + bias[c]); S is w x C (ld w).
void row_argmax(const double* S, int w, int C, const double* bias, int* labels);
// top_k labels / scores per row (descending; ties keep the lower index first).
void row_topk(const double* S, int w, int C, const double* bias, int top_k, int* idx,
              double* score);

struct LdaModelsDev {
  double* means;      // C x kmax x L  (slice a uses the first ncomp[a] columns, ld C)
  double* linear;     // C x kmax x L
  double* constants;  // C x L
  double* priors;     // C
  double* lambda;     // L (host)
};

// lda_train_prefix_cpp (src/fastPLS.cpp:1817-1927) on scores T (n x kmax, ld n)
// with 1-based host labels y_host.  Throws on an empty class or out-of-range
// label.  Class sums run in a fixed order (no atomics): runs repeat bit for bit.
void lda_train_prefix(const double* T, int n, int kmax, const int* y_host, int C,
                      const int* ncomp_host, int L, double ridge, LdaModelsDev out);

}  // namespace fpls
