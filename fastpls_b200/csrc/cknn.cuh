// Candidate-kNN classifier pieces on device buffers (column-major FP64).
#pragma once

#include "common.cuh"

namespace fpls {

// dTn (n x k) = row_l2(dT dCk), or row_l2(dT) when dCk is null.
void candidate_scores_device(const double* dT, int n, int k, const double* dCk, double* dTn);

// dCent (C x k) = row_l2 of the per-class means of dTn rows (codes 1..C in dy).
void candidate_centroids_device(const double* dTn, int n, int k, const int* dy, int C, double* dCent);

// Candidate selection, smoothed class-kNN scoring and rerank; d_ti / d_ts are
// ntest x max(1, min(top_k, C)).  dbias may be null (zeros).  allow_filter =
// false keeps the similarity tiles on the FP64 kernels.
void candidate_knn_predict_device(const double* dTt, int ntest, const double* dTr, int ntrain, int kdim,
                                  const int* dy, const double* dC, int C, const double* dbias, int top_k,
                                  int top_m, int knn_k, double tau, double alpha, int* d_ti, double* d_ts,
                                  bool allow_filter = true);

}  // namespace fpls
