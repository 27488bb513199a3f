// Label-aware PLSSVD (segmented class-sum cross-covariance) on the device.
#pragma once

#include <vector>

#include "common.cuh"

namespace fpls {

// Device results of one label-aware fit (all buffers in the context arena).
struct LabelAwareFit {
  int n = 0, p = 0, m = 0, K = 0, rank = 0;
  std::vector<int> ncomp;               // capped ncomp values
  double* mX = nullptr;                 // p
  double* vX = nullptr;                 // p
  double* mY = nullptr;                 // m (class proportions)
  double* Xt = nullptr;                 // centred / scaled predictors, row-major (p x n col-major)
  double* S = nullptr;                  // p x m cross-covariance
  double* R = nullptr;                  // p x K left singular vectors
  double* Q = nullptr;                  // m x K right singular vectors
  double* d = nullptr;                  // K singular values
  double* T = nullptr;                  // n x K training scores X~R
  double* G = nullptr;                  // K x K latent Gram T^T T
  double* C = nullptr;                  // K x K x L latent coefficients
  double* W = nullptr;                  // K x m x L prediction weights C_k Q_k^T
};

// pmin(pmax(ncomp, 1), min(n, p, m)) (R/main.R:24-42).
std::vector<int> cap_plssvd_ncomp(const int* ncomp, int L, int n, int p, int m, int* max_rank);

// dX: n x p column-major FP32 or FP64 on the device; dy / y_host: class codes 1..m.
LabelAwareFit label_aware_fit(const void* dX, bool f32, int n, int p, const int* dy, const int* y_host,
                              int m, const std::vector<int>& ncomp, int scaling, int svd_method,
                              int oversample, int power_iters, unsigned int seed);

}  // namespace fpls
