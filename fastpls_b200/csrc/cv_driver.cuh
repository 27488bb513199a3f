// Cross-validation grids on the device: every fold fit of a CV (or double CV)
// runs in one batched SIMPLS engine pass over one resident predictor matrix,
// and the test rows' class predictions for every ncomp come from the scores
// of the same passes (no extra pass over X).
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"
#include "simpls_engine.cuh"

namespace fpls {

// A set of classification fits over the rows of a resident matrix.
struct CvFitSet {
  int n = 0, p = 0, m = 0;          // rows, predictors, classes
  int F = 0;                        // fits
  int G = 0;                        // prediction groups
  std::vector<uint8_t> train;       // F x n
  std::vector<uint8_t> test;        // F x n
  std::vector<int> group;           // F: prediction group of each fit
  std::vector<unsigned> seeds;      // F
  // Optional, filled by builders that know the fold structure: training-row
  // class counts (F x m) and training / test row counts (F); empty otherwise.
  std::vector<int> train_class_counts;
  std::vector<int> n_train, n_test;
};

struct CvGridOptions {
  int scaling = 1;                  // 1 centre, 2 autoscale, 3 none
  int precision = 0;                // 0 FP64, 1 BF16x3 split, 2 BF16x6 split
  bool batched = true;              // false: one fit after another (plain drop-in path)
  int power_iters = 2;              // FASTPLS_FAST_INC_ITERS
  bool want_scores = false;         // also keep the class scores behind every prediction
};

struct CvGridResult {
  int* d_pred = nullptr;            // device G x L x n (0 where the row is not predicted);
                                    // valid until the next call resets the arena
  double* d_score = nullptr;        // with opt.want_scores: device G x L x n x m class scores
                                    // (classes fastest; 0 where the row is not predicted or
                                    // its fold took a fallback class)
  std::vector<int> status;          // F: 1 ok, 2 empty test, 3 no train, 4 degenerate
};

// Per (group g, slice s): counts[2*(g*L+s)] = correct predictions and
// counts[2*(g*L+s)+1] = predicted rows, over the rows where exclude[i] != g
// (exclude may be null).  Device buffers in, host vector out.
// The same counts left on the device (no synchronisation).
long long* cv_prediction_counts_device(const int* d_pred, int G, int L, int n, const int* d_labels,
                                      const int* d_exclude);
void cv_prediction_counts(const int* d_pred, int G, int L, int n, const int* d_labels,
                          const int* d_exclude, std::vector<long long>& counts);

// The fold-independent X-side work of a batched CV grid: the column means, the
// BF16 planes of Xc (mixed row-space path) or a centred FP64 copy of X, its
// first centred column x0 and, on the row-space path, the row Gram
// K = Xc Xc^T with the operator of the per-component K products.
// cv_prepare_x enqueues it on the library stream (a host X is uploaded first,
// or in overlapped column chunks on the mixed row-space path);
// cv_grid_classify does the same itself unless it is given one prepared for
// the same X, class count, largest ncomp and options.
struct CvPreparedX {
  bool center = false, dual = false;
  int n = 0, p = 0, m = 0, kmax = 0, precision = 0;
  double* mall = nullptr;   // p column means when centred
  double* Kg = nullptr;     // n x n row Gram (row-space path)
  double* X = nullptr;      // centred FP64 copy (every path but the mixed row-space one)
  double* x0 = nullptr;     // first centred column
  std::unique_ptr<XOperator> xop, kop_f64, kop_int8;
  int kop_slices = 0;
  double* XOm = nullptr;    // X Omega of the row-space loop, when taken on the side stream
};

// Batched grids only (opt.batched with scaling != 2); x64 / x32 as in
// cv_grid_classify (the device buffer to fill when x_host is given).
std::unique_ptr<CvPreparedX> cv_prepare_x(const double* x64, const float* x32, int n, int p, int m, int kmax,
                                          const CvGridOptions& opt, const void* x_host);

// X: device predictor matrix n x p, FP64 (x64) or FP32 (x32, exactly widened).
// labels_host: 1-based class labels.  ncomp: L values (host).  With x_host the
// device buffer is empty and x_host holds the same matrix in host memory: the
// driver uploads it, in column chunks overlapped with the column means, the
// BF16 split and the row Gram on the mixed row-space path, else in one copy.
void cv_grid_classify(const CvFitSet& fs, const double* x64, const float* x32,
                      const int* labels_host, const int* ncomp, int L,
                      const CvGridOptions& opt, CvGridResult& res, const void* x_host = nullptr,
                      CvPreparedX* prep = nullptr);

}  // namespace fpls
