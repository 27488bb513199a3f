/*
 * fastpls_b200 — C ABI of the B200 (sm_100a) fit/predict library for fastPLS.
 *
 * Every entry point replaces one `.Call` routine of the R package fastPLS
 * (tkcaccia/fastPLS) for backend = "cuda"; the citation names the routine's
 * registration in src/RcppExports.cpp and the engine function it runs.
 *
 * Conventions
 *  - Matrices are column-major double (R / Armadillo layout); "cubes" are
 *    rows x cols x slices, slice-major, as R arrays.
 *  - Class labels are int32, 1-based.  ncomp vectors are int32.
 *  - Pointers are owned by the caller; outputs are written into
 *    caller-allocated buffers of the documented sizes.  Optional outputs may
 *    be NULL.  Scalars' arrays (labels, folds, ncomp lists, R2Y and the other
 *    per-component or per-class vectors) are HOST memory.  The matrices a call
 *    copies whole (X, Y, Xtest, the response Z, the filtered X and the
 *    prediction blocks of fpls_pls_model1, fpls_pls_model2_fast,
 *    fpls_predict_lowrank, fpls_lda_project_train_prefix,
 *    fpls_lda_project_predict, fpls_opls_filter, fpls_opls_apply_filter,
 *    fpls_gaussian_y_encode / _decode and fpls_x_upload) may instead be device
 *    memory of the library's device: unified addressing tells the two apart
 *    and the copy then stays in HBM (no counterpart in the reference, whose
 *    inputs are R objects in host memory).
 *  - Every function returns 0 on success or a non-zero fpls_status; on failure a
 *    NUL-terminated message is written to err[0..errlen-1] (err may be NULL).
 *    No exception crosses this boundary and there is no CPU fallback: without
 *    a B200 the calls return FPLS_ERR_NO_DEVICE.
 *  - The library keeps one device context per process (stream, scratch arena),
 *    used from one host thread at a time, like the reference's thread_local
 *    CUDA workspace (src/svd_cuda_rsvd.cpp:2092).
 */
#ifndef FASTPLS_B200_H
#define FASTPLS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fpls_status {
  FPLS_OK = 0,
  FPLS_ERR_ARGUMENT = 1,
  FPLS_ERR_CUDA = 2,
  FPLS_ERR_NUMERICAL = 3,
  FPLS_ERR_NO_DEVICE = 4,
  FPLS_ERR_INTERNAL = 5
};

/* Precision of the predictor passes in the batched CV grid. */
/* FP64: the drop-in.  BF16X3: operands split into two BF16 planes (hi, lo),
 * three tensor-core products (~2^-16 relative per product).  BF16X6: three
 * planes (hi, mid, lo), six products (~2^-24), FP32 accumulation in short
 * segments, FP64 sums. */
enum fpls_precision { FPLS_PREC_FP64 = 0, FPLS_PREC_BF16X3 = 1, FPLS_PREC_BF16X6 = 2, FPLS_PREC_INT8 = 3 };

/* 1 when a B200 (sm_100a) device is usable.
 * Replaces _fastPLS_has_cuda (RcppExports.cpp:87; fastPLS.cpp:1607-1609). */
int fpls_has_cuda(void);

/* Library version string. */
const char* fpls_version(void);

/* Releases the scratch arena and cached device state.
 * Replaces _fastPLS_cuda_reset_workspace (RcppExports.cpp:107; fastPLS.cpp:1617-1620). */
int fpls_reset_workspace(char* err, size_t errlen);

/* C (a_rows x b_cols) = A (a_rows x a_cols) * B (a_cols x b_cols), FP64.
 * Replaces _fastPLS_cuda_matrix_multiply (RcppExports.cpp:116; svd_cuda_rsvd.cpp:2106-2180). */
int fpls_matrix_multiply(const double* A, int a_rows, int a_cols, const double* B, int b_cols,
                         double* C, char* err, size_t errlen);

/* Truncated SVD of A (rows x cols) with the CPU recipe of the reference
 * (svd_method 3 exact, 4/5 randomized).  kcap = min(rows, cols, max(k,1));
 * U: rows x kcap, s: kcap, Vt: kcap x cols (NULL when left_only).  *rank_out is
 * the number of columns written (the rSVD may return fewer usable ones).
 * Replaces _fastPLS_truncated_svd_debug (RcppExports.cpp:334; fastPLS.cpp:2229-2257). */
int fpls_truncated_svd(const double* A, int rows, int cols, int k, int svd_method, int oversample,
                       int power_iters, double svds_tol, int seed, int left_only, double* U,
                       double* s, double* Vt, int* rank_out, char* err, size_t errlen);

/* PLSSVD fit.  ncomp values are capped to [1, min(n,p,m)] and written to
 * ncomp_out (L).  K0 = min(max(ncomp_out), min(n,p,m)).  Outputs:
 * C_latent K0 x K0 x L, W_latent K0 x m x L, Q m x K0, Ttrain n x K0, R p x K0,
 * mX p, vX p, mY m, B p x m x L (optional), Yfit n x m x L (optional, fit=1),
 * R2Y L, s K0; *k_eff = effective rank (columns of R/Q/Ttrain written).
 * Replaces _fastPLS_pls_model1_gpu (RcppExports.cpp:668; fastPLS.cpp:5989-6082);
 * numerics follow pls_model1 (fastPLS.cpp:4780-4986). */
int fpls_pls_model1(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                    int scaling, int fit, int svd_method, int oversample, int power_iters,
                    double svds_tol, int seed, int* ncomp_out, double* C_latent, double* W_latent,
                    double* Q, double* Ttrain, double* R, double* mX, double* vX, double* mY,
                    double* B, double* Yfit, double* R2Y, double* s, int* k_eff, char* err,
                    size_t errlen);

/* Matrix-free PLSSVD: as fpls_pls_model1 with the rank-K SVD of XᵀY taken
 * by the operator rSVD (sketch Ω m x l, A M = Xᵀ(Y M), Aᵀ M = Yᵀ(X M), QR,
 * B = (XQ)ᵀY, svd_econ(B)); XᵀY is formed only for the exact fallback
 * (min(n,p,m) <= 32, or l >= min(p, m)).  xprod_precision must be 3 (5 is
 * the CPU-only IRLBA operator; 1, 2, 4 were removed).  Outputs as
 * fpls_pls_model1.  Replaces _fastPLS_pls_model1_rsvd_xprod_precision
 * (RcppExports.cpp:628; fastPLS.cpp:5518-5690, 550-622). */
int fpls_pls_model1_xprod(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                          int L, int scaling, int fit, int oversample, int power_iters,
                          double svds_tol, int seed, int xprod_precision, int* ncomp_out,
                          double* C_latent, double* W_latent, double* Q, double* Ttrain, double* R,
                          double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                          double* s, int* k_eff, char* err, size_t errlen);

/* Matrix-free fast SIMPLS: the refresh applies P_V XᵀY implicitly
 * (P_V = I − V Vᵀ over the loadings so far) instead of deflating a stored
 * p x m matrix.  xprod_precision must be 3.  Outputs as fpls_pls_model2_fast.
 * Replaces _fastPLS_pls_model2_fast_rsvd_xprod_precision (RcppExports.cpp:648;
 * fastPLS.cpp:5695-5986, 936-1000). */
int fpls_pls_model2_fast_xprod(const double* X, int n, int p, const double* Y, int m,
                               const int* ncomp, int L, int scaling, int fit, int seed,
                               int xprod_precision, double* R, double* Q, double* mX, double* vX,
                               double* mY, double* B, double* Yfit, double* R2Y, int* n_components,
                               char* err, size_t errlen);

/* Fast SIMPLS fit (warm-started 1-column refresh, 2 power iterations).
 * K = max(ncomp).  Outputs: R p x K, Q m x K, mX p, vX p, mY m,
 * B p x m x L (optional), Yfit n x m x L (optional), R2Y L; *n_components =
 * components computed (the loop stops early on a degenerate component).
 * Replaces _fastPLS_pls_model2_fast_gpu (RcppExports.cpp:392; fastPLS.cpp:2781-3207);
 * numerics follow pls_model2_fast (fastPLS.cpp:2454-2778). */
int fpls_pls_model2_fast(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                         int L, int scaling, int fit, int seed, double* R, double* Q, double* mX,
                         double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                         int* n_components, char* err, size_t errlen);

/* Row-sharded fits (one process per GPU, each holding a block of the rows of
 * X and Y).  Every sum over rows -- the column sums of the centring (and the
 * sums of squares for scaling 2), S = XᵀY, per component Xᵀt, tᵀt and Yᵀt
 * (fast SIMPLS) or TᵀT (PLSSVD), and the residual sums of R2Y -- is completed
 * by `allreduce`, which must sum `count` doubles of device memory at `buf`
 * over all ranks in place.  `stream` is the library's cudaStream_t: the sum
 * must see the work already enqueued on it and finish before the work
 * enqueued after it (enqueue the collective on that stream, or synchronise
 * it).  Every rank calls the fit with the same p, m, ncomp, scaling, fit,
 * seed and SVD options, and the library makes the same calls in the same
 * order on every rank; the first sums the local row counts.  Return 0 on
 * success; any other value fails the fit with FPLS_ERR_CUDA (the other ranks
 * then wait in their next all-reduce: give the process group a timeout).
 * With one rank the outputs are the unsharded fit's, bit for bit. */
typedef int (*fpls_allreduce_fn)(double* buf, long long count, void* stream, void* user);

/* fpls_pls_model1 over this rank's n rows.  The model (C_latent, W_latent, Q,
 * R, mX, vX, mY, B, R2Y, s, ncomp_out, k_eff) is the fit of all ranks' rows
 * and is the same on every rank; Ttrain and Yfit are this rank's rows.
 * min(n, p, m) caps use the total row count.  Row sharding of
 * fastPLS.cpp:4780-4986 (the S all-reduce and the T^T T all-reduce). */
int fpls_pls_model1_rows(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                         int scaling, int fit, int svd_method, int oversample, int power_iters,
                         double svds_tol, int seed, fpls_allreduce_fn allreduce, void* user, int* ncomp_out,
                         double* C_latent, double* W_latent, double* Q, double* Ttrain, double* R, double* mX,
                         double* vX, double* mY, double* B, double* Yfit, double* R2Y, double* s, int* k_eff,
                         char* err, size_t errlen);

/* fpls_pls_model2_fast over this rank's n rows: one all-reduce of
 * [Xᵀt | tᵀt, Σt | Yᵀt] (p + 2 + m doubles) per component.  R, Q, mX, vX, mY,
 * B, R2Y and n_components are the fit of all ranks' rows; Yfit is this
 * rank's rows.  Row sharding of fastPLS.cpp:2454-2778. */
int fpls_pls_model2_fast_rows(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                              int L, int scaling, int fit, int seed, fpls_allreduce_fn allreduce, void* user,
                              double* R, double* Q, double* mX, double* vX, double* mY, double* B,
                              double* Yfit, double* R2Y, int* n_components, char* err, size_t errlen);

/* Classic SIMPLS with a fresh leading left singular vector per component
 * ("exact" mode when svd_method = 3).  K = max(ncomp).  Outputs: R p x K,
 * Q m x K, P p x K (optional), Ttrain n x K (optional; required when fit=1),
 * mX, vX, mY, B (optional), Yfit (optional), R2Y.
 * Replaces _fastPLS_pls_model2 (RcppExports.cpp:352; fastPLS.cpp:2260-2451). */
int fpls_pls_model2(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                    int L, int scaling, int fit, int svd_method, int oversample, int power_iters,
                    double svds_tol, int seed, double* R, double* Q, double* P, double* Ttrain,
                    double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y,
                    int* n_components, char* err, size_t errlen);

/* Low-rank prediction Ypred[:,:,a] = ((Xtest - mX)/vX) R[:, :mc] W[:mc, :, a] + mY,
 * mc = ncomp[a].  W is kmax x m x L (SIMPLS: Q^T prefixes; PLSSVD: W_latent).
 * Ypred w x m x L; Ttest w x kmax (optional).
 * Replaces _fastPLS_pls_predict_flash_cuda (RcppExports.cpp:425; fastPLS.cpp:3448-3585). */
int fpls_predict_lowrank(const double* Xtest, int w, int p, const double* mX, const double* vX,
                         const double* mY, int m, const double* R, int kmax, const double* W,
                         const int* ncomp, int L, double* Ypred, double* Ttest, char* err,
                         size_t errlen);

/* Class prediction from the same low-rank model: per slice, the top_k classes
 * of Ypred + class_bias (first maximum wins ties).  class_bias: m or NULL.
 * top_index w x top_k x L (1-based), top_score w x top_k x L (optional).
 * When the score cube of all rows would pass 1 GiB (large class counts or
 * many test rows), the rows are scored in blocks, the next block's copy in
 * flight, so device memory stays bounded (FASTPLS_PREDICT_BLOCK_ROWS sets the
 * block).
 * Replaces _fastPLS_pls_class_predict_topk_cuda (RcppExports.cpp:468;
 * fastPLS.cpp:3863-4113) and pls_predict_classes_compact_cuda (fastPLS.cpp:4156-4201). */
int fpls_predict_classes(const double* Xtest, int w, int p, const double* mX, const double* vX,
                         const double* mY, int m, const double* R, int kmax, const double* W,
                         const int* ncomp, int L, const double* class_bias, int top_k,
                         int* top_index, double* top_score, char* err, size_t errlen);

/* Prefix LDA models on latent scores T (n x kmax), labels y (n, 1-based).
 * For slice a (kk = ncomp[a]): means[:, :kk, a] (C x kmax x L, ld C),
 * linear[:, :kk, a] (C x kmax x L), constants[:, a] (C x L), priors C,
 * lambda L.  Replaces _fastPLS_lda_train_prefix_cuda (RcppExports.cpp:225);
 * numerics follow lda_train_prefix_cpp (fastPLS.cpp:1817-1927). */
int fpls_lda_train_prefix(const double* T, int n, int kmax, const int* y, int n_classes,
                          const int* ncomp, int L, double ridge, double* means, double* linear,
                          double* constants, double* priors, double* lambda, char* err,
                          size_t errlen);

/* Same on projected scores T = X R - offset (X n x p, R p x k, offset k).
 * Replaces _fastPLS_lda_project_train_prefix_cuda (RcppExports.cpp:240;
 * fastPLS.cpp:1930-1957). */
int fpls_lda_project_train_prefix(const double* X, int n, int p, const double* R, int k,
                                  const double* offset, const int* y, int n_classes,
                                  const int* ncomp, int L, double ridge, double* means,
                                  double* linear, double* constants, double* priors,
                                  double* lambda, char* err, size_t errlen);

/* LDA labels for scores T (w x k): argmax_c T linear^T + constants.
 * linear: C x k, constants: C.  labels w; scores w x C (optional, includes constants).
 * Replaces _fastPLS_lda_predict_cuda / _lda_predict_labels_cuda (RcppExports.cpp:295, 307). */
int fpls_lda_predict(const double* T, int w, int k, const double* linear,
                     const double* constants, int n_classes, int* labels, double* scores,
                     char* err, size_t errlen);

/* LDA labels for predictors X (w x p) with projection R (p x k) and offset (k):
 * the direct route X (R linear^T) when cheaper, else (X R - offset) linear^T.
 * scores (optional) w x C = (X R) linear^T + constants - offset linear^T.
 * Replaces _fastPLS_lda_project_predict_cuda (RcppExports.cpp:319;
 * fastPLS.cpp:2100-2147 for the route rule). */
int fpls_lda_project_predict(const double* X, int w, int p, const double* R, int k,
                             const double* offset, const double* linear,
                             const double* constants, int n_classes, int* labels,
                             double* scores, char* err, size_t errlen);

/* Kernel matrix K (n1 x n2) between the rows of X1 (n1 x p) and X2 (n2 x p):
 * kernel 1 linear x.y; 2 RBF exp(-gamma |x - y|^2) (tiny negative distances
 * above -1e-10 set to 0); 3 polynomial (gamma x.y + coef0)^degree.  FP64; the
 * dot products run on the FP64 tensor cores.
 * Replaces kernel_matrix_cpp (RcppExports.cpp; fastPLS.cpp:4314-4340). */
int fpls_kernel_matrix(const double* X1, int n1, const double* X2, int n2, int p, int kernel, double gamma,
                       int degree, double coef0, double* K, char* err, size_t errlen);

/* Double centring of a training kernel K (n x n): Kc = ((K - col_means) -
 * row_means) + grand_mean, with col_means (n) and grand_mean returned.
 * Replaces center_kernel_train_cpp (fastPLS.cpp:4344-4357). */
int fpls_center_kernel_train(const double* K, int n, double* Kc, double* col_means, double* grand_mean,
                             char* err, size_t errlen);

/* Centring of a test kernel Ktest (nt x n) with the training col_means and
 * grand_mean and its own row means.
 * Replaces center_kernel_test_cpp (fastPLS.cpp:4360-4375). */
int fpls_center_kernel_test(const double* Ktest, int nt, int n, const double* col_means, double grand_mean,
                            double* Kc, char* err, size_t errlen);

/* Kernel PLS fit on the device in one call: the preprocessing of X (scaling
 * 1 centre, 2 autoscale with sd 0 -> 1, 3 none; mX, vX (p) returned), the
 * kernel matrix of the preprocessed rows (gamma <= 0 selects 1 / p, the value
 * used is returned), its double centring (col_means (n), grand_mean), and the
 * fast SIMPLS fit on the centred kernel with scaling "none" (outputs as
 * fpls_pls_model2_fast with p = n: R (n x kmax), Q, mK, vK (n), mY, B, Yfit,
 * R2Y, n_components).  The R route .kernel_pls_fit (R/main.R:2826-2917) calls
 * kernel_matrix_cpp, center_kernel_train_cpp and the GPU fit one after another
 * through host memory. */
int fpls_kernel_pls_model2_fast(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                                int scaling, int kernel, double gamma, int degree, double coef0, int fit,
                                int seed, double* R, double* Q, double* mK, double* vK, double* mY, double* B,
                                double* Yfit, double* R2Y, int* n_components, double* mX, double* vX,
                                double* col_means, double* grand_mean, double* gamma_used, char* err,
                                size_t errlen);

/* C (M x N) = A (M x K) * B (K x N) through the BF16 split-precision tensor-core
 * path (hi/lo three-product tcgen05 GEMM, FP32 accumulation, FP64 reduction of
 * the K-split partials).  A diagnostic of the mixed-precision kernel; it has no
 * counterpart in the reference. */
int fpls_bf16x3_gemm(const double* A, int M, int K, const double* B, int N, double* C,
                     char* err, size_t errlen);

/* C (M x N) = A (M x K) * B (K x N) through the FP64-accurate INT8 tensor-core
 * product: every row of A and column of B is scaled by a power of two and
 * split into `slices` (4..7) signed 7-bit digit planes, the plane pairs with
 * s + t <= slices + 1 are multiplied exactly (tcgen05 kind::i8, int32
 * accumulation) and recombined in FP64 (Ozaki scheme).  Entry (i, j) differs
 * from the exact product by at most about 3 K 2^(eA_i + eB_j - 7 slices),
 * 2^e the scale of row i of A or column j of B.  The mixed-precision CV grids
 * use it for their row-space products; a diagnostic with no counterpart in
 * the reference. */
int fpls_int8_emulated_gemm(const double* A, int M, int K, const double* B, int N, int slices,
                            double* C, char* err, size_t errlen);

/* K (n x n) = (X - mean)(X - mean)^T through the INT8 tensor cores: the rows
 * of X (n x p, FP64 or FP32 with x_is_float32 = 1; mean p or null) cut into
 * `slices` (4..7) signed 7-bit digit planes with a power-of-two scale per row,
 * the plane pairs with s + t <= slices + 1 multiplied exactly (int32) on the
 * upper tiles and combined in FP64, the lower triangle mirrored; entry (i, j)
 * is within about 3 p 2^(e_i + e_j - 7 slices) of the exact product, 2^e_i the
 * scale of row i.  The row Gram of the FPLS_PREC_INT8 CV grids; a diagnostic
 * with no counterpart in the reference. */
int fpls_int8_gram(const void* X, int x_is_float32, int n, int p, const double* mean, int slices, double* K,
                   char* err, size_t errlen);

/* Cross-validated class predictions with the argmax classifier for method 3
 * (simpls_fast).  X is n x p, FP64 (x_is_float32 = 0) or FP32 (= 1); y are
 * 1-based labels; fold holds 0-based fold ids (drawn by the caller, as the R
 * shim draws them with R's RNG); fit f uses seed + f.  All fold fits run in one
 * batched engine pass when batched = 1 (precision FPLS_PREC_FP64,
 * FPLS_PREC_BF16X3, FPLS_PREC_BF16X6 or FPLS_PREC_INT8: the mixed forms build
 * the row Gram from two BF16 planes and three products, three planes and six,
 * or -- FPLS_PREC_INT8 -- from signed 7-bit digit planes of the centred rows
 * multiplied exactly on the INT8 tensor cores (Ozaki scheme; the sketch
 * product the same way; class scores within 1e-5 of the FP64 grid), and all
 * keep the per-component products FP64-accurate on the INT8 tensor cores;
 * FPLS_PREC_INT8 grids that do not take the row-space engine run in FP64),
 * else one after another in FP64 (the plain drop-in path).
 * class_pred n x L (1-based; 0 where not predicted), status kfold (1 ok,
 * 2 empty fold, 3 no training rows, 4 single-class training fold).
 * Replaces _fastPLS_pls_cv_predict_compiled (RcppExports.cpp:731;
 * fastPLS.cpp:6615-7151) with backend = 1 and classifier = 0. */
int fpls_cv_predict(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                    const int* fold, int kfold, const int* ncomp, int L, int method, int scaling,
                    int seed, int precision, int batched, int* class_pred, int* status,
                    char* err, size_t errlen);

/* fpls_cv_predict that also returns class_score L x n x n_classes (entry
 * (l n + i) n_classes + c), the Ypred rows the argmax of each prediction read
 * (zeros where a fold took a fallback class or predicted nothing).  The
 * reference's classifier-0 CV returns labels only; this is its score matrix
 * for margin checks. */
int fpls_cv_predict_scores(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                           const int* fold, int kfold, const int* ncomp, int L, int method, int scaling,
                           int seed, int precision, int batched, int* class_pred, int* status,
                           double* class_score, char* err, size_t errlen);

/* Fused PLS + LDA classifier: one call fits PLSSVD (method 1: seeded rSVD,
 * or the matrix-free operator with xprod = 1) or fast SIMPLS (method 3) on
 * Xtrain (n x p; FP64, or FP32 with x_is_float32 = 1, the same for Xtest) and
 * the response Ytrain (n x m, FP64; the one-hot of y for PLS-DA), trains one
 * LDA model per distinct ncomp on the fit's own training scores
 * (X - mX) / vX R, and predicts the ntest rows of Xtest with each ncomp slice.
 * X crosses to the device once.  Outputs (NULL to skip): ncomp_out (L, capped
 * at min(n, p, m) for PLSSVD), R (p x K0), Q (m x K0), mX, vX (p), mY (m), B
 * (p x m x L), Yfit (n x m x L, fit = 1), R2Y (L); n_unique = U and
 * unique_ncomp (U, increasing); lda_means and lda_linear (n_classes x K0 x U,
 * slice u filled in its first unique_ncomp[u] columns), lda_constants
 * (n_classes x U), lda_priors (n_classes), lda_lambda (U); R_predict (p x K0,
 * R with rows divided by vX) and R_offset (K0, mX R_predict); pred_codes
 * (ntest x L, 1-based, required when ntest > 0).  K0 = max(ncomp_out).
 * Replaces _fastPLS_pls_lda_gpu_native (RcppExports.cpp:706;
 * fastPLS.cpp:6182-6443). */
int fpls_pls_lda(const void* Xtrain, int x_is_float32, int n, int p, const double* Ytrain, int m,
                 const int* y, const void* Xtest, int ntest, const int* ncomp, int L, int n_classes,
                 int method, int scaling, int xprod, int fit, int oversample, int power_iters,
                 double svds_tol, int seed, double lda_ridge, int* ncomp_out, double* R, double* Q,
                 double* mX, double* vX, double* mY, double* B, double* Yfit, double* R2Y, int* n_unique,
                 int* unique_ncomp, double* lda_means, double* lda_linear, double* lda_constants,
                 double* lda_priors, double* lda_lambda, double* R_predict, double* R_offset,
                 int* pred_codes, char* err, size_t errlen);

/* Double cross-validation of SIMPLS PLS-DA (argmax classifier): for every outer
 * fold o, an inner CV over its training rows picks ncomp (first maximum of the
 * inner accuracy), then a refit on the outer training rows predicts fold o.
 * outer_fold: n 0-based ids; inner_fold: n x kfold_outer, inner fold id of row i
 * within outer fold o (ignored for the rows of fold o).  Seeds follow
 * pls.double.cv: inner fits seed + 1000 run + (o+1) + inner fold, refits
 * seed + 2000 run + (o+1).  All kfold_outer x (kfold_inner + 1) fits run in one
 * batched engine pass (batched = 1) or one after another (batched = 0).
 * Outputs: best_comp kfold_outer, inner_accuracy kfold_outer x L, outer_pred n,
 * inner_pred kfold_outer x L x n (optional), fit_status (optional).
 * Replaces the loop of pls.double.cv (R/main.R:6586-6760) over
 * _fastPLS_pls_cv_predict_compiled (RcppExports.cpp:731) and pls() refits; no
 * single reference routine covers the whole grid. */
int fpls_double_cv(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                   const int* outer_fold, int kfold_outer, const int* inner_fold, int kfold_inner,
                   const int* ncomp, int L, int scaling, int seed, int run, int precision,
                   int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                   int* inner_pred, int* fit_status, char* err, size_t errlen);

/* fpls_double_cv that also returns the class scores behind the labels, for
 * margin checks and precision studies: inner_score kfold_outer x L x n x
 * n_classes (entry ((o L + l) n + i) n_classes + c: the score of class c for
 * training row i of outer fold o, predicted by its inner fold at ncomp slice
 * l) and outer_score n x n_classes (row i's refit scores at the chosen ncomp,
 * entry i n_classes + c); either may be null, not both.  Scores are the
 * latent-route Ypred rows the argmax reads (pls_predict_classes_compact_cpu,
 * fastPLS.cpp:4115-4154); rows that no fit predicts, or that took a
 * single-class fallback, hold zeros.  No counterpart in the reference, whose
 * classifier-0 CV returns labels only. */
int fpls_double_cv_scores(const void* X, int x_is_float32, int n, int p, const int* y, int n_classes,
                          const int* outer_fold, int kfold_outer, const int* inner_fold, int kfold_inner,
                          const int* ncomp, int L, int scaling, int seed, int run, int precision,
                          int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                          int* inner_pred, int* fit_status, double* inner_score, double* outer_score,
                          char* err, size_t errlen);

/* fpls_double_cv over the outer folds listed in outer_ids (n_outer_ids distinct
 * 0-based ids) only, for fold-sharded grids: the caller splits the outer folds
 * of one double CV across processes or GPUs (X replicated) and merges.  The
 * inner and refit seeds are those of the full call (they depend on the fold id,
 * not on its position in the list), and every output is written at the listed
 * folds' own entries only: best_comp[o], inner_accuracy[o + l kfold_outer],
 * outer_pred[i] for the rows of the listed folds, inner_pred[(o L + l) n + i],
 * fit_status[o kfold_inner + i0] and fit_status[kfold_outer kfold_inner + o].
 * Everything else is left as the caller set it, so disjoint lists covering all
 * folds give, merged, the outputs of one fpls_double_cv call.  The per-call row
 * Gram of the whole X is computed by every call (it does not depend on the
 * folds).  Invalid lists (empty, an id out of range, a repeated id) return
 * FPLS_ERR_ARGUMENT. */
int fpls_double_cv_outer_subset(const void* X, int x_is_float32, int n, int p, const int* y,
                                int n_classes, const int* outer_fold, int kfold_outer,
                                const int* inner_fold, int kfold_inner, const int* outer_ids,
                                int n_outer_ids, const int* ncomp, int L, int scaling, int seed, int run,
                                int precision, int batched, int* best_comp, double* inner_accuracy,
                                int* outer_pred, int* inner_pred, int* fit_status, char* err,
                                size_t errlen);

/* Gaussian response compression, regression branch: Yc = Y - colMeans(Y),
 * Z = Yc * projection (projection q x d is drawn by the caller, as R draws it
 * with rnorm), decoder = (ZᵀZ + 1e-8·mean(diag(ZᵀZ)) I)⁻¹ ZᵀYc.
 * Outputs Z n x d, y_center q, decoder d x q.  Replaces the cuda_matrix_multiply
 * calls of .prepare_gaussian_y / .gaussian_y_ridge_decoder (R/main.R:1968-2064;
 * _fastPLS_cuda_matrix_multiply, RcppExports.cpp:116). */
int fpls_gaussian_y_encode(const double* Y, int n, int q, const double* projection, int d, double* Z,
                           double* y_center, double* decoder, char* err, size_t errlen);

/* Y (w x q) = Z (w x d) * decoder + y_center: .decode_gaussian_y_matrix
 * (R/main.R:2085-2104). */
int fpls_gaussian_y_decode(const double* Z, int w, int d, const double* decoder,
                           const double* y_center, int q, double* Y, char* err, size_t errlen);

/* labels[i] = 1 + argmax_c (2 z_i·code_c − ‖code_c‖²) for class codes
 * (n_classes x d): nearest_code_classes (fastPLS.cpp:4203-4215). */
int fpls_nearest_code_classes(const double* Z, int w, int d, const double* codes, int n_classes,
                              int* labels, char* err, size_t errlen);

/* OPLS orthogonal filter: centre (scale), then per orthogonal component
 * w = u1(XᵀY), t = Xw, p = Xᵀt/tᵀt, w_o = p − w(wᵀp)/(wᵀw) normalised,
 * t_o = Xw_o, p_o = Xᵀt_o/t_oᵀt_o, X −= t_o p_oᵀ.  Outputs the filtered X
 * (n x p), mX, vX, W_orth and P_orth (p x north, first *used columns).
 * Replaces _fastPLS_opls_filter_cpp (RcppExports.cpp:523; fastPLS.cpp:4377-4460). */
int fpls_opls_filter(const double* X, int n, int p, const double* Y, int q, int north, int scaling,
                     double* Xf, double* mX, double* vX, double* W_orth, double* P_orth, int* used,
                     char* err, size_t errlen);

/* Applies a fitted OPLS filter to new rows (w x p).  Replaces
 * _fastPLS_opls_apply_filter_cpp (RcppExports.cpp:537; fastPLS.cpp:4463-4483). */
int fpls_opls_apply_filter(const double* X, int w, int p, const double* mX, const double* vX,
                           const double* W_orth, const double* P_orth, int north, double* Xf,
                           char* err, size_t errlen);

/* Label-aware PLSSVD for a factor response, with no dense one-hot Y: column
 * statistics (mX; vX from sums of squares for scaling 2), class sums of the
 * centred rows, S = class_sums - total mYᵀ (mY = class counts / n), the SVD of
 * S (svd_method 3 = exact, as R's svd(); 4 / 5 = the seeded rSVD recipe with
 * oversample / power_iters), T = X̃R, G = TᵀT and per requested ncomp k
 * C_k = (G_k + 1e-10·mean(diag G_k) I)⁻¹ diag(d_k), W_k = C_k Q_kᵀ.  ncomp is
 * capped to [1, min(n, p, m)] (ncomp_out); K = max(ncomp_out) is written to
 * *max_rank and sizes the outputs: C_latent K x K x L, W_latent K x m x L,
 * Q m x K, R p x K, mX / vX p, mY m, s K (nullable), Ttrain n x K (nullable).
 * X is n x p column-major FP64 (x_is_float32 = 0) or FP32; y_codes in 1..m.
 * Replaces .plssvd_label_aware_stream_model (R/main.R:513-655), which runs in
 * R for both backends; no .Call counterpart. */
int fpls_plssvd_label_aware(const void* X, int x_is_float32, int n, int p, const int* y_codes, int m,
                            const int* ncomp, int L, int scaling, int svd_method, int oversample,
                            int power_iters, int seed, int* ncomp_out, double* C_latent,
                            double* W_latent, double* Q, double* R, double* mX, double* vX,
                            double* mY, double* s, double* Ttrain, int* max_rank, char* err,
                            size_t errlen);

/* Label-aware PLSSVD + candidate-kNN, end to end on the device: the
 * fpls_plssvd_label_aware fit at one ncomp, training scores T C_k row-
 * normalised, class centroids, test scores ((Xtest - mX)/vX) R C_k
 * row-normalised, then fpls_candidate_knn_predict.  Xtest has the same type
 * and p as Xtrain; top_index / top_score are ntest x max(1, min(top_k, m)).
 * Composes pls(method = "simpls") on the label-aware route (R/main.R:3281-3302),
 * .fit_candidate_knn (R/main.R:795-873) and .candidate_knn_predictions
 * (R/main.R:875-950); no .Call counterpart. */
int fpls_label_aware_cknn(const void* Xtrain, int x_is_float32, int n, int p, const int* y_codes, int m,
                          const void* Xtest, int ntest, int ncomp, int scaling, int svd_method,
                          int oversample, int power_iters, int seed, int knn_k, double tau,
                          double alpha, int top_m, int top_k, int* top_index, double* top_score,
                          char* err, size_t errlen);

/* The same on matrices registered with fpls_x_upload (training rows, test rows). */
int fpls_label_aware_cknn_resident(int xtrain_handle, const int* y_codes, int m, int xtest_handle,
                                   int ncomp, int scaling, int svd_method, int oversample,
                                   int power_iters, int seed, int knn_k, double tau, double alpha,
                                   int top_m, int top_k, int* top_index, double* top_score, char* err,
                                   size_t errlen);

/* The Gaussian sketch every randomized path draws (rSVD Ω, the SIMPLS start
 * vector, the OPLS and matrix-free subspace starts), generated on the device:
 * std::mt19937(seed) + std::normal_distribution<double>(0, 1) as libstdc++
 * implements them, filling a rows x cols column-major matrix (the reference's
 * gaussian_matrix, src/svd_cpu_rsvd.cpp:10-22).  No .Call counterpart. */
int fpls_gaussian_sketch(int rows, int cols, unsigned int seed, double* out, char* err, size_t errlen);

/* Candidate-kNN score space: Tn = row_l2(T Ck) (Ck k x k, or null for T
 * itself), T n x k column-major; zero row norms are replaced by 1.  Replaces
 * the R-side .candidate_score_space + .candidate_row_l2 arithmetic
 * (R/main.R:657-662, 700-730); no .Call counterpart. */
int fpls_candidate_scores(const double* T, int n, int k, const double* Ck, double* Tn, char* err,
                          size_t errlen);

/* Class centroids of row-normalised scores: per class mean of Tn rows with
 * code c (1-based; empty classes give a zero row), then row L2.  centroids is
 * n_classes x k column-major.  Replaces .candidate_centroids
 * (R/main.R:686-698); no .Call counterpart. */
int fpls_candidate_centroids(const double* Tn, int n, int k, const int* y_codes, int n_classes,
                             double* centroids, char* err, size_t errlen);

/* Candidate-kNN prediction.  base = Ttest_norm centroidsᵀ; the top_m classes
 * by base score (ties: lower class first) are candidates; each candidate c is
 * scored local + alpha*base + bias[c], local = mx + tau*log(mean_j
 * exp((s_j - mx)/tau)) over the k' = min(knn_k, 32, |c|) largest cosine
 * similarities s_j of the test row to the training rows of class c; the
 * candidates are reranked and the best top_k kept.  Effective parameters as
 * the reference: top_k in [1, n_classes], top_m in [top_k, n_classes],
 * tau <= 0 or non-finite -> 0.2, alpha non-finite -> 0.5, candidate_bias null
 * -> zeros.  top_index (int, 1-based class codes, -1 when absent) and
 * top_score are ntest x max(1, min(top_k, n_classes)) column-major.
 * Replaces _fastPLS_candidate_knn_predict_cuda (RcppExports.cpp:148;
 * fastPLS.cpp:1653-1711, 1322-1467; lda_cuda_kernels.cu:180-243). */
int fpls_candidate_knn_predict(const double* Ttest_norm, int ntest, const double* Ttrain_norm,
                               int ntrain, int kdim, const int* y_codes, const double* centroids,
                               int n_classes, const double* candidate_bias, int top_k, int top_m,
                               int knn_k, double tau, double alpha, int* top_index,
                               double* top_score, char* err, size_t errlen);

/* C (M x N) = A (M x K) * B (K x N) through the BF16 split tensor-core kernel,
 * for callers that cannot allocate device memory (a host that runs inside
 * another runtime's fixed memory pool, a stream callback, an allocation-free
 * loop).  No counterpart in the reference.  A, B and C are DEVICE pointers
 * (column-major, FP64) owned by the caller on the calling thread's current
 * device, where the work runs; the call never changes the current device, and
 * a pointer that is not device (or managed) memory of that device is refused
 * with FPLS_ERR_ARGUMENT before anything runs.  The call allocates nothing: every temporary
 * lives in one fixed 16 MiB device array that each GPU loading the library
 * holds until exit; shapes needing more (about (M + N) x K above 2.5 million
 * elements at N <= 64) are rejected with FPLS_ERR_ARGUMENT.  The first call on
 * a device resolves that array's address (cudaGetSymbolAddress), so make it
 * before any stream capture.  Work runs on the legacy default stream and the
 * call returns after it finishes.  All calls share the one array, which keeps
 * the last call's contents: calls that overlap on the GPU (other threads,
 * other streams) race. */
int fpls_bf16x3_gemm_noalloc(const double* A, int M, int K, const double* B, int N, double* C,
                             char* err, size_t errlen);

/* Autotuning of the batched double-CV grids (off by default).  With on = 1,
 * the first fpls_double_cv / fpls_double_cv_resident call of a grid shape
 * (device, n, p, fit count, ncomp slices, largest ncomp, classes, precision,
 * scaling) times the candidate kernel configurations on its own inputs --
 * the row Gram's output tile width (128 or 64 columns), the row-space step
 * layout (512 threads x 2 rows or 256 x 8 per CTA), the merged refresh, the
 * INT8 digit slices of the K products -- each run whole, and caches for that
 * shape the fastest configuration whose chosen ncomp, outer predictions and
 * inner accuracies equal the default configuration's.  Later calls of the
 * shape (fpls_double_cv_scores included) run with it while autotuning is on;
 * with it off every call runs the default configuration.  The
 * first call costs about 3 grid runs per candidate.  No counterpart in the
 * reference. */
int fpls_set_autotune(int on, char* err, size_t errlen);

/* The tuned shapes as newline-separated JSON objects (shape, chosen
 * configuration, every candidate's device ms and whether its results equaled
 * the default's), NUL-terminated into buf (truncated to len); *needed gets
 * the full size. */
int fpls_autotune_report(char* buf, size_t len, size_t* needed, char* err, size_t errlen);

/* Registers a predictor matrix (n x p, FP64 or FP32) in device memory for
 * repeated calls; *handle identifies it until fpls_x_free.  Lets a caller keep
 * X resident across CV runs instead of re-sending it (the reference re-uploads
 * X for every fold, fastPLS.cpp:6834-6836); no counterpart in the reference. */
int fpls_x_upload(const void* X, int x_is_float32, int n, int p, int* handle, char* err,
                  size_t errlen);
int fpls_x_free(int handle, char* err, size_t errlen);

/* A registered device matrix created empty (zeros, n x p, FP32 or FP64), for
 * outputs that should stay in HBM (e.g. the filtered X of fpls_opls_filter);
 * fpls_x_device_pointer gives the device address of a registered matrix, to
 * pass where the matrix entry points accept device memory, and
 * fpls_x_download copies a registered matrix back (n x p, column-major).  With
 * them a host caller sends X across PCIe once for a whole pipeline.  No
 * counterpart in the reference. */
int fpls_x_alloc(int n, int p, int x_is_float32, int* handle, char* err, size_t errlen);
int fpls_x_device_pointer(int handle, void** ptr, char* err, size_t errlen);
int fpls_x_download(int handle, void* out, char* err, size_t errlen);

/* Session precision of the single-fit and prediction entry points
 * (fpls_pls_model1[_xprod], fpls_pls_model2_fast[_xprod], fpls_pls_model2's
 * cross-covariance, fpls_predict_*, the LDA projections, Gaussian-Y, OPLS,
 * label-aware PLSSVD): FPLS_PREC_FP64 (default, the drop-in), FPLS_PREC_BF16X3
 * or FPLS_PREC_BF16X6, where the products with the predictor block (XᵀY, X·R,
 * Xᵀ·T, the matrix-free operator passes, the response projections) with a
 * contraction of at least 256 run as split-BF16 tensor-core GEMMs with FP32
 * accumulation and FP64 sums of the partials, while the small core
 * (sketch of S, QR, eigen/SVD, Cholesky, Gram–Schmidt, LDA) stays FP64.  The
 * CV entry points take their precision as an argument instead.  No reference
 * counterpart (the reference's CUDA backend is FP64 only). */
int fpls_set_precision(int precision, char* err, size_t errlen);
int fpls_get_precision(void);

/* Page-locks (pins) an existing host buffer so that the host-buffer entry
 * points copy it to and from the device at full link speed, e.g. an R matrix
 * reused across calls; undo with fpls_host_unregister before freeing it. */
int fpls_host_register(void* ptr, size_t bytes, char* err, size_t errlen);
int fpls_host_unregister(void* ptr, char* err, size_t errlen);

/* fpls_double_cv on a registered (device-resident) predictor matrix. */
int fpls_double_cv_resident(int handle, const int* y, int n_classes, const int* outer_fold,
                            int kfold_outer, const int* inner_fold, int kfold_inner,
                            const int* ncomp, int L, int scaling, int seed, int run, int precision,
                            int batched, int* best_comp, double* inner_accuracy, int* outer_pred,
                            int* inner_pred, int* fit_status, char* err, size_t errlen);

/* fpls_double_cv_outer_subset on a registered predictor matrix. */
int fpls_double_cv_resident_outer_subset(int handle, const int* y, int n_classes, const int* outer_fold,
                                         int kfold_outer, const int* inner_fold, int kfold_inner,
                                         const int* outer_ids, int n_outer_ids, const int* ncomp, int L,
                                         int scaling, int seed, int run, int precision, int batched,
                                         int* best_comp, double* inner_accuracy, int* outer_pred,
                                         int* inner_pred, int* fit_status, char* err, size_t errlen);

/* Instrumentation: number of kernels this library has launched since load, and
 * the device time (CUDA events on the library stream) of the last call,
 * host <-> device copies included. */
long long fpls_launch_count(void);
double fpls_last_call_ms(void);

/* Profiling window of the tensor-core GEMM: enable = 1 opens it, enable = 0
 * closes it and returns the summed device time of its launches (CUDA events on
 * the launching stream), the launch count and their algorithmic bytes. */
int fpls_profile(int enable, double* gemm_ms, long long* gemm_launches, double* gemm_bytes,
                 char* err, size_t errlen);

/* Per-class view of the same profiling window: the index-th kernel class
 * recorded ("dual_step", "k_products_f64", "gram_bf16x3", "split_gemm_bf16x3"),
 * its summed launch time in ms (CUDA events around each launch), launch count
 * and the algorithmic bytes and flops of those launches.  Call after the
 * window is closed; an index past the last class returns FPLS_ERR_ARGUMENT. */
int fpls_profile_class(int index, char* name, size_t namelen, double* ms, long long* launches,
                       double* bytes, double* flops, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* FASTPLS_B200_H */
