// Mixed-precision predictor operator: X held once as BF16 hi/lo pairs (in both
// row- and column-major order), both passes run as three-product BF16 GEMMs
// (hi*hi + hi*lo + lo*hi) on the tcgen05 tensor cores with FP32 accumulation in
// TMEM and FP64 reduction of the K-split partials.
#pragma once

#include <memory>

#include "simpls_engine.cuh"

namespace fpls {

// Frees the per-shape GEMM plans kept on the device (fpls_reset_workspace).
void split_gemm_release_cache();

// Builds the split operator from an FP64 device matrix (n x p, ld n); without
// need_t only the row-major copy (for times() and gram()) is kept.  planes: 2
// (BF16x3: hi, lo, three products) or 3 (BF16x6: hi, mid, lo, six products).
std::unique_ptr<XOperator> make_split_operator(const double* X, int n, int p, bool need_t = true,
                                               int planes = 2);

// Row-major planes only (times() and gram()), split straight from the
// caller's n x p matrix (ld n; x64 or, when x64 is null, x32) with the column
// means `mean` (or nothing, when null) subtracted in FP64 on the way: the same
// planes as centring an FP64 copy and splitting it, without the copy.
std::unique_ptr<XOperator> make_split_operator_centered(const double* x64, const float* x32, const double* mean,
                                                        int n, int p, int planes = 2);

// The same operator filled column chunk by column chunk (so that the upload
// of X overlaps its split and its row Gram): planes allocated only;
// split_operator_fill_columns writes columns [j0, j1) (j0 a multiple of 8) from
// the chunk X[:, j0:j1] (device, ld n) minus mean[0 .. j1-j0) (or nothing);
// split_operator_gram_columns sets (accumulate false) or adds to the upper
// tiles of K (n x n) the chunk's X[:, j0:j1] X[:, j0:j1]^T; the lower triangle
// is filled by mirror_upper_triangle once all chunks are in.
std::unique_ptr<XOperator> make_split_operator_chunked(int n, int p, int planes = 2);
void split_operator_fill_columns(XOperator& op, const double* x64, const float* x32, const double* mean, int j0,
                                 int j1);
void split_operator_gram_columns(XOperator& op, double* K, int j0, int j1, bool accumulate);
void mirror_upper_triangle(double* K, int n);

// C (M x N) = op(A) B with op(A) = A (M x K) or A^T (A is K x M), B K x N,
// column-major device matrices.  In the mixed precision modes (session setting
// FPLS_PREC_BF16X3 or FPLS_PREC_BF16X6) products with a contraction of at
// least 256 and 1e7 multiply-adds run as the split BF16 tensor-core GEMM (two
// or three planes per operand, FP32 accumulation in segments, FP64
// reduction); everything else, and every product in the FP64 mode, runs the
// FP64 GEMM.
void xgemm(bool transA, int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
           int ldc);

// Plain C = A (M x K) * B^T (N x K) with A, B given as FP64 and split on the fly
// into BF16 hi/lo; used by tests of the tensor-core kernel.  C is M x N (ld M).
void split_gemm_test(const double* A, const double* B, int M, int N, int K, double* C);

// Same product with every temporary (split operands, stream-K tables and
// partials) placed in a caller-provided device buffer, on stream `st`, with no
// allocation.  Throws when the shape needs more than scratch_bytes (see
// split_gemm_scratch_need).  A, B, C: device, column-major (M x K, K x N, M x N).
size_t split_gemm_scratch_need(int M, int N, int K, int sm_count);
void split_gemm_in_scratch(const double* A, const double* B, int M, int N, int K, double* C,
                           void* scratch, size_t scratch_bytes, int* err, cudaStream_t st,
                           int sm_count);

}  // namespace fpls
