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
// need_t only the row-major copy (for times() and gram()) is kept.
std::unique_ptr<XOperator> make_split_operator(const double* X, int n, int p, bool need_t = true);

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
