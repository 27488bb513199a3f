// FP64-accurate matrix products on the INT8 tensor cores: the operands are
// split into signed 7-bit digit planes with a power-of-two scale per row, the
// plane pairs are multiplied exactly (tcgen05.mma kind::i8, int32 in TMEM) and
// recombined in FP64 (Ozaki, Ogita and Oishi 2012, integer form of Ootomo,
// Ozaki and Yokota 2024).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "simpls_engine.cuh"

namespace fpls {

// Digit planes of one operand: `rows` rows of the contraction length k, each
// row scaled by scale[r] = 2^e_r and held as `slices` int8 planes (plane s at
// data + s * rows_pad * ldk), rows_pad and ldk padded to 128 with zeros.
struct OzakiPlanes {
  int8_t* data = nullptr;
  double* scale = nullptr;
  int rows = 0, rows_pad = 0, k = 0, ldk = 0, slices = 0;
  // Row stride in bytes when these planes are a column range of wider planes
  // (a view: data points at the range's first column, ldk is the range's
  // padded width); 0 when the rows are ldk apart.
  int ld = 0;
  int row_stride() const { return ld ? ld : ldk; }
};

// Slices per operand accepted by the kernel.
constexpr int kOzakiMinSlices = 4;
constexpr int kOzakiMaxSlices = 7;

OzakiPlanes ozaki_alloc(int rows, int k, int slices);

// Planes of the columns of the column-major FP64 matrix X (k x rows, ld ldx):
// row j of the planes is column j of X.  A non-finite column gets a NaN scale,
// so that its products are NaN.
void ozaki_split(const double* X, int ldx, const OzakiPlanes& out);

// C (M x N, ld ldc, FP64) = A B^T with A (M x k) and B (N x k) given as planes
// with the same slice count and contraction length.  The digit pairs whose
// levels s + t exceed slices + 1 are dropped; the result differs from the
// exact product by at most about 3 k 2^(eA_i + eB_j - 7 slices) per entry.
// a_static: A's planes were written before the kernel launched just before
// this product (so their loads may start before waiting for that kernel).
void ozaki_gemm(const OzakiPlanes& A, const OzakiPlanes& B, double* C, int ldc, bool a_static = false);

// The same product left as FP64 stream-K partials for a consumer that sums
// them (in segment order) while it reads C: entry (i, j) of C is
//   sum_{s = tile_seg[t] .. tile_seg[t+1]-1} part[(s * 64 + j % 64) * 128 + i % 128],
// t = (i / 128) * n_tiles_n + j / 64.  The buffers belong to the cached plan
// of this shape and are overwritten by the next product of the same shape.
struct OzakiPartials {
  const double* part = nullptr;
  const int* tile_seg = nullptr;
  int n_tiles_n = 0;
};
OzakiPartials ozaki_gemm_partials(const OzakiPlanes& A, const OzakiPlanes& B, bool a_static = false);

// Planes of the rows of a column-major n x p matrix (x64, or x32 widened
// exactly) with the column means `mean` subtracted (none when null): row i of
// the planes is row i of X - mean, scaled by the power of two above its largest
// magnitude.  A row with a non-finite entry gets a NaN scale.
OzakiPlanes ozaki_split_rows(const double* x64, const float* x32, int n, int p, const double* mean, int slices);

// C (n x n, ld ldc) = A A^T for A given as planes: the upper tiles on an
// L2-sharing stream-K plan (every CTA takes its share of each K chunk in turn),
// the lower triangle mirrored.  Entry (i, j) is within about
// 3 k 2^(eA_i + eA_j - 7 slices) of the exact product.
void ozaki_gram(const OzakiPlanes& A, double* C, int ldc);

// Operator over X (n x p) held as its centred rows' digit planes: times() is
// X M (the sketch product of the row-space grids) and gram() is X X^T, both on
// the INT8 tensor cores; no transposed product.
std::unique_ptr<XOperator> make_ozaki_rows_operator(const double* x64, const float* x32, const double* mean, int n,
                                                    int p, int slices);

// X (n x p) arriving in column chunks (bounds[c] .. bounds[c+1], every inner
// bound a multiple of 128): each chunk keeps its own power-of-two row scales
// (the largest |x - mean| of the row within the chunk), so its digits are
// made, and its share of X X^T taken, as soon as it has landed.
//   ozaki_rows_fill_chunk   digit planes of chunk c of X - mean (c64 / c32:
//                           the chunk's first column, ld n; mean: the chunk's
//                           column means, or null);
//   ozaki_rows_gram_chunk   the upper tiles of K (n x n, ld n) set (accumulate
//                           false) or increased by chunk c's A_c A_c^T.
// times() of the operator is X M summed over the chunks; gram() is not
// provided (the chunks' Gram calls make it).
std::unique_ptr<XOperator> make_ozaki_rows_chunked(int n, int p, int slices, const std::vector<int>& bounds);
void ozaki_rows_fill_chunk(XOperator& op, const double* c64, const float* c32, const double* mean, int c);
void ozaki_rows_gram_chunk(XOperator& op, double* K, int c, bool accumulate);

// Releases the cached stream-K plans (fpls_reset_workspace).
void ozaki_release_cache();

// Operator over a symmetric n x n FP64 matrix K, split once into planes:
// times() and t_times() are K * M through the INT8 tensor cores; gram() is not
// provided.
std::unique_ptr<XOperator> make_ozaki_sym_operator(const double* K, int n, int slices);
// K * M (n x F) of an operator made by make_ozaki_sym_operator, as partials.
OzakiPartials ozaki_sym_times_partials(XOperator& op, const double* M, int F);
// The same with the planes of M already made (rows = the F columns, k = n).
OzakiPartials ozaki_sym_partials_from_planes(XOperator& op, const OzakiPlanes& b);
// Makes the plan (and kernel attribute) of those partial products ahead of
// time, so that later calls enqueue launches only (stream capture).
void ozaki_sym_prepare_partials(XOperator& op, const OzakiPlanes& b);

// Slice count of the mixed-precision row-space products (environment
// FASTPLS_OZAKI_SLICES, else the tuned or built-in default of 5).
int ozaki_default_slices();

}  // namespace fpls
