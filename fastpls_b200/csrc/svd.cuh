// Truncated SVD on the device following the reference CPU recipe.
#pragma once

#include "common.cuh"

namespace fpls {

enum SvdMethod : int {
  kSvdIrlba = 1,      // CPU-only in the reference; rejected here
  kSvdExact = 3,
  kSvdCpuRsvd = 4,
  kSvdCudaRsvd = 5,   // follows the CPU rSVD recipe (parity target)
};


struct SvdResult {
  int rank = 0;   // columns written to U / s / V
};

// A is rows x cols (lda) on the device.  U (rows x kcap), s (kcap) and
// V (cols x kcap, i.e. Vt transposed; may be null when left_only) are device
// buffers with kcap >= min(rows, cols, max(k,1)).  Mirrors
// fastpls_svd::truncated_svd (src/svd_iface.cpp:58-116).
SvdResult truncated_svd_device(const double* A, int rows, int cols, int lda, int k, int method,
                               int oversample, int power_iters, unsigned int seed, bool left_only,
                               bool use_full_svd, double* U, int ldu, double* s, double* V,
                               int ldv);

}  // namespace fpls
