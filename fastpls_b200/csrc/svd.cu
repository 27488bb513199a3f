#include "gaussian.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "linalg_small.cuh"
#include "svd.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <random>
#include <vector>

namespace fpls {
namespace {

__global__ void sqrt_clamp_kernel(const double* ev, double* s, int k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < k) s[i] = sqrt(fmax(ev[i], 0.0));
}

__global__ void scale_cols_inv_kernel(double* V, int rows, int cols, int ldv, const double* s) {
  const size_t total = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % rows), j = static_cast<int>(t / rows);
    V[i + (size_t)j * ldv] /= s[j];
  }
}

// Above this many singular values the exact SVD runs across the whole GPU.
constexpr int kCoopSvdMin = 96;

SvdResult exact_svd(const double* A, int rows, int cols, int lda, int k, bool left_only,
                    double* U, int ldu, double* s, double* V, int ldv) {
  Context& ctx = Context::get();
  const int max_rank = std::min(rows, cols);
  const int rank = std::min(max_rank, std::max(k, 1));
  SvdResult res;
  if (rank == 0) return res;
  double* Uw = ctx.arena.alloc_n<double>((size_t)rows * max_rank);
  double* sw = ctx.arena.alloc_n<double>(max_rank);
  double* Vw = ctx.arena.alloc_n<double>((size_t)cols * max_rank);
  if (max_rank > kCoopSvdMin) svd_jacobi_coop(rows, cols, A, lda, Uw, rows, sw, Vw, cols);
  else svd_thin(rows, cols, A, lda, Uw, rows, sw, Vw, cols);
  copy_matrix(U, ldu, Uw, rows, rows, rank);
  d2d(s, sw, rank * sizeof(double));
  if (!left_only && V) copy_matrix(V, ldv, Vw, cols, cols, rank);
  res.rank = rank;
  return res;
}

}  // namespace


SvdResult truncated_svd_device(const double* A, int rows, int cols, int lda, int k, int method,
                               int oversample, int power_iters, unsigned int seed, bool left_only,
                               bool use_full_svd, double* U, int ldu, double* s, double* V,
                               int ldv) {
  FPLS_REQUIRE(k >= 1, "truncated_svd: k must be >= 1");
  FPLS_REQUIRE(method != kSvdIrlba, "IRLBA is a CPU-only method in fastPLS; use rsvd or exact");
  const int min_dim = std::min(rows, cols);
  if (use_full_svd || min_dim < 6 || (method != kSvdCpuRsvd && method != kSvdCudaRsvd)) {
    return exact_svd(A, rows, cols, lda, k, left_only, U, ldu, s, V, ldv);
  }
  // src/svd_cpu_rsvd.cpp:95-126
  const int max_rank = min_dim;
  const int target = std::min(max_rank, std::max(k, 1));
  const int l = std::min(max_rank, target + std::max(oversample, 0));
  if (l >= max_rank) return exact_svd(A, rows, cols, lda, target, left_only, U, ldu, s, V, ldv);

  Context& ctx = Context::get();
  PhaseTimer pt("randomized SVD");
  double* Omega = ctx.arena.alloc_n<double>((size_t)cols * l);
  device_gaussian(Omega, (long long)cols * l, seed);
  pt.mark("sketch");
  double* Y = ctx.arena.alloc_n<double>((size_t)rows * l);
  double* Z = ctx.arena.alloc_n<double>((size_t)cols * l);
  double* Qz = ctx.arena.alloc_n<double>((size_t)cols * l);
  gemm(false, false, rows, l, cols, 1.0, A, lda, Omega, cols, 0.0, Y, rows);
  power_iters = std::max(power_iters, 0);
  if (power_iters == 1) {
    gemm(true, false, cols, l, rows, 1.0, A, lda, Y, rows, 0.0, Z, cols);
    gemm(false, false, rows, l, cols, 1.0, A, lda, Z, cols, 0.0, Y, rows);
  } else {
    for (int it = 0; it < power_iters; ++it) {
      gemm(true, false, cols, l, rows, 1.0, A, lda, Y, rows, 0.0, Z, cols);
      qr_orthonormalize(cols, l, Z, cols, Qz, cols);
      gemm(false, false, rows, l, cols, 1.0, A, lda, Qz, cols, 0.0, Y, rows);
    }
  }
  pt.mark("power iterations");
  // finalize_rsvd_from_sample (src/svd_cpu_rsvd.cpp:26-93)
  double* Q = ctx.arena.alloc_n<double>((size_t)rows * l);
  qr_orthonormalize(rows, l, Y, rows, Q, rows);
  pt.mark("QR of the sample");
  double* B = ctx.arena.alloc_n<double>((size_t)l * cols);
  gemm(true, false, l, cols, rows, 1.0, Q, rows, A, lda, 0.0, B, l);
  const int rank = std::min(max_rank, std::max(k, 1));
  SvdResult res;
  if (l <= cols) {
    double* G = ctx.arena.alloc_n<double>((size_t)l * l);
    double* ev = ctx.arena.alloc_n<double>(l);
    double* Uh = ctx.arena.alloc_n<double>((size_t)l * l);
    gemm(false, true, l, l, cols, 1.0, B, l, B, l, 0.0, G, l);
    eig_psd_desc(l, G, l, ev, Uh, l);
    std::vector<double> evh(l);
    d2h(evh.data(), ev, l * sizeof(double));
    ctx.sync();
    pt.mark("eig of B B^T");
    const double eps = std::numeric_limits<double>::epsilon();
    const double tol = eps * static_cast<double>(std::max(l, cols)) * std::max(evh[0], 1.0);
    int usable = 0;
    while (usable < l && evh[usable] > tol) ++usable;
    usable = std::min(usable, rank);
    if (usable > 0) {
      sqrt_clamp_kernel<<<1, 256, 0, ctx.stream>>>(ev, s, usable); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      gemm(false, false, rows, usable, l, 1.0, Q, rows, Uh, l, 0.0, U, ldu);
      if (!left_only && V) {
        gemm(true, false, cols, usable, l, 1.0, B, l, Uh, l, 0.0, V, ldv);
        scale_cols_inv_kernel<<<64, 256, 0, ctx.stream>>>(V, cols, usable, ldv, s); ::fpls::note_launch();
        FPLS_CHECK_LAUNCH();
      }
      res.rank = usable;
      pt.mark("U, V");
      pt.report();
      return res;
    }
  }
  // svd_econ(B) fallback
  const int bmr = std::min(l, cols);
  double* Ub = ctx.arena.alloc_n<double>((size_t)l * bmr);
  double* sb = ctx.arena.alloc_n<double>(bmr);
  double* Vb = ctx.arena.alloc_n<double>((size_t)cols * bmr);
  svd_thin(l, cols, B, l, Ub, l, sb, Vb, cols);
  const int r2 = std::min(rank, bmr);
  gemm(false, false, rows, r2, l, 1.0, Q, rows, Ub, l, 0.0, U, ldu);
  d2d(s, sb, r2 * sizeof(double));
  if (!left_only && V) copy_matrix(V, ldv, Vb, cols, cols, r2);
  res.rank = r2;
  return res;
}

}  // namespace fpls
