// Kernel matrices and their centring on the device.  Restates, in FP64 and
// column-major layout, kernel_matrix_cpp (src/fastPLS.cpp:4314-4340),
// center_kernel_train_cpp (src/fastPLS.cpp:4344-4357), center_kernel_test_cpp
// (src/fastPLS.cpp:4360-4375) and .fastpls_preprocess_train
// (R/main.R:2764-2779): the dot products run on the FP64 tensor cores (DMMA),
// the element-wise kernels and the centring are single passes over K.
#include "kernel_pls.cuh"

#include <cmath>

#include "blas_f64.cuh"
#include "context.cuh"

namespace fpls {
namespace {

// out[i] = sum_k X[i + k*ld]^2; one thread per row, columns read coalesced.
__global__ void row_sqnorm_kernel(const double* __restrict__ X, int n, int p, int ld, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < p; ++k) {
      const double v = X[i + static_cast<size_t>(k) * ld];
      s += v * v;
    }
    out[i] = s;
  }
}

// out[i] = mean_j K[i + j*ld] over n2 columns.
__global__ void row_mean_kernel(const double* __restrict__ K, int n1, int n2, int ld, double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < n2; ++j) s += K[i + static_cast<size_t>(j) * ld];
    out[i] = s / static_cast<double>(n2);
  }
}

// *out = mean of v[0 .. n) (one block, fixed reduction order).
__global__ void mean_kernel(const double* __restrict__ v, int n, double* __restrict__ out) {
  __shared__ double part[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) *out = t / static_cast<double>(n);
  }
}

__global__ void kernel_transform_kernel(double* __restrict__ K, int n1, int n2, int kernel, double gamma,
                                        double degree, double coef0, const double* __restrict__ s1,
                                        const double* __restrict__ s2) {
  const size_t total = static_cast<size_t>(n1) * n2;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double d = K[t];
    if (kernel == 3) {
      K[t] = pow(gamma * d + coef0, degree);
    } else {
      const int i = static_cast<int>(t % n1), j = static_cast<int>(t / n1);
      double d2 = s1[i] + s2[j] - 2.0 * d;
      if (d2 < 0.0 && d2 > -1e-10) d2 = 0.0;
      K[t] = exp(-gamma * d2);
    }
  }
}

__global__ void center_kernel_apply(double* __restrict__ K, int n1, int n2, const double* __restrict__ col_means,
                                    const double* __restrict__ row_means, const double* __restrict__ grand) {
  const size_t total = static_cast<size_t>(n1) * n2;
  const double g = *grand;
  for (size_t t = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t % n1), j = static_cast<int>(t / n1);
    K[t] = ((K[t] - col_means[j]) - row_means[i]) + g;
  }
}

__global__ void fix_scale_kernel(double* v, int p) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x)
    if (!isfinite(v[j]) || v[j] == 0.0) v[j] = 1.0;
}

int grid_of(size_t total, int threads, int sm) {
  size_t g = (total + threads - 1) / threads;
  const size_t cap = static_cast<size_t>(sm) * 16;
  return static_cast<int>(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

void kernel_matrix_device(const double* X1, int n1, const double* X2, int n2, int p, int kernel, double gamma,
                          int degree, double coef0, double* K) {
  Context& ctx = Context::get();
  FPLS_REQUIRE(kernel >= 1 && kernel <= 3, "Unknown kernel id");
  FPLS_REQUIRE(n1 > 0 && n2 > 0 && p > 0, "kernel matrix: empty input");
  const bool same = X1 == X2 && n1 == n2;
  if (same) gram_f64(X1, n1, p, n1, K, n1);
  else gemm(false, true, n1, n2, p, 1.0, X1, n1, X2, n2, 0.0, K, n1);
  if (kernel == 1) return;
  double* s1 = nullptr;
  double* s2 = nullptr;
  if (kernel == 2) {
    s1 = ctx.arena.alloc_n<double>(n1);
    row_sqnorm_kernel<<<grid_of(n1, 256, ctx.sm_count), 256, 0, ctx.stream>>>(X1, n1, p, n1, s1); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    if (same) {
      s2 = s1;
    } else {
      s2 = ctx.arena.alloc_n<double>(n2);
      row_sqnorm_kernel<<<grid_of(n2, 256, ctx.sm_count), 256, 0, ctx.stream>>>(X2, n2, p, n2, s2); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
  }
  kernel_transform_kernel<<<grid_of(static_cast<size_t>(n1) * n2, 256, ctx.sm_count), 256, 0, ctx.stream>>>(
      K, n1, n2, kernel, gamma, static_cast<double>(degree), coef0, s1, s2);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void center_kernel_train_device(double* K, int n, double* col_means, double* grand_mean) {
  Context& ctx = Context::get();
  double* row_means = ctx.arena.alloc_n<double>(n);
  col_mean(K, n, n, n, col_means);
  row_mean_kernel<<<grid_of(n, 256, ctx.sm_count), 256, 0, ctx.stream>>>(K, n, n, n, row_means); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  mean_kernel<<<1, 1024, 0, ctx.stream>>>(col_means, n, grand_mean); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  center_kernel_apply<<<grid_of(static_cast<size_t>(n) * n, 256, ctx.sm_count), 256, 0, ctx.stream>>>(
      K, n, n, col_means, row_means, grand_mean);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void center_kernel_test_device(double* Kt, int nt, int n, const double* col_means, const double* grand_mean) {
  Context& ctx = Context::get();
  double* row_means = ctx.arena.alloc_n<double>(nt);
  row_mean_kernel<<<grid_of(nt, 256, ctx.sm_count), 256, 0, ctx.stream>>>(Kt, nt, n, nt, row_means); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  center_kernel_apply<<<grid_of(static_cast<size_t>(nt) * n, 256, ctx.sm_count), 256, 0, ctx.stream>>>(
      Kt, nt, n, col_means, row_means, grand_mean);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void preprocess_kernel_x_device(double* X, int n, int p, int scaling, double* mX, double* vX) {
  Context& ctx = Context::get();
  if (scaling < 3) {
    col_mean(X, n, p, n, mX);
    center_scale(X, n, p, n, mX, nullptr);
  } else {
    fill(mX, p, 0.0);
  }
  if (scaling == 2) {
    col_sd_centered(X, n, p, n, vX);
    fix_scale_kernel<<<grid_of(p, 256, ctx.sm_count), 256, 0, ctx.stream>>>(vX, p); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    center_scale(X, n, p, n, nullptr, vX);
  } else {
    fill(vX, p, 1.0);
  }
}

}  // namespace fpls
