// Gaussian response compression (encode / decode, class codebook decisions)
// and the OPLS orthogonal filter, on the device.
#include "../../include/fastpls_b200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "xop_split.cuh"
#include "gaussian.cuh"
#include "blas_f64.cuh"
#include "capi_util.cuh"
#include "context.cuh"
#include "fits.cuh"
#include "linalg_small.cuh"
#include "svd.cuh"

namespace fpls {
namespace {

__global__ void opls_rank1_update_kernel(double* X, int n, int p, const double* t, const double* pv) {
  const size_t total = (size_t)n * p;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total;
       k += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(k % n), j = static_cast<int>(k / n);
    X[k] -= t[i] * pv[j];
  }
}

__global__ void dot2_kernel(const double* x, const double* y, int n, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i] * y[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) *out = s;
}

// w_orth = p - w (w.p / w.w)
__global__ void orth_against_kernel(const double* pv, const double* w, int p, const double* wp_ww,
                                    double* out) {
  const double c = wp_ww[0] / wp_ww[1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p; i += gridDim.x * blockDim.x)
    out[i] = pv[i] - w[i] * c;
}

__global__ void sd_fix_kernel(double* v, int p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p; i += gridDim.x * blockDim.x)
    if (!isfinite(v[i]) || v[i] == 0.0) v[i] = 1.0;
}

__global__ void nearest_code_kernel(const double* __restrict__ S, int w, int C, const double* __restrict__ cn,
                                    int* labels) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  int best = 0;
  double bv = 2.0 * S[i] - cn[0];
  for (int c = 1; c < C; ++c) {
    const double v = 2.0 * S[i + (size_t)c * w] - cn[c];
    if (v > bv) { bv = v; best = c; }
  }
  labels[i] = best + 1;
}

__global__ void row_sqnorm_kernel(const double* A, int rows, int cols, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double s = 0.0;
  for (int j = 0; j < cols; ++j) s += A[r + (size_t)j * rows] * A[r + (size_t)j * rows];
  out[r] = s;
}

double scalar_d2h(const double* d) {
  double h = 0.0;
  d2h(&h, d, sizeof(double));
  Context::get().sync();
  return h;
}

__global__ void unit_vector_kernel(double* u, int p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p; i += gridDim.x * blockDim.x)
    u[i] = (i == 0) ? 1.0 : 0.0;
}

// Leading left singular vector u (p) of S (p x q), to rounding, as the first
// column of svd_econ(S) in the reference filter (src/fastPLS.cpp:4410-4414).
// Block subspace iteration on the small Gram matrix G (m x m, m = min(p, q))
// with a Rayleigh-Ritz step every few sweeps; it stops once the leading Ritz
// vector no longer moves (|1 - |v.v_prev|| < 1e-15), so the result does not
// depend on the spectrum's gap beyond the iteration count.  The sign is
// arbitrary; the filter is invariant to it.  A zero S yields e_1, the first
// column LAPACK returns for a zero matrix.
void leading_left_vector(const double* S, int p, int q, double* u, unsigned int seed) {
  Context& ctx = Context::get();
  const int m = std::min(p, q);
  const bool right = q <= p;  // iterate on S^T S (q x q), else on S S^T (p x p)
  if (m <= 32) {
    double* s = ctx.arena.alloc_n<double>(m);
    truncated_svd_device(S, p, q, p, 1, kSvdExact, 0, 0, seed, true, true, u, p, s, nullptr, 0);
    return;
  }
  double* G = ctx.arena.alloc_n<double>((size_t)m * m);
  // the Gram matrix by its upper tiles only (half the multiply-adds), mirrored
  if (right) gram_t_f64(S, p, q, p, G, q);
  else gram_f64(S, p, q, p, G, p);
  const int l = std::min(m, 8);
  double* Y = ctx.arena.alloc_n<double>((size_t)m * l);
  double* Q = ctx.arena.alloc_n<double>((size_t)m * l);
  double* GQ = ctx.arena.alloc_n<double>((size_t)m * l);
  double* H = ctx.arena.alloc_n<double>((size_t)l * l);
  double* ev = ctx.arena.alloc_n<double>(l);
  double* Uh = ctx.arena.alloc_n<double>((size_t)l * l);
  double* v = ctx.arena.alloc_n<double>(m);
  double* vprev = ctx.arena.alloc_n<double>(m);
  double* dots = ctx.arena.alloc_n<double>(2);
  device_gaussian(Y, (long long)m * l, seed);
  qr_orthonormalize(m, l, Y, m, Q, m);
  fill(vprev, m, 0.0);
  double lam1 = 0.0;
  const int kMaxSweeps = 2000, kCheck = 4;
  for (int it = 1; it <= kMaxSweeps; ++it) {
    gemm(false, false, m, l, m, 1.0, G, m, Q, m, 0.0, GQ, m);
    qr_orthonormalize(m, l, GQ, m, Q, m);
    if (it % kCheck) continue;
    gemm(false, false, m, l, m, 1.0, G, m, Q, m, 0.0, GQ, m);
    gemm(true, false, l, l, m, 1.0, Q, m, GQ, m, 0.0, H, l);
    eig_psd_desc(l, H, l, ev, Uh, l);
    gemv(false, m, l, 1.0, Q, m, Uh, 0.0, v);
    dot2_kernel<<<1, 512, 0, ctx.stream>>>(v, vprev, m, dots); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    double hd[2] = {0.0, 0.0};
    d2h(hd, dots, sizeof(double));
    d2h(hd + 1, ev, sizeof(double));
    ctx.sync();
    lam1 = hd[1];
    if (!(lam1 > 0.0)) break;
    if (std::fabs(1.0 - std::fabs(hd[0])) < 1e-15) break;
    d2d(vprev, v, (size_t)m * sizeof(double));
  }
  if (!(lam1 > 0.0)) {
    unit_vector_kernel<<<ceil_div(p, 256), 256, 0, ctx.stream>>>(u, p); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    return;
  }
  if (right) {
    gemv(false, p, q, 1.0, S, p, v, 0.0, u);
  } else {
    d2d(u, v, (size_t)p * sizeof(double));
  }
}

}  // namespace
}  // namespace fpls

using namespace fpls;

using capi::upload;

extern "C" {

int fpls_gaussian_y_encode(const double* Y, int n, int q, const double* projection, int d, double* Z,
                           double* y_center, double* decoder, char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && q > 0 && d > 0, "gaussian_y_encode: empty input");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dY = upload(Y, (size_t)n * q);
    const double* dG = upload(projection, (size_t)q * d);
    double* dmu = ctx.arena.alloc_n<double>(q);
    col_mean(dY, n, q, n, dmu);
    center_scale(dY, n, q, n, dmu, nullptr);
    double* dZ = ctx.arena.alloc_n<double>((size_t)n * d);
    xgemm(false, n, d, q, dY, n, dG, q, dZ, n);
    // decoder = (Z^T Z + 1e-8 mean(diag) I)^{-1} Z^T Yc
    double* ztz = ctx.arena.alloc_n<double>((size_t)d * d);
    double* rhs = ctx.arena.alloc_n<double>((size_t)d * q);
    double* dec = ctx.arena.alloc_n<double>((size_t)d * q);
    gemm(true, false, d, d, n, 1.0, dZ, n, dZ, n, 0.0, ztz, d);
    xgemm(true, d, q, n, dZ, n, dY, n, rhs, d);
    spd_solve(d, ztz, d, q, rhs, d, dec, d, ctx.d_status + 6, 1e-8);
    d2h(Z, dZ, (size_t)n * d * sizeof(double));
    d2h(y_center, dmu, q * sizeof(double));
    d2h(decoder, dec, (size_t)d * q * sizeof(double));
    int bad = 0;
    d2h(&bad, ctx.d_status + 6, sizeof(int));
    ctx.sync();
    if (bad) throw Error(kErrNumerical, "gaussian_y decoder system is singular");
  });
}

int fpls_gaussian_y_decode(const double* Z, int w, int d, const double* decoder,
                           const double* y_center, int q, double* Y, char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && d > 0 && q > 0, "gaussian_y_decode: empty input");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dZ = upload(Z, (size_t)w * d);
    const double* dD = upload(decoder, (size_t)d * q);
    const double* dmu = upload(y_center, q);
    double* dY = ctx.arena.alloc_n<double>((size_t)w * q);
    gemm(false, false, w, q, d, 1.0, dZ, w, dD, d, 0.0, dY, w);
    add_row_vector(dY, w, q, w, dmu);
    d2h(Y, dY, (size_t)w * q * sizeof(double));
    ctx.sync();
  });
}

int fpls_nearest_code_classes(const double* Z, int w, int d, const double* codes, int n_classes,
                              int* labels, char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && d > 0 && n_classes > 0, "nearest_code_classes: empty input");
    Context& ctx = Context::get();
    ctx.begin_call();
    const double* dZ = upload(Z, (size_t)w * d);
    const double* dC = upload(codes, (size_t)n_classes * d);
    double* dS = ctx.arena.alloc_n<double>((size_t)w * n_classes);
    double* cn = ctx.arena.alloc_n<double>(n_classes);
    int* dl = ctx.arena.alloc_n<int>(w);
    gemm(false, true, w, n_classes, d, 1.0, dZ, w, dC, n_classes, 0.0, dS, w);
    row_sqnorm_kernel<<<ceil_div(n_classes, 128), 128, 0, ctx.stream>>>(dC, n_classes, d, cn); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    nearest_code_kernel<<<ceil_div(w, 256), 256, 0, ctx.stream>>>(dS, w, n_classes, cn, dl); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    d2h(labels, dl, w * sizeof(int));
    ctx.sync();
  });
}

int fpls_opls_filter(const double* X, int n, int p, const double* Y, int q, int north, int scaling,
                     double* Xf, double* mX, double* vX, double* W_orth, double* P_orth, int* used,
                     char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(n > 0 && p > 0 && q > 0, "opls_filter: X and Y must be non-empty");
    FPLS_REQUIRE(north >= 0, "north must be >= 0");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dX = upload(X, (size_t)n * p);
    double* dY = upload(Y, (size_t)n * q);
    double* dmX = ctx.arena.alloc_n<double>(p);
    double* dvX = ctx.arena.alloc_n<double>(p);
    double* dmY = ctx.arena.alloc_n<double>(q);
    // Centre / scale (scaling 2 uses the (n-1) standard deviation, zeros -> 1).
    if (scaling < 3) {
      col_mean(dX, n, p, n, dmX);
      center_scale(dX, n, p, n, dmX, nullptr);
    } else {
      fill(dmX, p, 0.0);
    }
    if (scaling == 2) {
      col_sd_centered(dX, n, p, n, dvX);
      sd_fix_kernel<<<ceil_div(p, 256), 256, 0, ctx.stream>>>(dvX, p); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      center_scale(dX, n, p, n, nullptr, dvX);
    } else {
      fill(dvX, p, 1.0);
    }
    col_mean(dY, n, q, n, dmY);
    center_scale(dY, n, q, n, dmY, nullptr);
    double* S = ctx.arena.alloc_n<double>((size_t)p * q);
    double* u = ctx.arena.alloc_n<double>(p);
    double* t = ctx.arena.alloc_n<double>(n);
    double* pv = ctx.arena.alloc_n<double>(p);
    double* wo = ctx.arena.alloc_n<double>(p);
    double* to = ctx.arena.alloc_n<double>(n);
    double* po = ctx.arena.alloc_n<double>(p);
    double* sc = ctx.arena.alloc_n<double>(4);
    double* dW = ctx.arena.alloc_n<double>((size_t)p * std::max(north, 1));
    double* dP = ctx.arena.alloc_n<double>((size_t)p * std::max(north, 1));
    int k = 0;
    for (int a = 0; a < north; ++a) {
      xgemm(true, p, q, n, dX, n, dY, n, S, p);
      leading_left_vector(S, p, q, u, 1234567u + a);
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(u, u, p, sc); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      const double wn = std::sqrt(scalar_d2h(sc));
      if (!(wn > 0.0) || !std::isfinite(wn)) break;
      scale_vec(u, p, 1.0 / wn);
      gemv(false, n, p, 1.0, dX, n, u, 0.0, t);
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(t, t, n, sc); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      const double tss = scalar_d2h(sc);
      if (!(tss > 0.0) || !std::isfinite(tss)) break;
      gemv(true, n, p, 1.0 / tss, dX, n, t, 0.0, pv);
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(u, pv, p, sc); ::fpls::note_launch();
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(u, u, p, sc + 1); ::fpls::note_launch();
      orth_against_kernel<<<ceil_div(p, 256), 256, 0, ctx.stream>>>(pv, u, p, sc, wo); ::fpls::note_launch();
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(wo, wo, p, sc + 2); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      const double won = std::sqrt(scalar_d2h(sc + 2));
      if (!(won > 0.0) || !std::isfinite(won)) break;
      scale_vec(wo, p, 1.0 / won);
      gemv(false, n, p, 1.0, dX, n, wo, 0.0, to);
      dot2_kernel<<<1, 512, 0, ctx.stream>>>(to, to, n, sc + 3); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      const double toss = scalar_d2h(sc + 3);
      if (!(toss > 0.0) || !std::isfinite(toss)) break;
      gemv(true, n, p, 1.0 / toss, dX, n, to, 0.0, po);
      opls_rank1_update_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(dX, n, p, to, po); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      d2d(dW + (size_t)k * p, wo, p * sizeof(double));
      d2d(dP + (size_t)k * p, po, p * sizeof(double));
      ++k;
    }
    d2h(Xf, dX, (size_t)n * p * sizeof(double));
    d2h(mX, dmX, p * sizeof(double));
    d2h(vX, dvX, p * sizeof(double));
    if (k > 0) {
      d2h(W_orth, dW, (size_t)p * k * sizeof(double));
      d2h(P_orth, dP, (size_t)p * k * sizeof(double));
    }
    ctx.sync();
    if (used) *used = k;
  });
}

int fpls_opls_apply_filter(const double* X, int w, int p, const double* mX, const double* vX,
                           const double* W_orth, const double* P_orth, int north, double* Xf,
                           char* err, size_t errlen) {
  return capi::guarded(err, errlen, [&] {
    FPLS_REQUIRE(w > 0 && p > 0 && north >= 0, "opls_apply_filter: empty input");
    Context& ctx = Context::get();
    ctx.begin_call();
    double* dX = upload(X, (size_t)w * p);
    const double* dm = upload(mX, p);
    const double* dv = upload(vX, p);
    center_scale(dX, w, p, w, dm, dv);
    if (north > 0) {
      const double* dW = upload(W_orth, (size_t)p * north);
      const double* dP = upload(P_orth, (size_t)p * north);
      double* t = ctx.arena.alloc_n<double>(w);
      for (int a = 0; a < north; ++a) {
        gemv(false, w, p, 1.0, dX, w, dW + (size_t)a * p, 0.0, t);
        opls_rank1_update_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(dX, w, p, t, dP + (size_t)a * p); ::fpls::note_launch();
        FPLS_CHECK_LAUNCH();
      }
    }
    d2h(Xf, dX, (size_t)w * p * sizeof(double));
    ctx.sync();
  });
}

}  // extern "C"
