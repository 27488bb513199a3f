// Matrix-free ("xprod") PLS on the device: the cross-covariance A = X^T Y is
// never formed; it is applied as A M = X^T (Y M) and A^T M = Y^T (X M).
//
//   truncated_rsvd_crossprod_device   src/fastPLS.cpp:550-622 (+ 434-473)
//   simpls_xprod_fit                  src/fastPLS.cpp:5695-5986 with the
//                                     refresh of :936-1000 (k_block = 1)
//
// X (n x p) and Y (n x m) are the centred (scaled) device matrices.
#include "xop_split.cuh"
#include "gaussian.cuh"
#include "xprod.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "blas_f64.cuh"
#include "context.cuh"
#include "linalg_small.cuh"

namespace fpls {
namespace {

// Single-column Householder QR as arma::qr_econ: q = -sign(y0) y / ||y||
// (sign(0) = +1).  out[0] = ||y||.
__global__ void householder_q1_kernel(const double* __restrict__ y, int p, double* __restrict__ q,
                                      double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < p; i += blockDim.x) s += y[i] * y[i];
  s = block_sum(s, scratch);
  const double nrm = sqrt(s);
  const double sg = (y[0] >= 0.0) ? -1.0 : 1.0;
  const double f = (nrm > 0.0) ? sg / nrm : 0.0;
  for (int i = threadIdx.x; i < p; i += blockDim.x) q[i] = y[i] * f;
  if (threadIdx.x == 0) out[0] = nrm;
}

// t /= ||t||, r /= ||t||; out[0] = ||t||.
__global__ void normalize_pair_kernel(double* __restrict__ t, int n, double* __restrict__ r, int p,
                                      double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += t[i] * t[i];
  s = block_sum(s, scratch);
  const double nrm = sqrt(s);
  if (threadIdx.x == 0) out[0] = nrm;
  if (!(nrm > 0.0) || !isfinite(nrm)) return;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] /= nrm;
  for (int i = threadIdx.x; i < p; i += blockDim.x) r[i] /= nrm;
}

// v /= ||v||; out[0] = ||v||.
__global__ void normalize_kernel(double* __restrict__ v, int p, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < p; i += blockDim.x) s += v[i] * v[i];
  s = block_sum(s, scratch);
  const double nrm = sqrt(s);
  if (threadIdx.x == 0) out[0] = nrm;
  if (!(nrm > 0.0) || !isfinite(nrm)) return;
  for (int i = threadIdx.x; i < p; i += blockDim.x) v[i] /= nrm;
}

// A (rows x cols, lda) += x y^T
__global__ void rank1_update_kernel(double* A, int rows, int cols, int lda, const double* __restrict__ x,
                                    const double* __restrict__ y) {
  const size_t total = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % rows), j = static_cast<int>(t / rows);
    A[i + (size_t)j * lda] += x[i] * y[j];
  }
}

// M -= V[:, :a] (V[:, :a]^T M) for a single column M (p); w: a scratch.
void project_deflated(double* M, int p, const double* V, int a, double* w) {
  if (a <= 0) return;
  gemv(true, p, a, 1.0, V, p, M, 0.0, w);
  gemv(false, p, a, -1.0, V, p, w, 1.0, M);
}

}  // namespace

SvdResult truncated_rsvd_crossprod_device(const double* X, int n, int p, const double* Y, int m, int k,
                                          int oversample, int power_iters, unsigned int seed,
                                          bool use_full_svd, double* U, int ldu, double* s, double* V,
                                          int ldv) {
  Context& ctx = Context::get();
  const int max_rank = std::min(p, m);
  const int target = std::min(max_rank, std::max(k, 1));
  const int l = std::min(max_rank, target + std::max(oversample, 0));
  SvdResult res;
  if (target == 0) return res;
  if (use_full_svd || l >= max_rank) {
    double* S = ctx.arena.alloc_n<double>((size_t)p * m);
    gemm(true, false, p, m, n, 1.0, X, n, Y, n, 0.0, S, p);
    return truncated_svd_device(S, p, m, p, target, kSvdCpuRsvd, oversample, power_iters, seed, false, true,
                                U, ldu, s, V, ldv);
  }
  double* T = ctx.arena.alloc_n<double>((size_t)n * l);
  double* Ys = ctx.arena.alloc_n<double>((size_t)p * l);
  double* Zm = ctx.arena.alloc_n<double>((size_t)m * l);
  double* Qp = ctx.arena.alloc_n<double>((size_t)p * l);
  double* Qm = ctx.arena.alloc_n<double>((size_t)m * l);
  auto a_times = [&](const double* M, double* out) {  // (m x l) -> (p x l)
    xgemm(false, n, l, m, Y, n, M, m, T, n);
    xgemm(true, p, l, n, X, n, T, n, out, p);
  };
  auto at_times = [&](const double* M, double* out) {  // (p x l) -> (m x l)
    xgemm(false, n, l, p, X, n, M, p, T, n);
    xgemm(true, m, l, n, Y, n, T, n, out, m);
  };
  device_gaussian(Zm, (long long)m * l, seed);
  a_times(Zm, Ys);
  power_iters = std::max(power_iters, 0);
  if (power_iters == 1) {
    at_times(Ys, Zm);
    a_times(Zm, Ys);
  } else {
    for (int it = 0; it < power_iters; ++it) {
      at_times(Ys, Zm);
      qr_orthonormalize(m, l, Zm, m, Qm, m);
      a_times(Qm, Ys);
    }
  }
  qr_orthonormalize(p, l, Ys, p, Qp, p);
  // B = (X Q)^T Y  (l x m), then svd_econ(B)
  double* B = ctx.arena.alloc_n<double>((size_t)l * m);
  xgemm(false, n, l, p, X, n, Qp, p, T, n);
  xgemm(true, l, m, n, T, n, Y, n, B, l);
  const int r = std::min(l, m);
  double* Ub = ctx.arena.alloc_n<double>((size_t)l * r);
  double* sb = ctx.arena.alloc_n<double>(r);
  double* Vb = ctx.arena.alloc_n<double>((size_t)m * r);
  if (r > 96) svd_jacobi_coop(l, m, B, l, Ub, l, sb, Vb, m);
  else svd_thin(l, m, B, l, Ub, l, sb, Vb, m);
  const int actual = std::min(target, r);
  gemm(false, false, p, actual, l, 1.0, Qp, p, Ub, l, 0.0, U, ldu);
  d2d(s, sb, actual * sizeof(double));
  if (V) copy_matrix(V, ldv, Vb, m, m, actual);
  res.rank = actual;
  return res;
}

int simpls_xprod_fit(const double* X, int n, int p, const double* Y, int m, const int* ncomp, int L,
                     bool fit, unsigned int seed, const double* mY, double* R, double* Q, double* B,
                     double* Yfit, double* R2Y) {
  Context& ctx = Context::get();
  const int K = *std::max_element(ncomp, ncomp + L);
  int inc_power_iters = 2;  // FASTPLS_FAST_INC_ITERS, clamped to [1, 6] as the reference
  if (const char* e = std::getenv("FASTPLS_FAST_INC_ITERS")) {
    char* endp = nullptr;
    const long v = std::strtol(e, &endp, 10);
    if (endp != e) inc_power_iters = static_cast<int>(std::min(6L, std::max(1L, v)));
  }
  double* Vv = ctx.arena.alloc_n<double>((size_t)p * K);
  double* y = ctx.arena.alloc_n<double>(p);
  double* z = ctx.arena.alloc_n<double>(p);
  double* q = ctx.arena.alloc_n<double>(p);
  double* rr = ctx.arena.alloc_n<double>(p);
  double* pp = ctx.arena.alloc_n<double>(p);
  double* u = ctx.arena.alloc_n<double>(n);
  double* tt = ctx.arena.alloc_n<double>(n);
  double* w = ctx.arena.alloc_n<double>(m);
  double* qq = ctx.arena.alloc_n<double>(m);
  double* wk = ctx.arena.alloc_n<double>(std::max(K, 1));
  double* sc = ctx.arena.alloc_n<double>(4);
  double* Bcur = B ? ctx.arena.alloc_n<double>((size_t)p * m) : nullptr;
  double* Ycur = fit ? ctx.arena.alloc_n<double>((size_t)n * m) : nullptr;
  double* rq = fit ? ctx.arena.alloc_n<double>(2 * L) : nullptr;
  dzero(R, (size_t)p * K * sizeof(double));
  dzero(Q, (size_t)m * K * sizeof(double));
  dzero(Vv, (size_t)p * K * sizeof(double));
  if (Bcur) dzero(Bcur, (size_t)p * m * sizeof(double));
  if (Ycur) dzero(Ycur, (size_t)n * m * sizeof(double));
  auto scalar = [&](int i) {
    double h = 0.0;
    d2h(&h, sc + i, sizeof(double));
    ctx.sync();
    return h;
  };
  int i_out = 0, a = 0;
  for (; a < K; ++a) {
    // refresh: start vector, projections, two power iterations of A A^T
    if (a == 0) {
      device_gaussian(y, p, seed + a);
    } else {
      d2d(y, rr, p * sizeof(double));
    }
    project_deflated(y, p, Vv, a, wk);
    for (int it = 0; it < inc_power_iters; ++it) {
      d2d(z, y, p * sizeof(double));
      project_deflated(z, p, Vv, a, wk);
      gemv(false, n, p, 1.0, X, n, z, 0.0, u);
      gemv(true, n, m, 1.0, Y, n, u, 0.0, w);
      gemv(false, n, m, 1.0, Y, n, w, 0.0, u);
      gemv(true, n, p, 1.0, X, n, u, 0.0, y);
      project_deflated(y, p, Vv, a, wk);
    }
    householder_q1_kernel<<<1, 512, 0, ctx.stream>>>(y, p, q, sc); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    if (!(scalar(0) > 0.0)) break;
    project_deflated(q, p, Vv, a, wk);
    householder_q1_kernel<<<1, 512, 0, ctx.stream>>>(q, p, rr, sc); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    if (!(scalar(0) > 0.0)) break;
    // Bsmall = (X q)^T Y is 1 x m: its left singular vector is 1, so the
    // refreshed direction is the projected q itself.
    project_deflated(rr, p, Vv, a, wk);
    // append_component
    gemv(false, n, p, 1.0, X, n, rr, 0.0, tt);
    normalize_pair_kernel<<<1, 512, 0, ctx.stream>>>(tt, n, rr, p, sc + 1); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    const double tn = scalar(1);
    if (!(tn > 0.0) || !std::isfinite(tn)) break;
    gemv(true, n, p, 1.0, X, n, tt, 0.0, pp);
    gemv(true, n, m, 1.0, Y, n, tt, 0.0, qq);
    double* vv = Vv + (size_t)a * p;
    d2d(vv, pp, p * sizeof(double));
    project_deflated(vv, p, Vv, a, wk);
    normalize_kernel<<<1, 512, 0, ctx.stream>>>(vv, p, sc + 2); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    const double vn = scalar(2);
    if (!(vn > 0.0) || !std::isfinite(vn)) {
      dzero(vv, p * sizeof(double));
      break;
    }
    d2d(R + (size_t)a * p, rr, p * sizeof(double));
    d2d(Q + (size_t)a * m, qq, m * sizeof(double));
    if (Bcur) {
      rank1_update_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(Bcur, p, m, p, rr, qq); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
    while (i_out < L && a == ncomp[i_out] - 1) {
      if (B) d2d(B + (size_t)i_out * p * m, Bcur, (size_t)p * m * sizeof(double));
      if (fit) {
        // reference quirk: t q^T is accumulated only at requested ncomp values
        rank1_update_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(Ycur, n, m, n, tt, qq); ::fpls::note_launch();
        FPLS_CHECK_LAUNCH();
        rq_sums(Y, Ycur, n, m, rq + 2 * i_out);
        double* yf = Yfit + (size_t)i_out * n * m;
        d2d(yf, Ycur, (size_t)n * m * sizeof(double));
        add_row_vector(yf, n, m, n, mY);
      }
      ++i_out;
    }
  }
  // slices never reached keep zeros (the reference leaves them unset)
  for (int io = i_out; io < L; ++io) {
    if (B) dzero(B + (size_t)io * p * m, (size_t)p * m * sizeof(double));
    if (fit) dzero(Yfit + (size_t)io * n * m, (size_t)n * m * sizeof(double));
  }
  if (fit) {
    std::vector<double> h(2 * L, 0.0);
    if (i_out > 0) d2h(h.data(), rq, 2 * i_out * sizeof(double));
    ctx.sync();
    for (int io = 0; io < L; ++io) R2Y[io] = io < i_out ? 1.0 - h[2 * io] / h[2 * io + 1] : 0.0;
  } else {
    for (int io = 0; io < L; ++io) R2Y[io] = 0.0;
  }
  return a;
}

}  // namespace fpls
