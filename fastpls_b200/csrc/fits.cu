#include "xop_split.cuh"
#include "gaussian.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "fits.cuh"
#include "linalg_small.cuh"
#include "svd.cuh"
#include "xprod.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fpls {
namespace {

__global__ void diag_kernel(double* D, int k, const double* s) {
  for (int t = threadIdx.x; t < k * k; t += blockDim.x) {
    const int i = t % k, j = t / k;
    D[t] = (i == j) ? s[i] : 0.0;
  }
}

// out = x . y over n (single block, deterministic)
__global__ void dot_kernel(const double* x, const double* y, int n, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i] * y[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) *out = s;
}

__global__ void sum_kernel(const double* x, int n, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) *out = s;
}

__global__ void affine_kernel(double* x, int n, double a, double b) {
  // x = (x - b) * a
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = (x[i] - b) * a;
}

// S -= v (v^T S): vS computed first (m values), then rank-1 update.
__global__ void rank1_left_kernel(double* S, int p, int m, const double* v, const double* vS) {
  const size_t total = (size_t)p * m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % p), j = static_cast<int>(t / p);
    S[t] -= v[i] * vS[j];
  }
}

// Leading left vector of S by normalised power iterations with the residual
// stopping rule of src/fastPLS.cpp:202-238.  One block; S is p x m.
__global__ void leading_left_power_kernel(const double* __restrict__ S, int p, int m,
                                          const double* __restrict__ omega, int max_iters,
                                          double tol, double* u, double* v, double* unew,
                                          int* d_flag) {
  __shared__ double scratch[32];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  // u = S * omega
  for (int i = threadIdx.x; i < p; i += blockDim.x) {
    double a = 0.0;
    for (int j = 0; j < m; ++j) a += S[i + (size_t)j * p] * omega[j];
    u[i] = a;
  }
  __syncthreads();
  double nn = 0.0;
  for (int i = threadIdx.x; i < p; i += blockDim.x) nn += u[i] * u[i];
  nn = sqrt(block_sum(nn, scratch));
  if (!(nn > 0.0) || !isfinite(nn)) {
    if (threadIdx.x == 0) atomicExch(d_flag, 1);
    return;
  }
  for (int i = threadIdx.x; i < p; i += blockDim.x) u[i] /= nn;
  __syncthreads();
  for (int it = 0; it < max_iters; ++it) {
    for (int j = 0; j < m; ++j) {
      double a = 0.0;
      for (int i = threadIdx.x; i < p; i += blockDim.x) a += S[i + (size_t)j * p] * u[i];
      a = block_sum(a, scratch);
      if (threadIdx.x == 0) v[j] = a;
    }
    __syncthreads();
    double vn = 0.0;
    for (int j = threadIdx.x; j < m; j += blockDim.x) vn += v[j] * v[j];
    vn = sqrt(block_sum(vn, scratch));
    if (!(vn > 0.0) || !isfinite(vn)) { bad = 1; }
    __syncthreads();
    if (bad) break;
    for (int i = threadIdx.x; i < p; i += blockDim.x) {
      double a = 0.0;
      for (int j = 0; j < m; ++j) a += S[i + (size_t)j * p] * (v[j] / vn);
      unew[i] = a;
    }
    __syncthreads();
    double un = 0.0;
    for (int i = threadIdx.x; i < p; i += blockDim.x) un += unew[i] * unew[i];
    un = sqrt(block_sum(un, scratch));
    if (!(un > 0.0) || !isfinite(un)) { bad = 1; }
    __syncthreads();
    if (bad) break;
    double rr = 0.0;
    for (int i = threadIdx.x; i < p; i += blockDim.x) {
      const double x = unew[i] / un;
      const double d = x - u[i];
      rr += d * d;
      u[i] = x;
    }
    rr = sqrt(block_sum(rr, scratch));
    if (rr <= tol) break;
  }
  if (bad && threadIdx.x == 0) atomicExch(d_flag, 1);
}

double read_scalar(const double* d) {
  double h = 0.0;
  d2h(&h, d, sizeof(double));
  Context::get().sync();
  return h;
}

}  // namespace

// Row-sharded centre / scale: the column sums, the sums of the centred
// columns and their squared deviations are summed over the ranks, so every
// rank centres and scales with the statistics of all rows.  With one rank the
// results are those of the unsharded path bit for bit (same loops, same order).
static void center_scale_xy_sharded(double* X, int n, int p, double* Y, int m, int scaling, double* mX,
                                    double* vX, double* mY) {
  Context& ctx = Context::get();
  const double nt = static_cast<double>(shard_rows(n));
  const int my = Y ? m : 0;
  double* buf = ctx.arena.alloc_n<double>((size_t)p + my);
  dzero(buf, ((size_t)p + my) * sizeof(double));
  if (scaling < 3) col_sum(X, n, p, n, buf);
  if (Y) col_sum(Y, n, m, n, buf + p);
  shard_sum(buf, (size_t)p + my);
  if (scaling < 3) {
    div_vec(buf, p, nt, false, mX);
    center_scale(X, n, p, n, mX, nullptr);
  } else {
    fill(mX, p, 0.0);
  }
  if (Y) {
    div_vec(buf + p, m, nt, false, mY);
    center_scale(Y, n, m, n, mY, nullptr);
  }
  if (scaling == 2) {
    // sd of the centred columns: their mean (zero up to rounding), then the
    // squared deviations from it, divided by n - 1 (two passes, as col_sd_centered)
    double* mu = ctx.arena.alloc_n<double>(p);
    col_sum(X, n, p, n, mu);
    shard_sum(mu, p);
    div_vec(mu, p, nt, false, mu);
    col_sqdev(X, n, p, n, mu, vX);
    shard_sum(vX, p);
    div_vec(vX, p, nt - 1.0, true, vX);
    center_scale(X, n, p, n, nullptr, vX);
  } else {
    fill(vX, p, 1.0);
  }
}

void center_scale_xy(double* X, int n, int p, double* Y, int m, int scaling, double* mX,
                     double* vX, double* mY) {
  if (sharded()) {
    center_scale_xy_sharded(X, n, p, Y, m, scaling, mX, vX, mY);
    return;
  }
  // src/fastPLS.cpp:4817-4834: mX = mean, X -= mX, vX = sd(X centred), X /= vX
  if (scaling < 3) {
    col_mean(X, n, p, n, mX);
    center_scale(X, n, p, n, mX, nullptr);
  } else {
    fill(mX, p, 0.0);
  }
  if (scaling == 2) {
    col_sd_centered(X, n, p, n, vX);
    center_scale(X, n, p, n, nullptr, vX);
  } else {
    fill(vX, p, 1.0);
  }
  if (Y) {
    col_mean(Y, n, m, n, mY);
    center_scale(Y, n, m, n, mY, nullptr);
  }
}

int plssvd_fit_centered(const double* X, int n, int p, const double* Y, int m, const int* ncomp,
                        int L, int K0, const FitOptions& opt, const double* mY, PlssvdOut out) {
  Context& ctx = Context::get();
  PhaseTimer pt("PLSSVD fit");
  const int max_rank = static_cast<int>(std::min<long long>(shard_rows(n), std::min(p, m)));
  double* S = nullptr;
  if (!opt.xprod) {
    S = ctx.arena.alloc_n<double>((size_t)p * m);
    xgemm(true, p, m, n, X, n, Y, n, S, p);
    shard_sum(S, (size_t)p * m);
  }
  pt.mark("S = X^T Y");
  int thr = 32;
  if (const char* e = std::getenv("FASTPLS_PLSSVD_SMALL_EXACT_MAX_RANK")) {
    char* endp = nullptr;
    long v = std::strtol(e, &endp, 10);
    if (endp != e) thr = static_cast<int>(std::min(512L, std::max(5L, v)));
  }
  const bool small_exact = max_rank <= thr;
  dzero(out.R, (size_t)p * K0 * sizeof(double));
  dzero(out.Q, (size_t)m * K0 * sizeof(double));
  dzero(out.s, (size_t)K0 * sizeof(double));
  SvdResult sr = opt.xprod
                     ? truncated_rsvd_crossprod_device(X, n, p, Y, m, K0, opt.oversample, opt.power_iters,
                                                       opt.seed, small_exact, out.R, p, out.s, out.Q, m)
                     : truncated_svd_device(S, p, m, p, K0, opt.svd_method, opt.oversample,
                                            opt.power_iters, opt.seed, false, small_exact, out.R, p,
                                            out.s, out.Q, m);
  pt.mark("SVD of S");
  int keff = std::min(K0, sr.rank);
  FPLS_REQUIRE(keff >= 1, "plssvd effective rank is < 1 after SVD");
  dzero(out.T, (size_t)n * K0 * sizeof(double));
  xgemm(false, n, keff, p, X, n, out.R, p, out.T, n);
  double* G = ctx.arena.alloc_n<double>((size_t)keff * keff);
  gemm(true, false, keff, keff, n, 1.0, out.T, n, out.T, n, 0.0, G, keff);
  shard_sum(G, (size_t)keff * keff);
  pt.mark("T = X R, G");
  dzero(out.C_latent, (size_t)K0 * K0 * L * sizeof(double));
  dzero(out.W_latent, (size_t)K0 * m * L * sizeof(double));
  double* D = ctx.arena.alloc_n<double>((size_t)keff * keff);
  double* Cw = ctx.arena.alloc_n<double>((size_t)keff * keff);
  double* Wa = ctx.arena.alloc_n<double>((size_t)keff * m);
  double* Yf = opt.fit ? ctx.arena.alloc_n<double>((size_t)n * m) : nullptr;
  double* rq = ctx.arena.alloc_n<double>(2 * L);
  const double* rq_mu = opt.fit ? shard_rq_means(Y, n, m) : nullptr;
  for (int a = 0; a < L; ++a) {
    const int mc = std::min(ncomp[a], keff);
    diag_kernel<<<1, 256, 0, ctx.stream>>>(D, mc, out.s); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    // G_a is the leading mc x mc block of G (leading dimension keff).
    spd_solve(mc, G, keff, mc, D, mc, Cw, mc, ctx.d_status + 2);
    copy_matrix(out.C_latent + (size_t)a * K0 * K0, K0, Cw, mc, mc, mc);
    // W_a = C V_a^T  (mc x m)
    gemm(false, true, mc, m, mc, 1.0, Cw, mc, out.Q, m, 0.0, Wa, mc);
    copy_matrix(out.W_latent + (size_t)a * K0 * m, K0, Wa, mc, mc, m);
    if (out.B) gemm(false, false, p, m, mc, 1.0, out.R, p, Wa, mc, 0.0, out.B + (size_t)a * p * m, p);
    if (opt.fit) {
      gemm(false, false, n, m, mc, 1.0, out.T, n, Wa, mc, 0.0, Yf, n);
      rq_sums(Y, Yf, n, m, rq + 2 * a, rq_mu);
      add_row_vector(Yf, n, m, n, mY);
      d2d(out.Yfit + (size_t)a * n * m, Yf, (size_t)n * m * sizeof(double));
    }
  }
  if (opt.fit) {
    shard_sum(rq, 2 * (size_t)L);
    std::vector<double> h(2 * L);
    d2h(h.data(), rq, 2 * L * sizeof(double));
    ctx.sync();
    for (int a = 0; a < L; ++a) out.R2Y[a] = 1.0 - h[2 * a] / h[2 * a + 1];
  } else {
    for (int a = 0; a < L; ++a) out.R2Y[a] = 0.0;
  }
  int st = 0;
  d2h(&st, ctx.d_status + 2, sizeof(int));
  ctx.sync();
  pt.mark("latent solves");
  pt.report();
  if (st) throw Error(kErrNumerical, "plssvd latent solve failed");
  return keff;
}

int simpls_classic_fit(const double* X, int n, int p, const double* Y, int m, const double* Yraw,
                       const int* ncomp, int L, const FitOptions& opt, const double* mY,
                       SimplsOut out) {
  Context& ctx = Context::get();
  int max_ncomp = 0;
  for (int i = 0; i < L; ++i) max_ncomp = std::max(max_ncomp, ncomp[i]);
  double* S = ctx.arena.alloc_n<double>((size_t)p * m);
  xgemm(true, p, m, n, X, n, Y, n, S, p);
  double* V = ctx.arena.alloc_n<double>((size_t)p * max_ncomp);
  double* t = ctx.arena.alloc_n<double>(n);
  double* pp = ctx.arena.alloc_n<double>(p);
  double* vv = ctx.arena.alloc_n<double>(p);
  double* w = ctx.arena.alloc_n<double>(max_ncomp + 1);
  double* vS = ctx.arena.alloc_n<double>(m);
  double* sc = ctx.arena.alloc_n<double>(4);
  double* u = ctx.arena.alloc_n<double>(p);
  double* u2 = ctx.arena.alloc_n<double>(p);
  double* vtmp = ctx.arena.alloc_n<double>(m);
  double* omega = ctx.arena.alloc_n<double>(m);
  const int kcap = std::min(p, m);
  double* Us = ctx.arena.alloc_n<double>((size_t)p * kcap);
  double* ss = ctx.arena.alloc_n<double>(kcap);
  double* Yf = opt.fit ? ctx.arena.alloc_n<double>((size_t)n * m) : nullptr;
  dzero(out.R, (size_t)p * max_ncomp * sizeof(double));
  dzero(out.Q, (size_t)m * max_ncomp * sizeof(double));
  if (out.T) dzero(out.T, (size_t)n * max_ncomp * sizeof(double));
  if (out.P) dzero(out.P, (size_t)p * max_ncomp * sizeof(double));
  dzero(V, (size_t)p * max_ncomp * sizeof(double));
  const bool rsvd = (opt.svd_method == kSvdCpuRsvd || opt.svd_method == kSvdCudaRsvd);
  int max_iters = std::max(opt.power_iters + 2, 4);
  if (const char* e = std::getenv("FASTPLS_LEADING_LEFT_MAX_ITERS")) {
    char* endp = nullptr;
    long v = std::strtol(e, &endp, 10);
    if (endp != e) max_iters = static_cast<int>(std::min(64L, std::max(1L, v)));
  }
  int i_out = 0;
  int done = 0;
  for (int a = 0; a < max_ncomp; ++a) {
    const double* rr_src = nullptr;
    if (rsvd) {
      device_gaussian(omega, m, opt.seed + a + std::max(opt.oversample, 0));
      dzero(ctx.d_status + 3, sizeof(int));
      leading_left_power_kernel<<<1, 1024, 0, ctx.stream>>>(S, p, m, omega, max_iters,
                                                            std::max(opt.svds_tol, 1e-8), u, vtmp,
                                                            u2, ctx.d_status + 3); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      int bad = 0;
      d2h(&bad, ctx.d_status + 3, sizeof(int));
      ctx.sync();
      if (bad) break;
      rr_src = u;
    } else {
      SvdResult r = truncated_svd_device(S, p, m, p, 1, opt.svd_method, opt.oversample,
                                         opt.power_iters, opt.seed + a, true, false, Us, p, ss,
                                         nullptr, 0);
      if (r.rank < 1) break;
      rr_src = Us;
    }
    double* rr = out.R + (size_t)a * p;
    d2d(rr, rr_src, p * sizeof(double));
    // tt = X rr, centred, normalised
    gemv(false, n, p, 1.0, X, n, rr, 0.0, t);
    sum_kernel<<<1, 512, 0, ctx.stream>>>(t, n, sc); ::fpls::note_launch();
    const double mt = read_scalar(sc) / static_cast<double>(n);
    affine_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(t, n, 1.0, mt); ::fpls::note_launch();
    dot_kernel<<<1, 512, 0, ctx.stream>>>(t, t, n, sc); ::fpls::note_launch();
    const double tnorm = std::sqrt(read_scalar(sc));
    affine_kernel<<<ceil_div(n, 256), 256, 0, ctx.stream>>>(t, n, 1.0 / tnorm, 0.0); ::fpls::note_launch();
    scale_vec(rr, p, 1.0 / tnorm);
    FPLS_CHECK_LAUNCH();
    gemv(true, n, p, 1.0, X, n, t, 0.0, pp);
    gemv(true, n, m, 1.0, Y, n, t, 0.0, out.Q + (size_t)a * m);
    d2d(vv, pp, p * sizeof(double));
    if (a > 0) {
      gemv(true, p, a, 1.0, V, p, pp, 0.0, w);
      gemv(false, p, a, -1.0, V, p, w, 1.0, vv);
    }
    dot_kernel<<<1, 512, 0, ctx.stream>>>(vv, vv, p, sc); ::fpls::note_launch();
    const double vn = std::sqrt(read_scalar(sc));
    scale_vec(vv, p, 1.0 / vn);
    gemv(true, p, m, 1.0, S, p, vv, 0.0, vS);
    rank1_left_kernel<<<256, 256, 0, ctx.stream>>>(S, p, m, vv, vS); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    d2d(V + (size_t)a * p, vv, p * sizeof(double));
    if (out.T) d2d(out.T + (size_t)a * n, t, n * sizeof(double));
    if (out.P) d2d(out.P + (size_t)a * p, pp, p * sizeof(double));
    done = a + 1;
    if (i_out < L && a == ncomp[i_out] - 1) {
      if (out.B) gemm(false, true, p, m, a + 1, 1.0, out.R, p, out.Q, m, 0.0, out.B + (size_t)i_out * p * m, p);
      if (opt.fit) {
        gemm(false, true, n, m, a + 1, 1.0, out.T, n, out.Q, m, 0.0, Yf, n);
        add_row_vector(Yf, n, m, n, mY);
        d2d(out.Yfit + (size_t)i_out * n * m, Yf, (size_t)n * m * sizeof(double));
        rq_sums(Yraw, Yf, n, m, sc);
        double h[2];
        d2h(h, sc, 2 * sizeof(double));
        ctx.sync();
        out.R2Y[i_out] = 1.0 - h[0] / h[1];
      }
      ++i_out;
    }
  }
  for (int i = 0; i < L; ++i)
    if (!opt.fit) out.R2Y[i] = 0.0;
  return done;
}

}  // namespace fpls
