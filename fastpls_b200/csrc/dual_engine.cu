#include "dual_engine.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "blas_f64.cuh"
#include "context.cuh"

namespace fpls {
namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxN = 8192;     // n-vectors staged in shared memory
constexpr int kMaxM = 128;
constexpr int kMaxK = 256;

struct DualEng {
  int n, m, F, K, iters, m1, center;
  const double* x0;
  const double* XOmega;
  const uint8_t* mask;
  const int* labels;
  const double* mY_all;
  const double* dY;
  const int* ntrain;
  double* CS;    // F x n x m
  double* KCS;   // F x n x m
  double* CV;    // F x n x K
  double* KCV;   // F x n x K
  double* Kcy;   // F x n   K image of the warm start r / ||t|| of the last component
  double* cp;    // n x F   loading coefficients (input of the K product)
  double* Gp;    // n x F   K cp
  double* scal;  // F x 2   ||t||, sum(t)
  double* qs;    // F x m   Y^T t
  double* Q;
  double* tnorm;
  double* Tkeep;
  int* ncomp_done;
  int* status;
};

constexpr int kRows = kMaxN / kThreads;   // rows of an n-vector held per thread

// out[j] = sum_i M[i + j*ld] * xs[i] for j < ncols, xs in shared memory.  With
// fewer columns than warps, several warps split the rows of one column; every
// lane keeps four independent partial sums.  Ends with a barrier.
__device__ void dots_smem(const double* __restrict__ M, size_t ld, int ncols, const double* xs, int rows,
                          double* out) {
  __shared__ double red[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = ncols >= kWarps ? 1 : kWarps / max(ncols, 1);   // warps per column
  const int cols_per_pass = kWarps / g;
  for (int j0 = 0; j0 < ncols; j0 += cols_per_pass) {
    const int j = j0 + warp / g, sub = warp % g;
    double acc = 0.0;
    if (j < ncols && warp / g < cols_per_pass) {
      const double* col = M + (size_t)j * ld;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      const int step = 32 * g;
      int r = sub * 32 + lane;
      for (; r + 3 * step < rows; r += 4 * step) {
        a0 += col[r] * xs[r];
        a1 += col[r + step] * xs[r + step];
        a2 += col[r + 2 * step] * xs[r + 2 * step];
        a3 += col[r + 3 * step] * xs[r + 3 * step];
      }
      for (; r < rows; r += step) a0 += col[r] * xs[r];
      acc = warp_sum((a0 + a1) + (a2 + a3));
    }
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x < cols_per_pass && j0 + threadIdx.x < ncols) {
      double t = 0.0;
      for (int u = 0; u < g; ++u) t += red[threadIdx.x * g + u];
      out[j0 + threadIdx.x] = t;
    }
    __syncthreads();
  }
}

// Block sum of up to 4 values per thread; result broadcast to every thread.
__device__ void block_sum4(double (&v)[4], int count) {
  __shared__ double red[kWarps][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = 0; k < count; ++k) {
    const double w = warp_sum(v[k]);
    if (lane == 0) red[warp][k] = w;
  }
  __syncthreads();
  for (int k = 0; k < count; ++k) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[w][k];
    v[k] = s;
  }
  __syncthreads();
}

// C_S of every fit: mask_f * (onehot(label) - (mY_all + dY_f)).
__global__ void k_dual_cs0(DualEng e) {
  const size_t total = (size_t)e.F * e.n * e.m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % e.n);
    const size_t col = t / e.n;
    const int f = static_cast<int>(col / e.m), j = static_cast<int>(col % e.m);
    double v = 0.0;
    if (e.mask[(size_t)f * e.n + i]) {
      const double off = e.mY_all[j] + (e.dY ? e.dY[(size_t)f * e.m + j] : 0.0);
      v = (e.labels[i] == j ? 1.0 : 0.0) - off;
    }
    e.CS[t] = v;
  }
}

// Refresh (power iterations of S S^T from the sketch or the warm start),
// Householder normalisation, scores t = X_f r, q = Y^T t, and the loading
// coefficients c_p for the K product.
__device__ bool dual_a(const DualEng& e, int a, double* sm) {
  double* vy = sm;            // n: c_y, later t
  double* vk = sm + e.n;      // n: K c_y, later K c_r
  __shared__ double z[kMaxM];
  __shared__ double zq[kMaxM];
  const int f = blockIdx.x;
  if (e.status[f]) return false;
  const int n = e.n, m = e.m;
  const double* CS = e.CS + (size_t)f * n * m;
  const double* KCS = e.KCS + (size_t)f * n * m;
  const uint8_t* mk = e.mask + (size_t)f * n;
  int steps = e.iters;
  if (e.m1) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      vy[i] = CS[i];
      vk[i] = KCS[i];
    }
    __syncthreads();
    steps = 0;
  } else {
    // z = S^T (start): the sketch through X Omega at the first component,
    // else the warm start r_{a-1} through its K image.
    const double* src = (a == 0) ? e.XOmega + (size_t)f * n : e.Kcy + (size_t)f * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) vk[i] = src[i];
    __syncthreads();
    dots_smem(CS, n, m, vk, n, z);
  }
  for (int it = 0; it < steps; ++it) {
    // y = S z: c_y = C_S z, K c_y = (K C_S) z (rows held in registers)
    double c[kRows], k[kRows];
#pragma unroll
    for (int r = 0; r < kRows; ++r) c[r] = k[r] = 0.0;
    for (int j = 0; j < m; ++j) {
      const double zj = z[j];
      const double* cs = CS + (size_t)j * n;
      const double* ks = KCS + (size_t)j * n;
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int i = threadIdx.x + r * kThreads;
        if (i < n) {
          c[r] += cs[i] * zj;
          k[r] += ks[i] * zj;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int i = threadIdx.x + r * kThreads;
      if (i < n) {
        vy[i] = c[r];
        vk[i] = k[r];
      }
    }
    __syncthreads();
    if (it + 1 < steps) dots_smem(CS, n, m, vk, n, z);
  }
  // ||y||^2 = c_y^T K c_y, y[0] = Xc[:,0]^T c_y, and the train-row count
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s[0] += vy[i] * vk[i];
    s[1] += e.x0[i] * vy[i];
  }
  block_sum4(s, 2);
  const double nrm = sqrt(s[0]);
  if (!(nrm > 0.0) || !isfinite(nrm)) {
    if (threadIdx.x == 0) e.status[f] = 1;
    return false;
  }
  const double sg = ((s[1] >= 0.0) ? -1.0 : 1.0) / nrm;
  const double nf = static_cast<double>(e.ntrain[f]);
  // U = X r = sg * K c_y; c = mean of U over the train rows
  double u[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (mk[i]) u[0] += sg * vk[i];
  block_sum4(u, 1);
  const double cmean = e.center ? u[0] / nf : 0.0;
  double* keep = e.Tkeep ? e.Tkeep + ((size_t)f * e.K + a) * n : nullptr;
  for (int j = threadIdx.x; j < m; j += blockDim.x) zq[j] = 0.0;
  __syncthreads();
  double t2[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double U = sg * vk[i];
    const double uc = U - cmean;
    const double t = mk[i] ? uc : 0.0;
    if (keep) keep[i] = uc;
    t2[0] += t * t;
    t2[1] += t;
    if (t != 0.0) atomicAdd(&zq[e.labels[i]], t);
    vk[i] = U;
    vy[i] = t;
  }
  block_sum4(t2, 2);
  const double tn = sqrt(t2[0]);
  const double st = t2[1];
  if (!(tn > 0.0) || !isfinite(tn)) {
    if (threadIdx.x == 0) e.status[f] = 1;
    return false;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    e.cp[(size_t)f * n + i] = (vy[i] - ((e.center && mk[i]) ? st / nf : 0.0)) / tn;
    e.Kcy[(size_t)f * n + i] = vk[i] / tn;
  }
  for (int j = threadIdx.x; j < m; j += blockDim.x) e.qs[(size_t)f * m + j] = zq[j];
  if (threadIdx.x == 0) {
    e.scal[2 * f] = tn;
    e.scal[2 * f + 1] = st;
  }
  return true;
}

// Gram-Schmidt of the loading against the earlier ones in K-coordinates,
// normalisation, rank-1 deflation of C_S and K C_S, and the component outputs.
__device__ bool dual_b(const DualEng& e, int a, double* sm) {
  double* g = sm;             // n: K c_p, then K c_v
  double* c = sm + e.n;       // n: c_p, then c_v
  __shared__ double w[kMaxK];
  __shared__ double vs[kMaxM];
  const int f = blockIdx.x;
  if (e.status[f]) return false;
  const int n = e.n, m = e.m, K = e.K;
  double* CV = e.CV + (size_t)f * n * K;
  double* KCV = e.KCV + (size_t)f * n * K;
  double* CS = e.CS + (size_t)f * n * m;
  double* KCS = e.KCS + (size_t)f * n * m;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    g[i] = e.Gp[(size_t)f * n + i];
    c[i] = e.cp[(size_t)f * n + i];
  }
  __syncthreads();
  if (a > 0) dots_smem(CV, n, a, g, n, w);   // V^T p = C_V^T K c_p
  double cv[kRows], kv[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const int i = threadIdx.x + r * kThreads;
    cv[r] = i < n ? c[i] : 0.0;
    kv[r] = i < n ? g[i] : 0.0;
  }
  for (int l = 0; l < a; ++l) {
    const double wl = w[l];
    const double* vc = CV + (size_t)l * n;
    const double* vk = KCV + (size_t)l * n;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int i = threadIdx.x + r * kThreads;
      if (i < n) {
        cv[r] -= vc[i] * wl;
        kv[r] -= vk[i] * wl;
      }
    }
  }
  double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const int i = threadIdx.x + r * kThreads;
    if (i < n) {
      c[i] = cv[r];
      g[i] = kv[r];
      s[0] += cv[r] * kv[r];
    }
  }
  block_sum4(s, 1);
  const double vn = sqrt(s[0]);
  if (!(vn > 0.0) || !isfinite(vn)) {
    if (threadIdx.x == 0) e.status[f] = 1;
    return false;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    c[i] /= vn;
    g[i] /= vn;
    CV[i + (size_t)a * n] = c[i];
    KCV[i + (size_t)a * n] = g[i];
  }
  __syncthreads();
  dots_smem(CS, n, m, g, n, vs);             // S^T v = C_S^T K c_v
  for (int j = 0; j < m; ++j) {
    const double vj = vs[j];
    double* cs = CS + (size_t)j * n;
    double* ks = KCS + (size_t)j * n;
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      const int i = threadIdx.x + r * kThreads;
      if (i < n) {
        cs[i] -= c[i] * vj;
        ks[i] -= g[i] * vj;
      }
    }
  }
  const double tn = e.scal[2 * f], st = e.scal[2 * f + 1];
  double* Qcol = e.Q + ((size_t)f * K + a) * m;
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const double off = e.mY_all[j] + (e.dY ? e.dY[(size_t)f * m + j] : 0.0);
    Qcol[j] = (e.qs[(size_t)f * m + j] - off * st) / tn;
  }
  if (threadIdx.x == 0) {
    e.tnorm[(size_t)f * K + a] = tn;
    e.ncomp_done[f] = a + 1;
  }
  return true;
}

// One launch per component boundary: the Gram-Schmidt / deflation of
// component a - 1 and then the refresh / scores of component a, per fit.
__global__ void __launch_bounds__(kThreads) k_dual_step(DualEng e, int a) {
  extern __shared__ double sm[];
  if (a > 0 && !dual_b(e, a - 1, sm)) return;
  if (a < e.K) {
    __syncthreads();
    dual_a(e, a, sm);
  }
}

__global__ void symmetrize_kernel(double* K, int n) {
  const size_t total = (size_t)n * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % n), j = static_cast<int>(t / n);
    if (i < j) {
      const double v = 0.5 * (K[t] + K[j + (size_t)i * n]);
      K[t] = v;
      K[j + (size_t)i * n] = v;
    }
  }
}

}  // namespace

void symmetrize(double* K, int n) {
  Context& ctx = Context::get();
  symmetrize_kernel<<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(K, n); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

bool dual_engine_applies(int n, int p, int m, int K) {
  if (const char* e = std::getenv("FASTPLS_DUAL"))
    if (e[0] == '0') return false;
  return n >= 2 && n <= kMaxN && 2 * n <= p && m <= kMaxM && K <= kMaxK;
}

void dual_simpls_run(const DualBatch& b) {
  Context& ctx = Context::get();
  Arena& ar = ctx.arena;
  FPLS_REQUIRE(dual_engine_applies(b.n, 2 * b.n, b.m, b.K), "dual SIMPLS: shape outside its limits");
  DualEng e{};
  e.n = b.n; e.m = b.m; e.F = b.F; e.K = b.K;
  e.iters = b.m1_mode ? 0 : std::max(b.power_iters, 0);
  e.m1 = b.m1_mode ? 1 : 0;
  e.center = b.center ? 1 : 0;
  e.x0 = b.x0; e.XOmega = b.XOmega; e.mask = b.mask; e.labels = b.labels; e.mY_all = b.mY_all; e.dY = b.dY;
  e.Q = b.Q; e.tnorm = b.tnorm; e.Tkeep = b.Tkeep; e.ncomp_done = b.ncomp_done; e.status = b.status;
  const size_t F = b.F, n = b.n, m = b.m, K = b.K;
  e.CS = ar.alloc_n<double>(F * n * m);
  e.KCS = ar.alloc_n<double>(F * n * m);
  e.CV = ar.alloc_n<double>(F * n * K);
  e.KCV = ar.alloc_n<double>(F * n * K);
  e.Kcy = ar.alloc_n<double>(F * n);
  e.cp = ar.alloc_n<double>(F * n);
  e.Gp = ar.alloc_n<double>(F * n);
  e.scal = ar.alloc_n<double>(2 * F);
  e.qs = ar.alloc_n<double>(F * m);
  e.ntrain = b.ntrain;
  dzero(b.status, F * sizeof(int));
  dzero(b.ncomp_done, F * sizeof(int));
  dzero(b.Q, F * m * K * sizeof(double));
  dzero(b.tnorm, F * K * sizeof(double));
  cudaStream_t st = ctx.stream;
  k_dual_cs0<<<2 * ctx.sm_count, 256, 0, st>>>(e); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  b.Kop->times(e.CS, static_cast<int>(F * m), e.KCS);   // K C_S for every fit
  const size_t smem = 2 * n * sizeof(double);
  static bool attr = false;
  if (!attr) {
    FPLS_CUDA(cudaFuncSetAttribute(k_dual_step, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kMaxN * 8));
    attr = true;
  }
  PhaseTimer pt("dual SIMPLS engine");
  for (int a = 0; a <= b.K; ++a) {
    k_dual_step<<<b.F, kThreads, smem, st>>>(e, a); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    pt.mark("per-fit steps");
    if (a == b.K) break;
    b.Kop->times(e.cp, b.F, e.Gp);
    pt.mark("K products");
  }
  pt.report();
}

}  // namespace fpls
