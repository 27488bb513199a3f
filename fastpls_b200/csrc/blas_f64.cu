#include "blas_f64.cuh"
#include "context.cuh"

namespace fpls {
namespace {

constexpr int BM = 64;
constexpr int BN = 64;
constexpr int BK = 16;
constexpr int PAD = 4;  // row stride of 68 doubles keeps the DMMA fragment loads conflict-free
constexpr int GEMM_THREADS = 128;

// Tile loader: fetches the BK x BM slice of op(A) (or BK x BN of op(B)) for the
// k-block starting at k0 into registers; out-of-range elements read as zero.
template <bool KContig>
__device__ __forceinline__ void load_tile(double (&r)[8], const double* __restrict__ P, int ld,
                                          int mn0, int k0, int MN, int K, int kend) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int mn, k;
    if (KContig) {  // element (mn, k) at P[k + mn*ld]
      k = t & 15;
      mn = (t >> 4) + 8 * i;
    } else {        // element (mn, k) at P[mn + k*ld]
      mn = t & 63;
      k = (t >> 6) + 2 * i;
    }
    const int gm = mn0 + mn;
    const int gk = k0 + k;
    double v = 0.0;
    if (gm < MN && gk < kend && gk < K) {
      v = KContig ? __ldg(P + (size_t)gm * ld + gk) : __ldg(P + gm + (size_t)gk * ld);
    }
    r[i] = v;
  }
}

template <bool KContig>
__device__ __forceinline__ void store_tile(double (*S)[BM + PAD], const double (&r)[8]) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int mn, k;
    if (KContig) {
      k = t & 15;
      mn = (t >> 4) + 8 * i;
    } else {
      mn = t & 63;
      k = (t >> 6) + 2 * i;
    }
    S[k][mn] = r[i];
  }
}

// op(A) (m,k): transA ? A[k + m*lda] : A[m + k*lda]   -> K-contiguous when transA
// op(B) (k,n): transB ? B[n + k*ldb] : B[k + n*ldb]   -> K-contiguous when !transB
template <bool TA, bool TB>
__global__ void __launch_bounds__(GEMM_THREADS)
gemm_f64_dmma(int M, int N, int K, double alpha, const double* __restrict__ A, int lda,
              const double* __restrict__ B, int ldb, double beta, double* __restrict__ C, int ldc,
              int k_per_split, long long split_stride, int upper) {
  __shared__ double As[2][BK][BM + PAD];
  __shared__ double Bs[2][BK][BN + PAD];
  const int bm = blockIdx.x * BM;
  const int bn = blockIdx.y * BN;
  if (upper && bm >= bn + BN) return;  // tile entirely below the diagonal
  const int kbeg = blockIdx.z * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int gid = lane >> 2;
  const int tig = lane & 3;
  const int wm = (warp & 1) * 32;
  const int wn = (warp >> 1) * 32;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  double ra[8], rb[8];
  if (kbeg < kend) {
    load_tile<TA>(ra, A, lda, bm, kbeg, M, K, kend);
    load_tile<!TB>(rb, B, ldb, bn, kbeg, N, K, kend);
    store_tile<TA>(As[0], ra);
    store_tile<!TB>(Bs[0], rb);
  }
  __syncthreads();
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    const bool has_next = (k0 + BK) < kend;
    if (has_next) {
      load_tile<TA>(ra, A, lda, bm, k0 + BK, M, K, kend);
      load_tile<!TB>(rb, B, ldb, bn, k0 + BK, N, K, kend);
    }
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[buf][kk + tig][wm + i * 8 + gid];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk + tig][wn + j * 8 + gid];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    if (has_next) {
      store_tile<TA>(As[buf ^ 1], ra);
      store_tile<!TB>(Bs[buf ^ 1], rb);
    }
    __syncthreads();
    buf ^= 1;
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = bm + wm + i * 8 + gid;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int n = bn + wn + j * 8 + tig * 2 + e;
        if (n >= N) continue;
        // split-K: each K range stores its own partial (summed in range order
        // by splitk_reduce_kernel, so runs repeat bit for bit)
        double* cp = C + (size_t)blockIdx.z * split_stride + m + (size_t)n * ldc;
        const double v = alpha * acc[i][j][e];
        if (split_stride) {
          *cp = v;
        } else {
          *cp = (beta == 0.0) ? v : (v + beta * *cp);
        }
      }
    }
  }
}

__global__ void scale_matrix_kernel(double* C, int M, int N, int ldc, double beta) {
  const size_t total = (size_t)M * N;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int m = static_cast<int>(idx % M);
    const int n = static_cast<int>(idx / M);
    double* cp = C + m + (size_t)n * ldc;
    *cp = (beta == 0.0) ? 0.0 : beta * *cp;
  }
}

// y[m] = alpha * sum_k A[m + k*lda] x[k] (+ beta y) ; grid.y splits K, atomics combine.
__global__ void gemv_n_kernel(int M, int K, double alpha, const double* __restrict__ A, int lda,
                              const double* __restrict__ x, double* __restrict__ y,
                              int k_per_split, long long split_stride, double beta) {
  __shared__ double xs[256];
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int kbeg = blockIdx.y * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  double acc = 0.0;
  for (int kc = kbeg; kc < kend; kc += 256) {
    const int kn = min(256, kend - kc);
    __syncthreads();
    if (threadIdx.x < kn) xs[threadIdx.x] = x[kc + threadIdx.x];
    __syncthreads();
    if (m < M) {
      const double* ap = A + m + (size_t)kc * lda;
      int k = 0;
      for (; k + 4 <= kn; k += 4) {
        acc = fma(__ldg(ap + (size_t)k * lda), xs[k], acc);
        acc = fma(__ldg(ap + (size_t)(k + 1) * lda), xs[k + 1], acc);
        acc = fma(__ldg(ap + (size_t)(k + 2) * lda), xs[k + 2], acc);
        acc = fma(__ldg(ap + (size_t)(k + 3) * lda), xs[k + 3], acc);
      }
      for (; k < kn; ++k) acc = fma(__ldg(ap + (size_t)k * lda), xs[k], acc);
    }
  }
  if (m < M) {
    if (split_stride) y[(size_t)blockIdx.y * split_stride + m] = alpha * acc;
    else y[m] = (beta == 0.0) ? alpha * acc : alpha * acc + beta * y[m];
  }
}

// C (M x N, ldc) = beta C + sum_{z < splits} W_z, W_z = W + z stride (ld ldw):
// the split-K partials added in K-range order.
__global__ void splitk_reduce_kernel(const double* __restrict__ W, int splits, long long stride, int M, int N,
                                     int ldw, double beta, double* __restrict__ C, int ldc) {
  const size_t total = (size_t)M * N;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int m = static_cast<int>(t % M), n = static_cast<int>(t / M);
    double acc = 0.0;
    for (int z = 0; z < splits; ++z) acc += W[(size_t)z * stride + m + (size_t)n * ldw];
    double* cp = C + m + (size_t)n * ldc;
    *cp = (beta == 0.0) ? acc : acc + beta * *cp;
  }
}

// y[n] = alpha * sum_k A[k + n*lda] x[k] + beta y[n] ; one warp per column.
__global__ void gemv_t_kernel(int K, int N, double alpha, const double* __restrict__ A, int lda,
                              const double* __restrict__ x, double beta, double* __restrict__ y) {
  const int warps_per_block = blockDim.x >> 5;
  const int n = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (n >= N) return;
  const double* ap = A + (size_t)n * lda;
  double acc = 0.0;
  for (int k = lane; k < K; k += 32) acc = fma(__ldg(ap + k), __ldg(x + k), acc);
  acc = warp_sum(acc);
  if (lane == 0) y[n] = (beta == 0.0) ? alpha * acc : alpha * acc + beta * y[n];
}

// FP64 column means; single-precision input is summed in FP64 in the same
// order, so its means equal those of the widened FP64 copy bit for bit.
template <typename T>
__global__ void col_mean_kernel(const T* __restrict__ X, int n, int p, int ldx,
                                double* __restrict__ out) {
  const int warps_per_block = blockDim.x >> 5;
  const int j = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= p) return;
  const T* xp = X + (size_t)j * ldx;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += static_cast<double>(xp[i]);
  s = warp_sum(s);
  if (lane == 0) out[j] = s / static_cast<double>(n);
}

__global__ void col_sd_kernel(const double* __restrict__ X, int n, int p, int ldx,
                              double* __restrict__ out) {
  const int warps_per_block = blockDim.x >> 5;
  const int j = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= p) return;
  const double* xp = X + (size_t)j * ldx;
  // Two-pass (mean of the centred column, then squares) matches Welford to rounding.
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += xp[i];
  s = warp_sum(s);
  const double mu = s / static_cast<double>(n);
  double q = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double d = xp[i] - mu;
    q += d * d;
  }
  q = warp_sum(q);
  if (lane == 0) out[j] = sqrt(q / static_cast<double>(n - 1));
}

// Column sums (the loop and warp reduction of col_mean_kernel, without the
// division): the partial sums of a row-sharded fit.
__global__ void col_sum_kernel(const double* __restrict__ X, int n, int p, int ldx, double* __restrict__ out) {
  const int warps_per_block = blockDim.x >> 5;
  const int j = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= p) return;
  const double* xp = X + (size_t)j * ldx;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += xp[i];
  s = warp_sum(s);
  if (lane == 0) out[j] = s;
}

// Sums of squared deviations from mu (the second pass of col_sd_kernel).
__global__ void col_sqdev_kernel(const double* __restrict__ X, int n, int p, int ldx, const double* __restrict__ mu,
                                 double* __restrict__ out) {
  const int warps_per_block = blockDim.x >> 5;
  const int j = blockIdx.x * warps_per_block + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= p) return;
  const double* xp = X + (size_t)j * ldx;
  const double m = mu[j];
  double q = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double d = xp[i] - m;
    q += d * d;
  }
  q = warp_sum(q);
  if (lane == 0) out[j] = q;
}

// out = in / d, or sqrt(in / d) when root is set.
__global__ void div_vec_kernel(const double* __restrict__ in, size_t count, double d, int root,
                               double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    out[i] = root ? sqrt(in[i] / d) : in[i] / d;
}

__global__ void center_scale_kernel(double* X, int n, int p, int ldx, const double* mean,
                                    const double* scale) {
  const size_t total = (size_t)n * p;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(idx % n);
    const int j = static_cast<int>(idx / n);
    double* xp = X + i + (size_t)j * ldx;
    double v = *xp;
    if (mean) v -= mean[j];
    if (scale) v /= scale[j];
    *xp = v;
  }
}

__global__ void copy_matrix_kernel(double* dst, int ldd, const double* src, int lds, int n, int p) {
  const size_t total = (size_t)n * p;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(idx % n);
    const int j = static_cast<int>(idx / n);
    dst[i + (size_t)j * ldd] = src[i + (size_t)j * lds];
  }
}

__global__ void add_row_vector_kernel(double* X, int n, int p, int ldx, const double* v) {
  const size_t total = (size_t)n * p;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(idx % n);
    const int j = static_cast<int>(idx / n);
    X[i + (size_t)j * ldx] += v[j];
  }
}

// Column sums of Y in the order rq_sums_kernel takes them (one block).
__global__ void rq_col_sums_kernel(const double* __restrict__ Y, int n, int m, double* __restrict__ out) {
  __shared__ double scratch[32];
  for (int j = 0; j < m; ++j) {
    const double* yc = Y + (size_t)j * n;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += yc[i];
    s = block_sum(s, scratch);
    if (threadIdx.x == 0) out[j] = s;
  }
}

// PRESS and TSS of Y against Yp; the TSS about the column means of these rows,
// or about mus (the means over all ranks' rows of a row-sharded fit).
__global__ void rq_sums_kernel(const double* __restrict__ Y, const double* __restrict__ Yp,
                               int n, int m, double* out2, const double* __restrict__ mus) {
  __shared__ double scratch[32];
  double press = 0.0, tss = 0.0;
  for (int j = 0; j < m; ++j) {
    const double* yc = Y + (size_t)j * n;
    double mu;
    if (mus) {
      mu = mus[j];
    } else {
      double s = 0.0;
      for (int i = threadIdx.x; i < n; i += blockDim.x) s += yc[i];
      s = block_sum(s, scratch);
      mu = s / static_cast<double>(n);
    }
    const double* pc = Yp + (size_t)j * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double d = yc[i] - pc[i];
      const double e = yc[i] - mu;
      press += d * d;
      tss += e * e;
    }
  }
  press = block_sum(press, scratch);
  tss = block_sum(tss, scratch);
  if (threadIdx.x == 0) {
    out2[0] = press;
    out2[1] = tss;
  }
}

__global__ void fill_kernel(double* x, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = v;
}

__global__ void scale_vec_kernel(double* x, size_t n, double a) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] *= a;
}

int grid_for(size_t total, int threads) {
  size_t g = (total + threads - 1) / threads;
  const size_t cap = (size_t)kSMCount * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

}  // namespace

void gemm(bool transA, bool transB, int M, int N, int K, double alpha, const double* A, int lda,
          const double* B, int ldb, double beta, double* C, int ldc) {
  if (M <= 0 || N <= 0) return;
  cudaStream_t st = Context::get().stream;
  if (K <= 0) {
    scale_matrix_kernel<<<grid_for((size_t)M * N, 256), 256, 0, st>>>(C, M, N, ldc, beta); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    return;
  }
  const int gm = ceil_div(M, BM);
  const int gn = ceil_div(N, BN);
  // Split K so that the grid covers the SMs at least twice for skinny outputs.
  int splits = 1;
  const int tiles = gm * gn;
  const int target = 2 * Context::get().sm_count;
  if (tiles < target && K >= 4 * BK) {
    splits = std::min(ceil_div(target, tiles), ceil_div(K, 8 * BK));
    if (splits < 1) splits = 1;
  }
  int kps = ceil_div(K, splits);
  kps = ceil_div(kps, BK) * BK;
  splits = ceil_div(K, kps);
  // split-K partials go to a per-stream workspace and are summed in order
  double* dst = C;
  int ldd = ldc;
  long long stride = 0;
  if (splits > 1) {
    stride = (long long)M * N;
    dst = Context::get().splitk_workspace(st, (size_t)splits * M * N);
    ldd = M;
  }
  const double beta_k = splits > 1 ? 0.0 : beta;
  dim3 grid(gm, gn, splits);
  Context& ctx = Context::get();
  const int slot = ctx.prof_begin("gemm_f64_dmma", st);
  if (!transA && !transB)
    gemm_f64_dmma<false, false><<<grid, GEMM_THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta_k, dst, ldd, kps, stride, 0);
  else if (transA && !transB)
    gemm_f64_dmma<true, false><<<grid, GEMM_THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta_k, dst, ldd, kps, stride, 0);
  else if (!transA && transB)
    gemm_f64_dmma<false, true><<<grid, GEMM_THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta_k, dst, ldd, kps, stride, 0);
  else
    gemm_f64_dmma<true, true><<<grid, GEMM_THREADS, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta_k, dst, ldd, kps, stride, 0);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  if (splits > 1) {
    splitk_reduce_kernel<<<grid_for((size_t)M * N, 256), 256, 0, st>>>(dst, splits, stride, M, N, ldd, beta, C, ldc);
    ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  // algorithmic work: 2MNK flops; each operand and the result once
  ctx.prof_end(slot, st, 8.0 * ((double)M * K + (double)K * N + (double)M * N), 2.0 * (double)M * N * K);
}

__global__ void mirror_upper_f64_kernel(double* K, int n, int ldk) {
  const size_t total = (size_t)n * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % n), j = static_cast<int>(t / n);
    if (i > j) K[i + (size_t)j * ldk] = K[j + (size_t)i * ldk];
  }
}

namespace {
// Upper tiles of op(X) op(X)^T (n x n) with n = rows of op(X) and p its
// columns, split-K partials summed in range order, then the lower triangle
// mirrored.  TX: X is stored p x n (op(X) = X^T).
template <bool TX>
void gram_tiles_f64(const double* X, int n, int p, int ldx, double* K, int ldk) {
  if (n <= 0) return;
  Context& ctx = Context::get();
  cudaStream_t st = ctx.stream;
  const int g = ceil_div(n, BM);
  int splits = 1;
  const int tiles = g * (g + 1) / 2;
  const int target = 2 * ctx.sm_count;
  if (tiles < target && p >= 4 * BK) splits = std::max(1, std::min(ceil_div(target, tiles), ceil_div(p, 8 * BK)));
  int kps = ceil_div(ceil_div(p, splits), BK) * BK;
  splits = ceil_div(p, kps);
  if (p <= 0) {
    scale_matrix_kernel<<<grid_for((size_t)n * n, 256), 256, 0, st>>>(K, n, n, ldk, 0.0); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  if (p > 0) {
    double* dst = K;
    int ldd = ldk;
    long long stride = 0;
    if (splits > 1) {  // partials of the K ranges, summed in order (lower tiles stay unused)
      stride = (long long)n * n;
      dst = ctx.splitk_workspace(st, (size_t)splits * n * n);
      ldd = n;
    }
    const int slot = ctx.prof_begin("gemm_f64_dmma", st);
    gemm_f64_dmma<TX, !TX><<<dim3(g, g, splits), GEMM_THREADS, 0, st>>>(n, n, p, 1.0, X, ldx, X, ldx, 0.0, dst,
                                                                       ldd, kps, stride, 1); ::fpls::note_launch();
    // algorithmic work: the upper tiles' share of 2 n^2 p flops
    ctx.prof_end(slot, st, 8.0 * ((double)n * p + (double)n * n), (double)n * (n + BM) * p);
    FPLS_CHECK_LAUNCH();
    if (splits > 1) {
      splitk_reduce_kernel<<<grid_for((size_t)n * n, 256), 256, 0, st>>>(dst, splits, stride, n, n, ldd, 0.0, K,
                                                                        ldk);
      ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
  }
  mirror_upper_f64_kernel<<<grid_for((size_t)n * n, 256), 256, 0, st>>>(K, n, ldk); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}
}  // namespace

void gram_f64(const double* X, int n, int p, int ldx, double* K, int ldk) {
  gram_tiles_f64<false>(X, n, p, ldx, K, ldk);
}

namespace {
// B (cols x rows, ld ldb) = A^T for A (rows x cols, ld lda), column-major both,
// through 32 x 32 shared-memory tiles (column reads and column writes).
__global__ void __launch_bounds__(256) transpose_f64_kernel(const double* __restrict__ A, int rows, int cols,
                                                            int lda, double* __restrict__ B, int ldb) {
  __shared__ double t[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int x = threadIdx.x & 31, y0 = threadIdx.x >> 5;
  for (int y = y0; y < 32; y += 8) {
    const int r = r0 + x, c = c0 + y;
    if (r < rows && c < cols) t[y][x] = A[r + static_cast<size_t>(c) * lda];
  }
  __syncthreads();
  for (int y = y0; y < 32; y += 8) {
    const int c = c0 + x, r = r0 + y;   // B(c, r) = A(r, c)
    if (r < rows && c < cols) B[c + static_cast<size_t>(r) * ldb] = t[x][y];
  }
}
}  // namespace

// G = S^T S through a transposed copy of S (q x p), so that the Gram's DMMA
// tiles read both operands in the layout of the row Gram X X^T (A along M,
// B along N) instead of reading S^T in place, for one extra pass over S.
void gram_t_f64(const double* S, int p, int q, int lds, double* G, int ldg) {
  if (q <= 0) return;
  if (p <= 0) {
    gram_tiles_f64<true>(S, q, p, lds, G, ldg);
    return;
  }
  Context& ctx = Context::get();
  double* St = ctx.arena.alloc_n<double>(static_cast<size_t>(q) * p);
  transpose_f64_kernel<<<dim3(ceil_div(p, 32), ceil_div(q, 32)), 256, 0, ctx.stream>>>(S, p, q, lds, St, q);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  gram_tiles_f64<false>(St, q, p, q, G, ldg);
}

void gemv(bool trans, int rows, int cols, double alpha, const double* A, int lda, const double* x,
          double beta, double* y) {
  Context& ctx = Context::get();
  cudaStream_t st = ctx.stream;
  const int slot = rows > 0 && cols > 0 ? ctx.prof_begin("gemv_f64", st) : -1;
  if (!trans) {
    if (rows <= 0) return;
    if (cols <= 0) {
      scale_matrix_kernel<<<grid_for(rows, 256), 256, 0, st>>>(y, rows, 1, rows, beta); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      return;
    }
    const int gx = ceil_div(rows, 256);
    int splits = 1;
    const int target = 4 * Context::get().sm_count;
    if (gx < target) splits = std::max(1, std::min(ceil_div(target, gx), ceil_div(cols, 256)));
    int kps = ceil_div(cols, splits);
    splits = ceil_div(cols, kps);
    if (splits > 1) {
      // partials of the column ranges, summed in order (runs repeat bit for bit)
      double* ws = ctx.splitk_workspace(st, (size_t)splits * rows);
      gemv_n_kernel<<<dim3(gx, splits), 256, 0, st>>>(rows, cols, alpha, A, lda, x, ws, kps, (long long)rows, 0.0);
      ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      splitk_reduce_kernel<<<grid_for(rows, 256), 256, 0, st>>>(ws, splits, rows, rows, 1, rows, beta, y, rows);
    } else {
      gemv_n_kernel<<<dim3(gx, splits), 256, 0, st>>>(rows, cols, alpha, A, lda, x, y, kps, 0ll, beta);
    }
    ::fpls::note_launch();
  } else {
    if (cols <= 0) return;
    gemv_t_kernel<<<ceil_div(cols, 8), 256, 0, st>>>(rows, cols, alpha, A, lda, x, beta, y); ::fpls::note_launch();
  }
  FPLS_CHECK_LAUNCH();
  // algorithmic bytes: the matrix once plus both vectors
  ctx.prof_end(slot, st, 8.0 * ((double)rows * cols + rows + cols), 2.0 * (double)rows * cols);
}

void col_mean(const double* X, int n, int p, int ldx, double* out) {
  if (p <= 0) return;
  col_mean_kernel<double><<<ceil_div(p, 8), 256, 0, Context::get().stream>>>(X, n, p, ldx, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void col_mean(const float* X, int n, int p, int ldx, double* out) {
  if (p <= 0) return;
  col_mean_kernel<float><<<ceil_div(p, 8), 256, 0, Context::get().stream>>>(X, n, p, ldx, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void col_sd_centered(const double* X, int n, int p, int ldx, double* out) {
  if (p <= 0) return;
  col_sd_kernel<<<ceil_div(p, 8), 256, 0, Context::get().stream>>>(X, n, p, ldx, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void col_sum(const double* X, int n, int p, int ldx, double* out) {
  if (p <= 0) return;
  col_sum_kernel<<<ceil_div(p, 8), 256, 0, Context::get().stream>>>(X, n, p, ldx, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void col_sqdev(const double* X, int n, int p, int ldx, const double* mu, double* out) {
  if (p <= 0) return;
  col_sqdev_kernel<<<ceil_div(p, 8), 256, 0, Context::get().stream>>>(X, n, p, ldx, mu, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void div_vec(const double* in, size_t count, double d, bool root, double* out) {
  if (count == 0) return;
  div_vec_kernel<<<grid_for(count, 256), 256, 0, Context::get().stream>>>(in, count, d, root ? 1 : 0, out); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void center_scale(double* X, int n, int p, int ldx, const double* mean, const double* scale) {
  if ((size_t)n * p == 0) return;
  center_scale_kernel<<<grid_for((size_t)n * p, 256), 256, 0, Context::get().stream>>>(X, n, p, ldx, mean, scale); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void copy_matrix(double* dst, int ldd, const double* src, int lds, int n, int p) {
  if ((size_t)n * p == 0) return;
  copy_matrix_kernel<<<grid_for((size_t)n * p, 256), 256, 0, Context::get().stream>>>(dst, ldd, src, lds, n, p); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void add_row_vector(double* X, int n, int p, int ldx, const double* v) {
  if ((size_t)n * p == 0) return;
  add_row_vector_kernel<<<grid_for((size_t)n * p, 256), 256, 0, Context::get().stream>>>(X, n, p, ldx, v); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void rq_sums(const double* Y, const double* Yp, int n, int m, double* out2, const double* mus) {
  rq_sums_kernel<<<1, 512, 0, Context::get().stream>>>(Y, Yp, n, m, out2, mus); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

const double* shard_rq_means(const double* Y, int n, int m) {
  if (!sharded()) return nullptr;
  Context& ctx = Context::get();
  double* mu = ctx.arena.alloc_n<double>(m);
  rq_col_sums_kernel<<<1, 512, 0, ctx.stream>>>(Y, n, m, mu); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  shard_sum(mu, m);
  div_vec(mu, m, static_cast<double>(shard_rows(n)), false, mu);
  return mu;
}

void fill(double* x, size_t n, double v) {
  if (n == 0) return;
  fill_kernel<<<grid_for(n, 256), 256, 0, Context::get().stream>>>(x, n, v); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void scale_vec(double* x, size_t n, double a) {
  if (n == 0) return;
  scale_vec_kernel<<<grid_for(n, 256), 256, 0, Context::get().stream>>>(x, n, a); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

}  // namespace fpls
