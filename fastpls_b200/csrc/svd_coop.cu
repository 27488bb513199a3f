// Thin SVD by one-sided (Hestenes) Jacobi spread over the whole GPU: one
// cooperative launch, one CTA per column pair of a round-robin round, a
// grid-wide barrier between rounds.  Used for the exact SVD of matrices too
// large for the single-CTA Jacobi (e.g. the 768 x 1000 class-sum
// cross-covariance of label-aware PLSSVD, which the reference hands to
// LAPACK gesdd through R's svd()).
#include "linalg_small.cuh"

#include <algorithm>
#include <cmath>

#include "blas_f64.cuh"
#include "context.cuh"

namespace fpls {
namespace {

constexpr int kCoopThreads = 256;
constexpr unsigned long long kBarrierSpinLimit = 1ull << 24;  // x 64 ns sleep: ~1 s

struct CoopJacobi {
  double* M;           // L x r, column-major; columns are rotated in place
  double* W;           // r x r accumulated rotations
  int L, r, ne;        // ne = r rounded up to even
  unsigned int* bar;   // [0] arrivals, [1] generation
  unsigned int* rot;   // 3 rotation counters (one per sweep, reused mod 3)
  int* flag;           // set when a barrier wait gives up
  int* sweeps;         // sweeps run
  double tol;
  int max_sweeps;
};

// Grid-wide barrier with a bounded wait: thread 0 of each CTA arrives on a
// counter; the last arrival resets it and advances the generation.  A wait
// that exceeds the limit (or sees the flag raised elsewhere) raises the flag,
// and every CTA then leaves the kernel.
__device__ bool coop_barrier(const CoopJacobi& J) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = J.bar + 1;
    volatile int* flag = J.flag;
    const unsigned int g = *gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(J.bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(J.bar, 0u);
      __threadfence();
      atomicAdd(J.bar + 1, 1u);
    } else {
      unsigned long long spins = 0;
      while (*gen == g && *flag == 0) {
        if (++spins > kBarrierSpinLimit) {
          atomicExch(J.flag, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *(volatile int*)J.flag == 0;
}

// Round-robin ("circle") schedule: in round rd every index meets exactly one
// other; index ne - 1 stays fixed.
__device__ __forceinline__ void circle_pair(int ne, int rd, int k, int& i, int& j) {
  const int m = ne - 1;
  if (k == 0) {
    i = rd;
    j = m;
  } else {
    i = (rd + k) % m;
    j = (rd - k + m) % m;
  }
}

__device__ __forceinline__ double block_sum3(double& a, double& b, double& c, double (*red)[3]) {
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[w][0] = a;
    red[w][1] = b;
    red[w][2] = c;
  }
  __syncthreads();
  a = b = c = 0.0;
  for (int u = 0; u < kCoopThreads / 32; ++u) {
    a += red[u][0];
    b += red[u][1];
    c += red[u][2];
  }
  __syncthreads();
  return a;
}

// One CTA per column pair of the round (the CTA loops when there are more
// pairs than CTAs); all threads of the CTA share the pair's dots and update.
__global__ void __launch_bounds__(kCoopThreads) jacobi_coop_kernel(CoopJacobi J) {
  __shared__ double red[kCoopThreads / 32][3];
  const int npairs = J.ne / 2;
  for (int sweep = 0; sweep < J.max_sweeps; ++sweep) {
    if (blockIdx.x == 0 && threadIdx.x == 0) J.rot[(sweep + 1) % 3] = 0u;
    for (int rd = 0; rd < J.ne - 1; ++rd) {
      for (int k = blockIdx.x; k < npairs; k += gridDim.x) {
        int i, j;
        circle_pair(J.ne, rd, k, i, j);
        if (i >= J.r || j >= J.r) continue;
        double* a = J.M + (size_t)i * J.L;
        double* b = J.M + (size_t)j * J.L;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int t = threadIdx.x; t < J.L; t += kCoopThreads) {
          const double x = __ldcg(a + t), y = __ldcg(b + t);
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        block_sum3(al, be, ga, red);
        if (!(ga != 0.0) || !(fabs(ga) > J.tol * sqrt(al) * sqrt(be))) continue;
        const double zeta = (be - al) / (2.0 * ga);
        double t;
        if (fabs(zeta) > 1e150) {
          t = 0.5 / zeta;
        } else {
          t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        }
        const double c = 1.0 / sqrt(1.0 + t * t);
        const double s = c * t;
        for (int u = threadIdx.x; u < J.L; u += kCoopThreads) {
          const double x = __ldcg(a + u), y = __ldcg(b + u);
          __stcg(a + u, c * x - s * y);
          __stcg(b + u, s * x + c * y);
        }
        double* wa = J.W + (size_t)i * J.r;
        double* wb = J.W + (size_t)j * J.r;
        for (int u = threadIdx.x; u < J.r; u += kCoopThreads) {
          const double x = __ldcg(wa + u), y = __ldcg(wb + u);
          __stcg(wa + u, c * x - s * y);
          __stcg(wb + u, s * x + c * y);
        }
        if (threadIdx.x == 0) atomicAdd(J.rot + (sweep % 3), 1u);
      }
      if (!coop_barrier(J)) return;
    }
    const unsigned int rotated = *(volatile unsigned int*)(J.rot + (sweep % 3));
    if (rotated == 0u) {
      if (blockIdx.x == 0 && threadIdx.x == 0) *J.sweeps = sweep + 1;
      return;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *J.sweeps = J.max_sweeps + 1;  // not converged
}

__global__ void identity_kernel(double* W, int r) {
  const size_t total = (size_t)r * r;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x)
    W[t] = (t % r == t / r) ? 1.0 : 0.0;
}

__global__ void transpose_into_kernel(const double* __restrict__ A, int rows, int cols, int lda,
                                      double* __restrict__ B) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (i < rows && j < cols) tile[r][threadIdx.x] = A[i + (size_t)j * lda];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (i < rows && j < cols) B[j + (size_t)i * cols] = tile[threadIdx.x][r];
  }
}

__global__ void col_norms_kernel(const double* __restrict__ M, int L, int r, double* __restrict__ nrm) {
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= r) return;
  double s = 0.0;
  for (int t = lane; t < L; t += 32) s += M[t + (size_t)w * L] * M[t + (size_t)w * L];
  s = warp_sum(s);
  if (lane == 0) nrm[w] = sqrt(s);
}

// order[rank] = column, descending norms, ties by index.
__global__ void rank_desc_kernel(const double* __restrict__ nrm, int r, int* __restrict__ order) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < r; j += gridDim.x * blockDim.x) {
    const double v = nrm[j];
    int rank = 0;
    for (int i = 0; i < r; ++i) {
      const double u = nrm[i];
      rank += (u > v) || (u == v && i < j);
    }
    order[rank] = j;
  }
}

// tall (M = A): U[:, k] = M[:, src] / s, V[:, k] = W[:, src]
// wide (M = A^T): U[:, k] = W[:, src], V[:, k] = M[:, src] / s
// Columns with s below tol are left for the completion kernel.
__global__ void write_svd_kernel(const double* __restrict__ M, const double* __restrict__ W, int L,
                                 int r, const double* __restrict__ nrm, const int* __restrict__ order,
                                 bool tall, double* U, int ldu, double* s, double* V, int ldv) {
  const int k = blockIdx.y;
  const int src = order[k];
  const double sk = nrm[src];
  const double smax = nrm[order[0]];
  const double tol = 2.220446049250313e-16 * (double)(L > r ? L : r) * smax;
  const bool ok = sk > tol && sk > 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) s[k] = sk;
  double* mdst = tall ? U + (size_t)k * ldu : V + (size_t)k * ldv;
  double* wdst = tall ? V + (size_t)k * ldv : U + (size_t)k * ldu;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L; t += gridDim.x * blockDim.x)
    mdst[t] = ok ? M[t + (size_t)src * L] / sk : 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < r; t += gridDim.x * blockDim.x)
    wdst[t] = W[t + (size_t)src * r];
}

// Negligible singular values: complete the L-dimensional side with unit
// vectors made orthogonal (two Gram-Schmidt passes) to the columns before
// them, as the single-CTA Jacobi does.  One CTA; a no-op when none is needed.
__global__ void complete_null_kernel(int L, int r, const double* __restrict__ s, bool tall, double* U,
                                     int ldu, double* V, int ldv) {
  __shared__ double scratch[32];
  const double smax = s[0];
  const double tol = 2.220446049250313e-16 * (double)(L > r ? L : r) * smax;
  for (int j = 0; j < r; ++j) {
    if (s[j] > tol && s[j] > 0.0) continue;
    double* uj = tall ? U + (size_t)j * ldu : V + (size_t)j * ldv;
    for (int e = 0; e < L; ++e) {
      for (int i = threadIdx.x; i < L; i += blockDim.x) uj[i] = (i == e) ? 1.0 : 0.0;
      __syncthreads();
      for (int pass = 0; pass < 2; ++pass) {
        for (int jj = 0; jj < j; ++jj) {
          const double* uo = tall ? U + (size_t)jj * ldu : V + (size_t)jj * ldv;
          double d = 0.0;
          for (int i = threadIdx.x; i < L; i += blockDim.x) d += uo[i] * uj[i];
          d = block_sum(d, scratch);
          for (int i = threadIdx.x; i < L; i += blockDim.x) uj[i] -= d * uo[i];
          __syncthreads();
        }
      }
      double nn = 0.0;
      for (int i = threadIdx.x; i < L; i += blockDim.x) nn += uj[i] * uj[i];
      nn = block_sum(nn, scratch);
      if (nn > 0.25) {
        const double inv = 1.0 / sqrt(nn);
        for (int i = threadIdx.x; i < L; i += blockDim.x) uj[i] *= inv;
        __syncthreads();
        break;
      }
    }
  }
}

}  // namespace

void svd_jacobi_coop(int rows, int cols, const double* A, int lda, double* U, int ldu, double* s,
                     double* V, int ldv) {
  if (rows <= 0 || cols <= 0) return;
  Context& ctx = Context::get();
  const bool tall = rows >= cols;
  const int L = tall ? rows : cols;
  const int r = tall ? cols : rows;
  FPLS_REQUIRE(r <= 65535, "svd_jacobi_coop: more than 65535 singular values requested");
  double* M = ctx.arena.alloc_n<double>((size_t)L * r);
  double* W = ctx.arena.alloc_n<double>((size_t)r * r);
  if (tall) {
    copy_matrix(M, L, A, lda, rows, cols);
  } else {
    dim3 grid(ceil_div(rows, 32), ceil_div(cols, 32));
    transpose_into_kernel<<<grid, dim3(32, 8), 0, ctx.stream>>>(A, rows, cols, lda, M); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  identity_kernel<<<std::min(ceil_div((long long)r * r, 256), 4 * ctx.sm_count), 256, 0, ctx.stream>>>(W, r); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();

  unsigned int* ctl = ctx.arena.alloc_n<unsigned int>(8);
  FPLS_CUDA(cudaMemsetAsync(ctl, 0, 8 * sizeof(unsigned int), ctx.stream));
  int* flag = reinterpret_cast<int*>(ctl + 5);
  int* sweeps = reinterpret_cast<int*>(ctl + 6);

  static int max_blocks_per_sm = -1;
  if (max_blocks_per_sm < 0) {
    FPLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_blocks_per_sm, jacobi_coop_kernel,
                                                            kCoopThreads, 0));
  }
  FPLS_REQUIRE(max_blocks_per_sm > 0, "svd_jacobi_coop: kernel cannot be resident");
  const int ne = r + (r & 1);
  const int blocks_needed = ne / 2;
  const int grid = std::max(1, std::min(blocks_needed, max_blocks_per_sm * ctx.sm_count));

  CoopJacobi J;
  J.M = M;
  J.W = W;
  J.L = L;
  J.r = r;
  J.ne = ne;
  J.bar = ctl;
  J.rot = ctl + 2;
  J.flag = flag;
  J.sweeps = sweeps;
  J.tol = (double)L * 2.220446049250313e-16;
  J.max_sweeps = 40;
  void* args[] = {&J};
  FPLS_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_coop_kernel, dim3(grid), dim3(kCoopThreads),
                                        args, 0, ctx.stream)); ::fpls::note_launch();
  int h[2] = {0, 0};
  FPLS_CUDA(cudaMemcpyAsync(h, flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  FPLS_CUDA(cudaStreamSynchronize(ctx.stream));
  if (h[0]) throw Error(kErrCuda, "svd_jacobi_coop: grid barrier wait exceeded its limit");
  // h[1] > max_sweeps means rotations were still being applied after the last
  // sweep; at that point they are rounding-level and the columns are used as is.

  double* nrm = ctx.arena.alloc_n<double>(r);
  int* order = ctx.arena.alloc_n<int>(r);
  col_norms_kernel<<<ceil_div((long long)r * 32, 256), 256, 0, ctx.stream>>>(M, L, r, nrm); ::fpls::note_launch();
  rank_desc_kernel<<<ceil_div(r, 128), 128, 0, ctx.stream>>>(nrm, r, order); ::fpls::note_launch();
  write_svd_kernel<<<dim3(std::max(1, std::min(ceil_div(L, 256), 8)), r), 256, 0, ctx.stream>>>(
      M, W, L, r, nrm, order, tall, U, ldu, s, V, ldv); ::fpls::note_launch();
  complete_null_kernel<<<1, 512, 0, ctx.stream>>>(L, r, s, tall, U, ldu, V, ldv); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void eig_psd_desc(int l, const double* G, int ldg, double* evals, double* V, int ldv) {
  if (l <= 64) {
    eig_sym_desc(l, G, ldg, evals, V, ldv);
    return;
  }
  double* U = Context::get().arena.alloc_n<double>((size_t)l * l);
  svd_jacobi_coop(l, l, G, ldg, U, l, evals, V, ldv);
}

}  // namespace fpls
