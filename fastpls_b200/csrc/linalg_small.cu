#include "blas_f64.cuh"
#include "context.cuh"
#include "linalg_small.cuh"

#include <vector>

namespace fpls {
namespace {

constexpr double kEps = 2.220446049250313e-16;

// ---------------------------------------------------------------- Cholesky ---
// In-place lower Cholesky of A (k x k, lda) in global scratch; returns false via
// *ok = 0 when a pivot is not positive.
__device__ void chol_lower_inplace(double* A, int k, int lda, int* ok) {
  for (int j = 0; j < k; ++j) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const double d = A[j + (size_t)j * lda];
      if (!(d > 0.0) || !isfinite(d)) *ok = 0;
      else A[j + (size_t)j * lda] = sqrt(d);
    }
    __syncthreads();
    if (!*ok) return;
    const double ljj = A[j + (size_t)j * lda];
    for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) A[i + (size_t)j * lda] /= ljj;
    __syncthreads();
    const int rem = k - j - 1;
    const long long tot = (long long)rem * rem;
    for (long long t = threadIdx.x; t < tot; t += blockDim.x) {
      const int ii = j + 1 + static_cast<int>(t % rem);
      const int ll = j + 1 + static_cast<int>(t / rem);
      if (ll <= ii) A[ii + (size_t)ll * lda] -= A[ii + (size_t)j * lda] * A[ll + (size_t)j * lda];
    }
  }
  __syncthreads();
}

__global__ void spd_solve_kernel(int k, const double* __restrict__ G, int ldg, int nrhs,
                                 const double* __restrict__ B, int ldb, double* __restrict__ X,
                                 int ldx, double* W, int* d_flag, double ridge_rel) {
  __shared__ int ok;
  __shared__ double ridge;
  __shared__ double scratch[32];
  // Copy G (+ ridge) into W.
  if (threadIdx.x == 0) ok = 1;
  double dsum = 0.0;
  for (int i = threadIdx.x; i < k; i += blockDim.x) dsum += G[i + (size_t)i * ldg];
  dsum = block_sum(dsum, scratch);
  if (threadIdx.x == 0) {
    double r = 0.0;
    if (ridge_rel > 0.0) {
      r = ridge_rel * dsum / static_cast<double>(k);
      if (!isfinite(r) || r <= 0.0) r = ridge_rel;
    }
    ridge = r;
  }
  __syncthreads();
  for (long long t = threadIdx.x; t < (long long)k * k; t += blockDim.x) {
    const int i = static_cast<int>(t % k), j = static_cast<int>(t / k);
    W[i + (size_t)j * k] = G[i + (size_t)j * ldg] + (i == j ? ridge : 0.0);
  }
  __syncthreads();
  chol_lower_inplace(W, k, k, &ok);
  if (ok) {
    // Forward and back substitution, one thread per right-hand side.
    for (int c = threadIdx.x; c < nrhs; c += blockDim.x) {
      double* x = X + (size_t)c * ldx;
      const double* b = B + (size_t)c * ldb;
      for (int i = 0; i < k; ++i) {
        double s = b[i];
        for (int l = 0; l < i; ++l) s -= W[i + (size_t)l * k] * x[l];
        x[i] = s / W[i + (size_t)i * k];
      }
      for (int i = k - 1; i >= 0; --i) {
        double s = x[i];
        for (int l = i + 1; l < k; ++l) s -= W[l + (size_t)i * k] * x[l];
        x[i] = s / W[i + (size_t)i * k];
      }
    }
    return;
  }
  // LU with partial pivoting on [G | B] (k x (k + nrhs)) in W.
  __syncthreads();
  const int ncol = k + nrhs;
  for (long long t = threadIdx.x; t < (long long)k * ncol; t += blockDim.x) {
    const int i = static_cast<int>(t % k), j = static_cast<int>(t / k);
    W[i + (size_t)j * k] = (j < k) ? G[i + (size_t)j * ldg] + (i == j ? ridge : 0.0)
                                   : B[i + (size_t)(j - k) * ldb];
  }
  __shared__ int piv;
  for (int j = 0; j < k; ++j) {
    __syncthreads();
    if (threadIdx.x == 0) {
      int best = j;
      double bv = fabs(W[j + (size_t)j * k]);
      for (int i = j + 1; i < k; ++i) {
        const double v = fabs(W[i + (size_t)j * k]);
        if (v > bv) { bv = v; best = i; }
      }
      piv = best;
      if (!(bv > 0.0)) { ok = -1; }
    }
    __syncthreads();
    if (ok == -1) break;
    if (piv != j) {
      for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
        const double a = W[j + (size_t)c * k];
        W[j + (size_t)c * k] = W[piv + (size_t)c * k];
        W[piv + (size_t)c * k] = a;
      }
    }
    __syncthreads();
    const double pv = W[j + (size_t)j * k];
    const int rem = k - j - 1;
    const int cols = ncol - j - 1;
    for (long long t = threadIdx.x; t < (long long)rem * cols; t += blockDim.x) {
      const int i = j + 1 + static_cast<int>(t % rem);
      const int c = j + 1 + static_cast<int>(t / rem);
      W[i + (size_t)c * k] -= (W[i + (size_t)j * k] / pv) * W[j + (size_t)c * k];
    }
  }
  __syncthreads();
  if (ok == -1) {
    if (threadIdx.x == 0) atomicExch(d_flag, 1);
    return;
  }
  for (int c = threadIdx.x; c < nrhs; c += blockDim.x) {
    double* x = X + (size_t)c * ldx;
    for (int i = k - 1; i >= 0; --i) {
      double s = W[i + (size_t)(k + c) * k];
      for (int l = i + 1; l < k; ++l) s -= W[i + (size_t)l * k] * x[l];
      x[i] = s / W[i + (size_t)i * k];
    }
  }
}

// --------------------------------------------------------------- CholeskyQR ---
// Upper Cholesky of the Gram in place (G = R^T R stored in the upper triangle).
__global__ void chol_upper_kernel(double* G, int k, int* d_flag) {
  __shared__ int ok;
  if (threadIdx.x == 0) ok = 1;
  __syncthreads();
  // Lower Cholesky of G equals the transpose of the upper factor.
  chol_lower_inplace(G, k, k, &ok);
  if (!ok && threadIdx.x == 0) atomicExch(d_flag, 1);
}

// Q[i, :] = Y[i, :] * R^{-1}, R upper given as L^T (lower factor L in G).
__global__ void trsm_rows_kernel(int rows, int k, const double* __restrict__ Y, int ldy,
                                 const double* __restrict__ L, double* __restrict__ Q, int ldq) {
  extern __shared__ double Ls[];
  for (int t = threadIdx.x; t < k * k; t += blockDim.x) Ls[t] = L[t];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  // Row solve: q_j = (y_j - sum_{l<j} q_l R[l][j]) / R[j][j], R[l][j] = L[j][l].
  for (int j = 0; j < k; ++j) {
    double s = Y[i + (size_t)j * ldy];
    for (int l = 0; l < j; ++l) s -= Q[i + (size_t)l * ldq] * Ls[j + l * k];
    Q[i + (size_t)j * ldq] = s / Ls[j + j * k];
  }
}

__global__ void normalize_col_kernel(double* q, int rows, const double* nrm2) {
  const double nr = sqrt(*nrm2);
  const double inv = (nr > 0.0 && isfinite(nr)) ? 1.0 / nr : 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
    q[i] *= inv;
}

__global__ void dot_self_kernel(const double* x, int n, double* out) {
  __shared__ double scratch[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i] * x[i];
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) *out = s;
}

// ------------------------------------------------------------- Jacobi eigen ---
__device__ void round_robin_next(int* arr, int n) {
  // keep arr[0]; rotate arr[1..n-1] right by one
  const int last = arr[n - 1];
  for (int i = n - 1; i > 1; --i) arr[i] = arr[i - 1];
  arr[1] = last;
}

// With in_smem the working matrices W and V live in shared memory (after the
// rotation tables): W is copied in first, and every rotation round touches
// shared memory only.
__global__ void jacobi_eig_kernel(int l, double* W, double* V, double* evals_out,
                                  double* V_out, int ldv, const int max_sweeps, int in_smem) {
  extern __shared__ double sm[];
  const int npair = (l + 1) / 2;
  const int le = 2 * npair;
  double* cs = sm;              // [npair] cos
  double* sn = sm + npair;      // [npair] sin
  int* arr = reinterpret_cast<int*>(sm + 2 * npair);   // [le]
  int* pp = arr + le;           // [npair]
  int* qq = pp + npair;         // [npair]
  __shared__ double scratch[32];
  __shared__ int sweep_done;
  if (in_smem) {
    double* Ws = reinterpret_cast<double*>(reinterpret_cast<char*>(sm) + 32 * npair);
    for (int t = threadIdx.x; t < l * l; t += blockDim.x) Ws[t] = W[t];
    W = Ws;
    V = Ws + (size_t)l * l;
  }
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) V[t] = (t % l == t / l) ? 1.0 : 0.0;
  __shared__ int rotated;
  __syncthreads();
  // Frobenius norm for the convergence test.
  double fro = 0.0;
  for (int t = threadIdx.x; t < l * l; t += blockDim.x) fro += W[t] * W[t];
  fro = block_sum(fro, scratch);
  const double thresh = kEps * kEps * fro;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    for (int t = threadIdx.x; t < l * l; t += blockDim.x) {
      const int i = t % l, j = t / l;
      if (i != j) off += W[t] * W[t];
    }
    off = block_sum(off, scratch);
    if (threadIdx.x == 0) {
      sweep_done = (off <= thresh) ? 1 : 0;
      rotated = 0;
    }
    __syncthreads();
    if (sweep_done) break;
    for (int r = 0; r < le - 1; ++r) {
      // round-robin pairing of round r: position 0 stays, positions 1..le-1
      // have turned r places (position i holds 1 + (i - 1 - r) mod (le - 1))
      for (int k = threadIdx.x; k < npair; k += blockDim.x) {
        const int ik = le - 1 - k;
        int p = k == 0 ? 0 : 1 + ((k - 1 - r) % (le - 1) + (le - 1)) % (le - 1);
        int q = 1 + ((ik - 1 - r) % (le - 1) + (le - 1)) % (le - 1);
        if (p > q) { const int t = p; p = q; q = t; }
        pp[k] = p; qq[k] = q;
        double c = 1.0, s = 0.0;
        if (q < l) {
          const double apq = W[p + (size_t)q * l];
          const double app = W[p + (size_t)p * l];
          const double aqq = W[q + (size_t)q * l];
          // a rotation is skipped once the pair is decoupled to rounding
          if (apq != 0.0 && fabs(apq) > 1e-300 && fabs(apq) > kEps * sqrt(fabs(app * aqq))) {
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
            rotated = 1;
          }
        }
        cs[k] = c; sn[k] = s;
      }
      __syncthreads();
      if (npair <= 32) {
        // lane = pair, warps stride over the rows / columns (no index division)
        const int k = threadIdx.x & 31, w0 = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const bool act = k < npair && qq[k] < l && sn[k] != 0.0;
        const int p = act ? pp[k] : 0, q = act ? qq[k] : 0;
        const double c = act ? cs[k] : 1.0, sv = act ? sn[k] : 0.0;
        // rows: W <- J^T W
        if (act)
          for (int j = w0; j < l; j += nw) {
            const double wp = W[p + j * l], wq = W[q + j * l];
            W[p + j * l] = c * wp - sv * wq;
            W[q + j * l] = sv * wp + c * wq;
          }
        __syncthreads();
        // columns: W <- W J, V <- V J
        if (act)
          for (int i = w0; i < l; i += nw) {
            const double wp = W[i + p * l], wq = W[i + q * l];
            W[i + p * l] = c * wp - sv * wq;
            W[i + q * l] = sv * wp + c * wq;
            const double vp = V[i + p * l], vq = V[i + q * l];
            V[i + p * l] = c * vp - sv * vq;
            V[i + q * l] = sv * vp + c * vq;
          }
        __syncthreads();
        continue;
      }
      // rows: W <- J^T W
      for (int t = threadIdx.x; t < npair * l; t += blockDim.x) {
        const int k = t % npair, j = t / npair;
        const int p = pp[k], q = qq[k];
        if (q >= l || sn[k] == 0.0) continue;
        const double c = cs[k], s = sn[k];
        const double wp = W[p + (size_t)j * l], wq = W[q + (size_t)j * l];
        W[p + (size_t)j * l] = c * wp - s * wq;
        W[q + (size_t)j * l] = s * wp + c * wq;
      }
      __syncthreads();
      // columns: W <- W J, V <- V J
      for (int t = threadIdx.x; t < npair * l; t += blockDim.x) {
        const int k = t % npair, i = t / npair;
        const int p = pp[k], q = qq[k];
        if (q >= l || sn[k] == 0.0) continue;
        const double c = cs[k], s = sn[k];
        const double wp = W[i + (size_t)p * l], wq = W[i + (size_t)q * l];
        W[i + (size_t)p * l] = c * wp - s * wq;
        W[i + (size_t)q * l] = s * wp + c * wq;
        const double vp = V[i + (size_t)p * l], vq = V[i + (size_t)q * l];
        V[i + (size_t)p * l] = c * vp - s * vq;
        V[i + (size_t)q * l] = s * vp + c * vq;
      }
      __syncthreads();
    }
    if (!rotated) break;   // a whole sweep without a rotation: converged
  }
  // Sort eigenvalues descending (selection order kept in arr).
  if (threadIdx.x == 0) {
    for (int i = 0; i < l; ++i) arr[i] = i;
    for (int i = 0; i < l; ++i) {
      int best = i;
      for (int j = i + 1; j < l; ++j)
        if (W[arr[j] + (size_t)arr[j] * l] > W[arr[best] + (size_t)arr[best] * l]) best = j;
      const int t = arr[i]; arr[i] = arr[best]; arr[best] = t;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < l; i += blockDim.x) evals_out[i] = W[arr[i] + (size_t)arr[i] * l];
  for (long long t = threadIdx.x; t < (long long)l * l; t += blockDim.x) {
    const int i = static_cast<int>(t % l), j = static_cast<int>(t / l);
    V_out[i + (size_t)j * ldv] = V[i + (size_t)arr[j] * l];
  }
}

// ---------------------------------------------------------- one-sided Jacobi ---
// W (r x c, r >= c) is overwritten; V (c x c) accumulates the rotations.
__global__ void jacobi_svd_kernel(int r, int c, double* W, double* V, int max_sweeps,
                                  double* U_out, int ldu, double* s_out, double* V_out, int ldv,
                                  int transpose_out) {
  extern __shared__ double sm[];
  const int npair = (c + 1) / 2;
  const int ce = 2 * npair;
  int* arr = reinterpret_cast<int*>(sm);
  int* order = arr + ce;
  double* norms = sm + (2 * ce + 1) / 2 + 1;
  __shared__ int rotated;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int t = threadIdx.x; t < c * c; t += blockDim.x) V[t] = (t % c == t / c) ? 1.0 : 0.0;
  if (threadIdx.x == 0) for (int i = 0; i < ce; ++i) arr[i] = i;
  __syncthreads();
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (int rr = 0; rr < ce - 1; ++rr) {
      for (int k = warp; k < npair; k += nwarps) {
        int p = arr[k], q = arr[ce - 1 - k];
        if (p > q) { const int t = p; p = q; q = t; }
        if (q >= c) continue;
        double* wp = W + (size_t)p * r;
        double* wq = W + (size_t)q * r;
        double a = 0.0, b = 0.0, g = 0.0;
        for (int i = lane; i < r; i += 32) {
          const double x = wp[i], y = wq[i];
          a += x * x; b += y * y; g += x * y;
        }
        a = warp_sum(a); b = warp_sum(b); g = warp_sum(g);
        if (fabs(g) > kEps * sqrt(a * b) && fabs(g) > 1e-300) {
          const double zeta = (b - a) / (2.0 * g);
          const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + t * t);
          const double sn = cs * t;
          for (int i = lane; i < r; i += 32) {
            const double x = wp[i], y = wq[i];
            wp[i] = cs * x - sn * y;
            wq[i] = sn * x + cs * y;
          }
          for (int i = lane; i < c; i += 32) {
            const double x = V[i + (size_t)p * c], y = V[i + (size_t)q * c];
            V[i + (size_t)p * c] = cs * x - sn * y;
            V[i + (size_t)q * c] = sn * x + cs * y;
          }
          if (lane == 0) rotated = 1;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) round_robin_next(arr, ce);
      __syncthreads();
    }
    if (!rotated) break;
  }
  // Column norms and descending order.
  for (int k = warp; k < c; k += nwarps) {
    double a = 0.0;
    for (int i = lane; i < r; i += 32) a += W[i + (size_t)k * r] * W[i + (size_t)k * r];
    a = warp_sum(a);
    if (lane == 0) norms[k] = sqrt(a);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < c; ++i) order[i] = i;
    for (int i = 0; i < c; ++i) {
      int best = i;
      for (int j = i + 1; j < c; ++j) if (norms[order[j]] > norms[order[best]]) best = j;
      const int t = order[i]; order[i] = order[best]; order[best] = t;
    }
  }
  __syncthreads();
  const double smax = norms[order[0]];
  const double tol = kEps * static_cast<double>(r > c ? r : c) * smax;
  // Output: U columns = W columns / s (completed when s is negligible).
  for (int j = 0; j < c; ++j) {
    const int src = order[j];
    const double sj = norms[src];
    double* uj = transpose_out ? V_out + (size_t)j * ldv : U_out + (size_t)j * ldu;
    double* vj = transpose_out ? U_out + (size_t)j * ldu : V_out + (size_t)j * ldv;
    if (threadIdx.x == 0) s_out[j] = sj;
    if (sj > tol && sj > 0.0) {
      for (int i = threadIdx.x; i < r; i += blockDim.x) uj[i] = W[i + (size_t)src * r] / sj;
      __syncthreads();
    } else {
      // Complete with a unit vector orthogonal to the earlier columns.
      for (int e = 0; e < r; ++e) {
        for (int i = threadIdx.x; i < r; i += blockDim.x) uj[i] = (i == e) ? 1.0 : 0.0;
        __syncthreads();
        for (int pass = 0; pass < 2; ++pass) {
          for (int jj = 0; jj < j; ++jj) {
            const double* uo = transpose_out ? V_out + (size_t)jj * ldv : U_out + (size_t)jj * ldu;
            __shared__ double scratch[32];
            double d = 0.0;
            for (int i = threadIdx.x; i < r; i += blockDim.x) d += uo[i] * uj[i];
            d = block_sum(d, scratch);
            for (int i = threadIdx.x; i < r; i += blockDim.x) uj[i] -= d * uo[i];
            __syncthreads();
          }
        }
        __shared__ double scratch2[32];
        double nn = 0.0;
        for (int i = threadIdx.x; i < r; i += blockDim.x) nn += uj[i] * uj[i];
        nn = block_sum(nn, scratch2);
        if (nn > 0.25) {
          const double inv = 1.0 / sqrt(nn);
          for (int i = threadIdx.x; i < r; i += blockDim.x) uj[i] *= inv;
          __syncthreads();
          break;
        }
      }
    }
    for (int i = threadIdx.x; i < c; i += blockDim.x) vj[i] = V[i + (size_t)src * c];
    __syncthreads();
  }
}

__global__ void transpose_kernel(const double* __restrict__ A, int rows, int cols, int lda,
                                 double* __restrict__ B) {
  const size_t total = (size_t)rows * cols;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int i = static_cast<int>(t % rows), j = static_cast<int>(t / rows);
    B[j + (size_t)i * cols] = A[i + (size_t)j * lda];
  }
}

}  // namespace

void spd_solve(int k, const double* G, int ldg, int nrhs, const double* B, int ldb, double* X,
               int ldx, int* d_flag, double ridge_rel) {
  if (k <= 0 || nrhs <= 0) return;
  Context& ctx = Context::get();
  double* W = ctx.arena.alloc_n<double>((size_t)k * (k + nrhs));
  spd_solve_kernel<<<1, 512, 0, ctx.stream>>>(k, G, ldg, nrhs, B, ldb, X, ldx, W,
                                              d_flag ? d_flag : ctx.d_status + 1, ridge_rel); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

static void cgs2_orthonormalize(int rows, int cols, const double* Y, int ldy, double* Q, int ldq) {
  Context& ctx = Context::get();
  double* w = ctx.arena.alloc_n<double>(cols > 0 ? cols : 1);
  double* nrm = ctx.arena.alloc_n<double>(1);
  for (int j = 0; j < cols; ++j) {
    double* q = Q + (size_t)j * ldq;
    copy_matrix(q, rows, Y + (size_t)j * ldy, rows, rows, 1);
    for (int pass = 0; pass < 2 && j > 0; ++pass) {
      gemv(true, rows, j, 1.0, Q, ldq, q, 0.0, w);
      gemv(false, rows, j, -1.0, Q, ldq, w, 1.0, q);
    }
    dot_self_kernel<<<1, 512, 0, ctx.stream>>>(q, rows, nrm); ::fpls::note_launch();
    normalize_col_kernel<<<ceil_div(rows, 256), 256, 0, ctx.stream>>>(q, rows, nrm); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
}

void qr_orthonormalize(int rows, int cols, const double* Y, int ldy, double* Q, int ldq) {
  if (cols <= 0 || rows <= 0) return;
  Context& ctx = Context::get();
  double* G = ctx.arena.alloc_n<double>((size_t)cols * cols);
  int* flag = ctx.d_status + 8;
  dzero(flag, sizeof(int));
  const double* src = Y;
  int lds = ldy;
  const size_t smem = (size_t)cols * cols * sizeof(double);
  const bool fits = smem <= 200 * 1024;
  if (fits) {
    static bool attr_set = false;
    if (!attr_set) {
      FPLS_CUDA(cudaFuncSetAttribute(trsm_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      attr_set = true;
    }
    for (int pass = 0; pass < 2; ++pass) {
      gemm(true, false, cols, cols, rows, 1.0, src, lds, src, lds, 0.0, G, cols);
      chol_upper_kernel<<<1, 512, 0, ctx.stream>>>(G, cols, flag); ::fpls::note_launch();
      trsm_rows_kernel<<<ceil_div(rows, 128), 128, smem, ctx.stream>>>(rows, cols, src, lds, G, Q, ldq); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
      src = Q;
      lds = ldq;
    }
    int h = 0;
    FPLS_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    FPLS_CUDA(cudaStreamSynchronize(ctx.stream));
    if (h == 0) return;
  }
  cgs2_orthonormalize(rows, cols, Y, ldy, Q, ldq);
}

void eig_sym_desc(int l, const double* G, int ldg, double* evals, double* V, int ldv) {
  if (l <= 0) return;
  Context& ctx = Context::get();
  double* W = ctx.arena.alloc_n<double>((size_t)l * l);
  double* Vw = ctx.arena.alloc_n<double>((size_t)l * l);
  copy_matrix(W, l, G, ldg, l, l);
  const int npair = (l + 1) / 2;
  const size_t tables = (size_t)npair * 2 * sizeof(double) + (size_t)(2 * npair + 2 * npair) * sizeof(int);
  const size_t with_mats = tables + 2 * (size_t)l * l * sizeof(double) + 64;
  constexpr size_t kEigSmemMax = 200 * 1024;
  const bool in_smem = with_mats <= kEigSmemMax;
  static bool attr_set = false;
  if (!attr_set) {
    FPLS_CUDA(cudaFuncSetAttribute(jacobi_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEigSmemMax));
    attr_set = true;
  }
  const size_t smem = in_smem ? with_mats : tables + 64;
  jacobi_eig_kernel<<<1, 1024, smem, ctx.stream>>>(l, W, Vw, evals, V, ldv, 60, in_smem ? 1 : 0);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

void svd_thin(int rows, int cols, const double* A, int lda, double* U, int ldu, double* s,
              double* V, int ldv) {
  if (rows <= 0 || cols <= 0) return;
  Context& ctx = Context::get();
  const bool tall = rows >= cols;
  const int r = tall ? rows : cols;
  const int c = tall ? cols : rows;
  double* W = ctx.arena.alloc_n<double>((size_t)r * c);
  double* Vw = ctx.arena.alloc_n<double>((size_t)c * c);
  if (tall) {
    copy_matrix(W, r, A, lda, rows, cols);
  } else {
    transpose_kernel<<<256, 256, 0, ctx.stream>>>(A, rows, cols, lda, W); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
  }
  const int ce = c + (c & 1);
  const size_t smem = (size_t)(2 * ce + 2) * sizeof(int) + (size_t)(c + 2) * sizeof(double) + 64;
  // tall: U (rows x c) <- normalised W, V (cols x c) <- rotations.
  // wide: A^T = U' S V'^T, so U (rows x c) <- V', V (cols x c) <- U'.
  jacobi_svd_kernel<<<1, 1024, smem, ctx.stream>>>(r, c, W, Vw, 60, U, ldu, s, V, ldv, tall ? 0 : 1); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

}  // namespace fpls
