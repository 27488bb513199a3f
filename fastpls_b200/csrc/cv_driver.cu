#include "autotune.cuh"
#include "blas_f64.cuh"
#include "context.cuh"
#include "cv_driver.cuh"
#include "dual_engine.cuh"
#include "gaussian.cuh"
#include "fits.cuh"
#include "heads.cuh"
#include "ozaki_gemm.cuh"
#include "simpls_engine.cuh"
#include "svd.cuh"
#include "xop_split.cuh"

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <numeric>
#include <string>
#include <thread>

namespace fpls {
namespace {

constexpr int kMaxClassesCv = 128;

// dst (n x p, ld n) = src - mean (per column; mean may be null), widened to
// FP64: the centred working copy in one pass over the caller's matrix.
template <typename T>
__global__ void load_centered_kernel(const T* __restrict__ src, int n, int p, const double* __restrict__ mean,
                                     double* __restrict__ dst) {
  const size_t total = (size_t)n * p;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    double v = static_cast<double>(src[idx]);
    if (mean) v -= mean[idx / n];
    dst[idx] = v;
  }
}

// The mixed-mode row-space products run on the INT8 tensor cores unless
// FASTPLS_KPROD=fp64 asks for FP64 DMMA.
bool int8_k_products() {
  const char* e = std::getenv("FASTPLS_KPROD");
  return !(e && std::string(e) == "fp64");
}

// Digit slices of the INT8 row Gram (FASTPLS_GRAM_SLICES, else 5: 35 bits of
// every centred row against its largest entry).  With 4 slices the omics
// double-CV grid's class scores sit within 4.1e-6 of the FP64 grid, with 5
// within 6.2e-7 (FP64 itself moves by 8.6e-7 under a 2^-24 relative change of
// X) for 0.06 ms more.
int int8_gram_slices() {
  if (const char* e = std::getenv("FASTPLS_GRAM_SLICES")) {
    const int v = std::atoi(e);
    if (v >= kOzakiMinSlices && v <= kOzakiMaxSlices) return v;
  }
  return 5;
}

// Digit slices of the INT8 grids' K products: 6 unless set.  The row-space loop
// amplifies product errors about 10^6-fold by the 30th component: with 5
// slices (2^-35) the last components' scores drift to 6.3e-5 of FP64, with 6
// and 7 they stay within the Gram's error.
int int8_mode_kprod_slices() {
  if (const char* e = std::getenv("FASTPLS_OZAKI_SLICES")) {
    const int v = std::atoi(e);
    if (v >= kOzakiMinSlices && v <= kOzakiMaxSlices) return v;
  }
  const int t = active_tune().ozaki_slices;
  if (t >= kOzakiMinSlices && t <= kOzakiMaxSlices) return t;
  return 6;
}

void load_centered(const double* x64, const float* x32, int n, int p, const double* mean, double* dst) {
  Context& ctx = Context::get();
  if (x64) load_centered_kernel<double><<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(x64, n, p, mean, dst);
  else load_centered_kernel<float><<<4 * ctx.sm_count, 256, 0, ctx.stream>>>(x32, n, p, mean, dst);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
}

__global__ void mask_to_double_kernel(const uint8_t* __restrict__ mask, size_t total,
                                      double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = mask[i] ? 1.0 : 0.0;
}

__global__ void scale_cols_kernel(double* P, int p, int F, const double* inv_nf) {
  const size_t total = (size_t)p * F;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x)
    P[t] *= inv_nf[t / p];
}

// Gathers rows `idx` (device, cnt) of X (n x p) into out (cnt x p).
__global__ void gather_rows_kernel(const double* __restrict__ X, int n, int p,
                                   const int* __restrict__ idx, int cnt, double* __restrict__ out) {
  const size_t total = (size_t)cnt * p;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int r = static_cast<int>(t % cnt);
    const int j = static_cast<int>(t / cnt);
    out[t] = X[idx[r] + (size_t)j * n];
  }
}

__global__ void onehot_kernel(const int* __restrict__ lab0, int cnt, int m, double* Y) {
  const size_t total = (size_t)cnt * m;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int r = static_cast<int>(t % cnt);
    const int j = static_cast<int>(t / cnt);
    Y[t] = (lab0[r] == j) ? 1.0 : 0.0;
  }
}

// Scatters the class labels of one fit's test rows into the prediction grid.
__global__ void scatter_pred_kernel(const int* __restrict__ lab, int nt, int L, const int* __restrict__ rows,
                                    int n, int g, int* __restrict__ pred) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt * L) return;
  const int r = t % nt, s = t / nt;
  pred[((size_t)g * L + s) * n + rows[r]] = lab[t];
}

// Class scores of the test rows of one sequential fit (Yp: L slices of nt x m,
// column-major) into the grid's score array at the rows' own indices.
__global__ void scatter_score_kernel(const double* __restrict__ Yp, int nt, int m, int L,
                                     const int* __restrict__ rows, int n, int g, double* __restrict__ score) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nt * m * L) return;
  const int r = static_cast<int>(t % nt);
  const int j = static_cast<int>((t / nt) % m);
  const int s = static_cast<int>(t / ((long long)nt * m));
  score[(((size_t)g * L + s) * n + rows[r]) * m + j] = Yp[t];
}

__global__ void pred_counts_kernel(const int* __restrict__ pred, int L, int n, const int* __restrict__ y,
                                   const int* __restrict__ exclude, long long* __restrict__ counts) {
  __shared__ double scratch[32];
  const int gs = blockIdx.x;          // g * L + s
  const int g = gs / L;
  const int* pr = pred + (size_t)gs * n;
  double ok = 0.0, tot = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (exclude && exclude[i] == g) continue;
    const int v = pr[i];
    if (v < 1) continue;
    tot += 1.0;
    ok += (v == y[i]) ? 1.0 : 0.0;
  }
  ok = block_sum(ok, scratch);
  tot = block_sum(tot, scratch);
  if (threadIdx.x == 0) {
    counts[2 * (size_t)gs] = static_cast<long long>(ok);
    counts[2 * (size_t)gs + 1] = static_cast<long long>(tot);
  }
}

// Class predictions of the test rows of every fit for every ncomp slice from the
// kept scores: y_a = sum_{b<=a} (t_b[i] / ||t_b||) q_b + mY_f, label = first argmax.
// MB bounds the class count so that the running scores stay in registers.
// Thread k of fit f takes the fit's k-th test row (tidx[f * tstride + k], k <
// tcnt[f]), so no warp runs for training rows.
template <int MB>
__global__ void cv_predict_kernel(int F, int n, int m, int K, int L, const int* __restrict__ ncomp,
                                  const int* __restrict__ order, const int* __restrict__ tidx,
                                  const int* __restrict__ tcnt, int tstride,
                                  const int* __restrict__ group, const double* __restrict__ Tkeep,
                                  const double* __restrict__ tnorm, const double* __restrict__ Q,
                                  const int* __restrict__ ncomp_done, const double* __restrict__ mYf,
                                  int* __restrict__ pred, double* __restrict__ score) {
  const int f = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= tcnt[f]) return;
  const int i = tidx[(size_t)f * tstride + k];
  const int done = ncomp_done[f];
  const int g = group[f];
  double y[MB];
#pragma unroll
  for (int j = 0; j < MB; ++j) y[j] = 0.0;
  const double* Qf = Q + (size_t)f * m * K;
  const double* mf = mYf + (size_t)f * m;
  const double* tk = Tkeep + (size_t)f * K * n + i;
  // the slices in increasing ncomp (order), each written once y holds its
  // components; the scores of four components are loaded together
  int next = 0;
  int nc_next = L > 0 ? ncomp[order[0]] : 0;
  for (int a0 = 0; a0 < K; a0 += 4) {
    double t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) t[u] = a0 + u < done ? tk[(size_t)(a0 + u) * n] : 0.0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int a = a0 + u;
      if (a >= K) break;
      if (a < done) {
        const double c = t[u] / tnorm[(size_t)f * K + a];
#pragma unroll
        for (int j = 0; j < MB; ++j)
          if (j < m) y[j] += c * Qf[j + (size_t)a * m];
      }
      while (next < L && nc_next == a + 1) {
        const int s = order[next];
        int best = 0;
        double bv = y[0] + mf[0];
#pragma unroll
        for (int j = 1; j < MB; ++j) {
          if (j >= m) break;
          const double v = y[j] + mf[j];
          if (v > bv) { bv = v; best = j; }
        }
        pred[((size_t)g * L + s) * n + i] = best + 1;
        if (score) {
          double* sc = score + (((size_t)g * L + s) * n + i) * m;
#pragma unroll
          for (int j = 0; j < MB; ++j)
            if (j < m) sc[j] = y[j] + mf[j];
        }
        if (++next < L) nc_next = ncomp[order[next]];
      }
    }
  }
}

// Fold status and class counts of each fit (host): the reference's rules
// (fastPLS.cpp:6805-6870): 2 empty test fold, 3 no training rows, 4 at most
// one class present in the training rows (constant prediction).
void classify_fits(const CvFitSet& fs, const int* y, std::vector<int>& status,
                   std::vector<int>& fallback, std::vector<double>& counts) {
  status.assign(fs.F, 1);
  fallback.assign(fs.F, 1);
  counts.assign((size_t)fs.F * fs.m, 0.0);
  const bool given = !fs.train_class_counts.empty();
  std::vector<int> cnt(fs.m);
  for (int f = 0; f < fs.F; ++f) {
    int ntest = 0, ntrain = 0;
    if (given) {
      ntest = fs.n_test[f];
      ntrain = fs.n_train[f];
      for (int c = 0; c < fs.m; ++c) counts[(size_t)f * fs.m + c] = fs.train_class_counts[(size_t)f * fs.m + c];
    } else {
      std::fill(cnt.begin(), cnt.end(), 0);
      const uint8_t* te = fs.test.data() + (size_t)f * fs.n;
      const uint8_t* tr = fs.train.data() + (size_t)f * fs.n;
      for (int i = 0; i < fs.n; ++i) {
        ntest += te[i];
        ntrain += tr[i];
        cnt[y[i] - 1] += tr[i];
      }
      for (int c = 0; c < fs.m; ++c) counts[(size_t)f * fs.m + c] = cnt[c];
    }
    if (ntest == 0) { status[f] = 2; continue; }
    if (ntrain == 0) { status[f] = 3; continue; }
    int active = 0, last = -1;
    for (int c = 0; c < fs.m; ++c)
      if (counts[(size_t)f * fs.m + c] > 0.5) { ++active; last = c; }
    if (active <= 1) {
      status[f] = 4;
      fallback[f] = active == 1 ? last + 1 : 1;
    }
  }
}

void fill_special_predictions(const CvFitSet& fs, const int* y, const std::vector<int>& status,
                              const std::vector<int>& fallback, int L, std::vector<int>& pred) {
  for (int f = 0; f < fs.F; ++f) {
    if (status[f] == 1 || status[f] == 2) continue;
    const int g = fs.group[f];
    for (int i = 0; i < fs.n; ++i) {
      if (!fs.test[(size_t)f * fs.n + i]) continue;
      const int v = status[f] == 3 ? y[i] : fallback[f];
      for (int s = 0; s < L; ++s) pred[((size_t)g * L + s) * fs.n + i] = v;
    }
  }
}

// Column chunks of the overlapped upload of X: 4096 columns each, except that
// the work of the LAST chunk (its means, split and Gram) follows the last copy
// instead of overlapping one, so the end of X goes in a narrow chunk of about
// kUploadTailCols columns.  Chunk starts are multiples of 64 (one K-block of
// the Gram).  Returns the nch + 1 column boundaries.
constexpr int kUploadChunkCols = 4096;
constexpr int kUploadTailCols = 1024;

std::vector<int> upload_chunks(int p, int align) {
  std::vector<int> b{0};
  while (p - b.back() > kUploadChunkCols + kUploadTailCols) b.push_back(b.back() + kUploadChunkCols);
  const int tail0 = (p - kUploadTailCols) / align * align;
  if (tail0 - b.back() >= kUploadTailCols / 2) b.push_back(tail0);
  b.push_back(p);
  return b;
}

}  // namespace

std::unique_ptr<CvPreparedX> cv_prepare_x(const double* x64, const float* x32, int n, int p, int m, int kmax,
                                          const CvGridOptions& opt, const void* x_host) {
  Context& ctx = Context::get();
  Arena& ar = ctx.arena;
  FPLS_REQUIRE(opt.batched && opt.scaling != 2, "X preparation is for batched grids");
  std::unique_ptr<CvPreparedX> px(new CvPreparedX());
  px->n = n; px->p = p; px->m = m; px->kmax = kmax; px->precision = opt.precision;
  PhaseTimer pt("CV grid X preparation");
  // Global centring (scaling < 3): Xc = X - mean(X); folds shift by delta_f.
  const bool center = px->center = opt.scaling < 3;
  // Short, wide predictor blocks run the loop in the row space of X (the
  // row Gram K = Xc Xc^T); otherwise in the predictor space.
  const bool dual = px->dual = dual_engine_applies(n, p, m, kmax);
  // The mixed row-space loop needs only the BF16 planes of Xc, split straight
  // from the caller's matrix; every other combination works on a centred FP64
  // copy.  x0 is the first column of Xc (the Householder sign of the sketch).
  // INT8 grids build the row Gram (and the sketch product) from digit planes
  // of the centred rows; off the row-space path they run in FP64.
  const bool int8_gram = opt.precision == 3 && dual;
  const bool planes_only = (opt.precision == 1 || opt.precision == 2) && dual;
  const int planes = opt.precision == 2 ? 3 : 2;  // BF16x6: hi, mid, lo planes
  // A host X goes up in overlapped column chunks on the mixed and INT8
  // row-space paths, else in one copy first.
  if (x_host && !planes_only && !int8_gram) {
    if (x64) h2d(const_cast<double*>(x64), x_host, (size_t)n * p * sizeof(double));
    else h2d(const_cast<float*>(x32), x_host, (size_t)n * p * sizeof(float));
    x_host = nullptr;
  }
  double* mall = px->mall = center ? ar.alloc_n<double>(p) : nullptr;
  double* Kg = px->Kg = dual ? ar.alloc_n<double>((size_t)n * n) : nullptr;
  bool gram_done = false;
  double* X = nullptr;
  double* x0 = nullptr;
  std::unique_ptr<XOperator> xop;

  if (x_host) {
    // X arrives in column chunks on the copy stream; each chunk's column means,
    // BF16 planes (or INT8 digit planes with the chunk's own row scales) and
    // row-Gram contribution run as soon as it has landed, while the next chunk
    // is in flight (copies and compute are enqueued in turn, so a pageable
    // host buffer overlaps too).
    const size_t esz = x64 ? sizeof(double) : sizeof(float);
    char* dst = x64 ? reinterpret_cast<char*>(const_cast<double*>(x64)) : reinterpret_cast<char*>(const_cast<float*>(x32));
    const char* src = static_cast<const char*>(x_host);
    const std::vector<int> bounds = upload_chunks(p, int8_gram ? 128 : 64);
    const int nch = static_cast<int>(bounds.size()) - 1;
    xop = int8_gram ? make_ozaki_rows_chunked(n, p, int8_gram_slices(), bounds)
                    : make_split_operator_chunked(n, p, planes);
    x0 = ar.alloc_n<double>(n);
    // the copies follow this call's earlier work on the main stream (an event
    // of their own: side_done marks the sketches, awaited later)
    FPLS_CUDA(cudaEventRecord(ctx.copy_event(nch), ctx.stream));
    FPLS_CUDA(cudaStreamWaitEvent(ctx.copy, ctx.copy_event(nch), 0));
    auto chunk_work = [&](int c) {
      const int j0 = bounds[c], j1 = bounds[c + 1];
      FPLS_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.copy_event(c), 0));
      const double* c64 = x64 ? x64 + (size_t)j0 * n : nullptr;
      const float* c32 = x32 ? x32 + (size_t)j0 * n : nullptr;
      if (center) {
        if (c64) col_mean(c64, n, j1 - j0, n, mall + j0);
        else col_mean(c32, n, j1 - j0, n, mall + j0);
      }
      if (int8_gram) ozaki_rows_fill_chunk(*xop, c64, c32, center ? mall + j0 : nullptr, c);
      else split_operator_fill_columns(*xop, c64, c32, center ? mall + j0 : nullptr, j0, j1);
      if (c == 0) load_centered(x64, x32, n, 1, mall, x0);
      if (c == nch - 1) FPLS_CUDA(cudaEventRecord(ctx.planes_ready, ctx.stream));
      if (int8_gram) ozaki_rows_gram_chunk(*xop, Kg, c, c > 0);
      else split_operator_gram_columns(*xop, Kg, j0, j1, c > 0);
    };
    for (int c = 0; c < nch; ++c) {
      const int j0 = bounds[c], j1 = bounds[c + 1];
      FPLS_CUDA(cudaMemcpyAsync(dst + (size_t)j0 * n * esz, src + (size_t)j0 * n * esz, (size_t)(j1 - j0) * n * esz,
                                cudaMemcpyDefault, ctx.copy));
      FPLS_CUDA(cudaEventRecord(ctx.copy_event(c), ctx.copy));
      if (c > 0) chunk_work(c - 1);
    }
    chunk_work(nch - 1);
    mirror_upper_triangle(Kg, n);
    gram_done = true;
    pt.mark("upload + split + row gram");
  } else {
    if (center) {
      if (x64) col_mean(x64, n, p, n, mall);
      else col_mean(x32, n, p, n, mall);
    }
    pt.mark("column means");
    if (planes_only) {
      x0 = ar.alloc_n<double>(n);
      load_centered(x64, x32, n, 1, mall, x0);
      xop = make_split_operator_centered(x64, x32, mall, n, p, planes);
    } else if (int8_gram) {
      x0 = ar.alloc_n<double>(n);
      load_centered(x64, x32, n, 1, mall, x0);
      xop = make_ozaki_rows_operator(x64, x32, mall, n, p, int8_gram_slices());
    } else {
      X = ar.alloc_n<double>((size_t)n * p);
      load_centered(x64, x32, n, p, mall, X);
      x0 = X;
      if (opt.precision == 1 || opt.precision == 2) xop = make_split_operator(X, n, p, !dual, planes);
      else xop.reset(new XOperatorF64(X, n, p));
    }
    FPLS_CUDA(cudaEventRecord(ctx.planes_ready, ctx.stream));
  }
  pt.mark("operator");
  // The Gram contracts over all p columns (BF16x3 on the tensor cores in the
  // mixed mode); the per-component products with the L2-resident K stay
  // FP64-accurate: the K-coordinate Gram-Schmidt carries K C_V and K C_S
  // forward, and split-precision products there drift from one component to
  // the next.  Mixed mode: the K products on the INT8 tensor cores (digit
  // planes of K split once); FP64 mode: FP64 DMMA.
  if (dual) {
    if (!gram_done) xop->gram(Kg);
    px->kop_f64.reset(new XOperatorF64(Kg, n, n));
    if ((opt.precision >= 1 && opt.precision <= 2 && int8_k_products()) || int8_gram) {
      px->kop_slices = int8_gram ? int8_mode_kprod_slices() : ozaki_default_slices();
      px->kop_int8 = make_ozaki_sym_operator(Kg, n, px->kop_slices);
    }
    pt.mark("row gram");
  }
  px->X = X;
  px->x0 = x0;
  px->xop = std::move(xop);
  pt.report();
  return px;
}

namespace {

void run_batched(const CvFitSet& fs, const int* y, const int* ncomp, int L, const CvGridOptions& opt,
                 const std::vector<int>& status, const std::vector<double>& counts, double* d_om,
                 CvGridResult& res, CvPreparedX& px) {
  Context& ctx = Context::get();
  Arena& ar = ctx.arena;
  const int n = fs.n, p = fs.p, m = fs.m;
  const int K = *std::max_element(ncomp, ncomp + L);
  FPLS_REQUIRE(m <= kMaxClassesCv, "batched CV supports at most 128 classes");
  FPLS_REQUIRE(px.n == n && px.p == p && px.m == m && px.kmax == K && px.precision == opt.precision,
               "prepared X does not match the grid");
  // Active fits only (status 1) go to the engine.
  std::vector<int> act;
  for (int f = 0; f < fs.F; ++f)
    if (status[f] == 1) act.push_back(f);
  const int Fa = static_cast<int>(act.size());
  if (Fa == 0) return;
  PhaseTimer pt("CV grid (batched)");
  const bool center = px.center, dual = px.dual;
  double* X = px.X;
  double* x0 = px.x0;
  std::unique_ptr<XOperator>& xop = px.xop;
  std::vector<uint8_t> tr((size_t)Fa * n), te((size_t)Fa * n);
  std::vector<int> grp(Fa), ntrain(Fa), tcnt(Fa, 0);
  std::vector<double> inv_nf(Fa), mYf((size_t)Fa * m), mYall(m, 0.0), dY((size_t)Fa * m);
  for (int i = 0; i < n; ++i) mYall[y[i] - 1] += 1.0 / n;
  for (int a = 0; a < Fa; ++a) {
    const int f = act[a];
    std::copy(fs.train.begin() + (size_t)f * n, fs.train.begin() + (size_t)(f + 1) * n, tr.begin() + (size_t)a * n);
    std::copy(fs.test.begin() + (size_t)f * n, fs.test.begin() + (size_t)(f + 1) * n, te.begin() + (size_t)a * n);
    grp[a] = fs.group[f];
    for (int i = 0; i < n; ++i) tcnt[a] += te[(size_t)a * n + i] != 0;
    int nt = 0;
    if (!fs.n_train.empty()) {
      nt = fs.n_train[f];
    } else {
      const uint8_t* trf = fs.train.data() + (size_t)f * n;
      for (int i = 0; i < n; ++i) nt += trf[i];
    }
    ntrain[a] = nt;
    inv_nf[a] = 1.0 / nt;
    for (int c = 0; c < m; ++c) {
      mYf[(size_t)a * m + c] = counts[(size_t)f * m + c] / nt;
      dY[(size_t)a * m + c] = mYf[(size_t)a * m + c] - mYall[c];
    }
  }
  uint8_t* d_tr = ar.alloc_n<uint8_t>(tr.size());
  int* d_grp = ar.alloc_n<int>(Fa);
  int* d_nt = ar.alloc_n<int>(Fa);
  double* d_inv = ar.alloc_n<double>(Fa);
  double* d_mYf = ar.alloc_n<double>(mYf.size());
  double* d_mYall = ar.alloc_n<double>(m);
  double* d_dY = ar.alloc_n<double>(dY.size());
  int* d_lab = ar.alloc_n<int>(n);
  int* d_nc = ar.alloc_n<int>(L);
  std::vector<int> lab0(n);
  for (int i = 0; i < n; ++i) lab0[i] = y[i] - 1;
  h2d(d_tr, tr.data(), tr.size());
  h2d(d_grp, grp.data(), Fa * sizeof(int));
  h2d(d_nt, ntrain.data(), Fa * sizeof(int));
  h2d(d_inv, inv_nf.data(), Fa * sizeof(double));
  h2d(d_mYf, mYf.data(), mYf.size() * sizeof(double));
  h2d(d_mYall, mYall.data(), m * sizeof(double));
  h2d(d_dY, dY.data(), dY.size() * sizeof(double));
  h2d(d_lab, lab0.data(), n * sizeof(int));
  h2d(d_nc, ncomp, L * sizeof(int));
  // slice indices in increasing ncomp (ties in slice order) for the predictions
  std::vector<int> order(L);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return ncomp[u] < ncomp[v]; });
  int* d_order = ar.alloc_n<int>(L);
  h2d(d_order, order.data(), L * sizeof(int));
  double* Qo = ar.alloc_n<double>((size_t)Fa * m * K);
  double* tno = ar.alloc_n<double>((size_t)Fa * K);
  double* Tko = ar.alloc_n<double>((size_t)Fa * n * K);
  int* ncd = ar.alloc_n<int>(Fa);
  int* sto = ar.alloc_n<int>(Fa);
  if (dual) {
    XOperator* kop = px.kop_int8 ? px.kop_int8.get() : px.kop_f64.get();
    const int kop_slices = px.kop_slices;
    pt.mark("fold set-up");
    FPLS_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.side_done, 0));
    double* XOm = px.XOm;
    if (!XOm) {
      XOm = ar.alloc_n<double>((size_t)n * Fa);
      xop->times(d_om, Fa, XOm);
    }
    pt.mark("sketch");
    DualBatch db;
    db.n = n; db.m = m; db.F = Fa; db.K = K;
    db.power_iters = opt.power_iters;
    db.m1_mode = (m == 1);
    db.center = center;
    db.Kop = kop;
    db.kop_int8_slices = kop_slices;
    db.x0 = x0;
    db.XOmega = XOm;
    db.mask = d_tr;
    db.labels = d_lab;
    db.mY_all = d_mYall;
    db.dY = d_dY;
    db.ntrain = d_nt;
    {
      std::vector<double> cc((size_t)Fa * m);
      for (int a = 0; a < Fa; ++a)
        for (int c = 0; c < m; ++c) cc[(size_t)a * m + c] = counts[(size_t)act[a] * m + c];
      double* d_cc = ar.alloc_n<double>(cc.size());
      h2d(d_cc, cc.data(), cc.size() * sizeof(double));
      db.class_cnt = d_cc;
    }
    db.Q = Qo; db.tnorm = tno; db.Tkeep = Tko; db.ncomp_done = ncd; db.status = sto;
    dual_simpls_run(db);
    pt.mark("simpls");
  } else {
    SimplsBatch b;
    b.n = n; b.p = p; b.m = m; b.F = Fa; b.K = K;
    b.power_iters = opt.power_iters;
    b.X = xop.get();
    b.labels = d_lab;
    b.mY_all = d_mYall;
    b.mask = d_tr;
    b.dY = d_dY;
    b.omega = d_om;
    b.m1_mode = (m == 1);
    // Fold column sums X^T D_f 1 centre the response in S_f; divided by the
    // fold sizes they are the fold offsets delta_f when X is centred.
    double* Mtr = ar.alloc_n<double>((size_t)Fa * n);
    double* colsum = ar.alloc_n<double>((size_t)Fa * p);
    mask_to_double_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(d_tr, (size_t)Fa * n, Mtr); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    xop->t_times(Mtr, Fa, colsum);
    double* delta = nullptr;
    if (center) {
      delta = ar.alloc_n<double>((size_t)Fa * p);
      d2d(delta, colsum, (size_t)Fa * p * sizeof(double));
      scale_cols_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(delta, p, Fa, d_inv); ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
    b.delta = delta;
    b.colsum = colsum;
    pt.mark("fold means");
    b.S = ar.alloc_n<double>((size_t)Fa * p * m);
    simpls_batch_crosscov(b, X, d_nt);
    pt.mark("crosscov");
    FPLS_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.side_done, 0));
    pt.mark("sketch");
    b.R = ar.alloc_n<double>((size_t)Fa * p * K);
    b.Q = Qo;
    b.V = ar.alloc_n<double>((size_t)Fa * p * K);
    b.tnorm = tno;
    b.Tkeep = Tko;
    b.ncomp_done = ncd;
    b.status = sto;
    simpls_batch_run(b);
    pt.mark("simpls");
  }
  int* d_pred = res.d_pred;
  // every fit's test rows as a compact list (the prediction threads)
  const int tstride = std::max(1, *std::max_element(tcnt.begin(), tcnt.end()));
  std::vector<int> tidx((size_t)Fa * tstride, 0);
  for (int a = 0; a < Fa; ++a) {
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (te[(size_t)a * n + i]) tidx[(size_t)a * tstride + k++] = i;
  }
  int* d_tidx = ar.alloc_n<int>(tidx.size());
  int* d_tcnt = ar.alloc_n<int>(Fa);
  h2d(d_tidx, tidx.data(), tidx.size() * sizeof(int));
  h2d(d_tcnt, tcnt.data(), Fa * sizeof(int));
  const dim3 pgrid(ceil_div(tstride, 128), Fa);
  if (m <= 8)
    cv_predict_kernel<8><<<pgrid, 128, 0, ctx.stream>>>(Fa, n, m, K, L, d_nc, d_order, d_tidx, d_tcnt, tstride, d_grp,
                                                        Tko, tno, Qo, ncd, d_mYf, d_pred, res.d_score);
  else if (m <= 32)
    cv_predict_kernel<32><<<pgrid, 128, 0, ctx.stream>>>(Fa, n, m, K, L, d_nc, d_order, d_tidx, d_tcnt, tstride, d_grp,
                                                         Tko, tno, Qo, ncd, d_mYf, d_pred, res.d_score);
  else
    cv_predict_kernel<kMaxClassesCv><<<pgrid, 128, 0, ctx.stream>>>(Fa, n, m, K, L, d_nc, d_order, d_tidx, d_tcnt,
                                                                    tstride, d_grp, Tko, tno, Qo, ncd, d_mYf, d_pred,
                                                                    res.d_score);
  ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  pt.mark("predict");
  pt.report();
}

void run_sequential(const CvFitSet& fs, const double* X, const int* y, const int* ncomp, int L,
                    const CvGridOptions& opt, const std::vector<int>& status, CvGridResult& res) {
  Context& ctx = Context::get();
  Arena& ar = ctx.arena;
  const int n = fs.n, p = fs.p, m = fs.m;
  const int K = *std::max_element(ncomp, ncomp + L);
  // Per-fit buffers sized for the largest fold, reused fit after fit.
  double* Xf = ar.alloc_n<double>((size_t)n * p);
  double* Xt = ar.alloc_n<double>((size_t)n * p);
  double* Yf = ar.alloc_n<double>((size_t)n * m);
  int* d_idx = ar.alloc_n<int>(n);
  int* d_lab = ar.alloc_n<int>(n);
  double* mX = ar.alloc_n<double>(p);
  double* vX = ar.alloc_n<double>(p);
  double* mY = ar.alloc_n<double>(m);
  double* om = ar.alloc_n<double>(p);
  double* S = ar.alloc_n<double>((size_t)p * m);
  double* R = ar.alloc_n<double>((size_t)p * K);
  double* Q = ar.alloc_n<double>((size_t)m * K);
  double* V = ar.alloc_n<double>((size_t)p * K);
  double* tn = ar.alloc_n<double>(K);
  int* ncd = ar.alloc_n<int>(1);
  int* st = ar.alloc_n<int>(1);
  double* W = ar.alloc_n<double>((size_t)K * m * L);
  double* T = ar.alloc_n<double>((size_t)n * K);
  double* Yp = ar.alloc_n<double>((size_t)n * m * L);
  int* lab = ar.alloc_n<int>((size_t)n * L);
  std::vector<double> Wh((size_t)K * m * L), Qh((size_t)m * K);
  std::vector<int> rows, trows, labs;
  for (int f = 0; f < fs.F; ++f) {
    if (status[f] != 1) continue;
    rows.clear();
    trows.clear();
    labs.clear();
    for (int i = 0; i < n; ++i) {
      if (fs.train[(size_t)f * n + i]) { rows.push_back(i); labs.push_back(y[i] - 1); }
      if (fs.test[(size_t)f * n + i]) trows.push_back(i);
    }
    const int nf = static_cast<int>(rows.size());
    const int nt = static_cast<int>(trows.size());
    h2d(d_idx, rows.data(), nf * sizeof(int));
    h2d(d_lab, labs.data(), nf * sizeof(int));
    gather_rows_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(X, n, p, d_idx, nf, Xf); ::fpls::note_launch();
    onehot_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(d_lab, nf, m, Yf); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    center_scale_xy(Xf, nf, p, Yf, m, opt.scaling, mX, vX, mY);
    gemm(true, false, p, m, nf, 1.0, Xf, nf, Yf, nf, 0.0, S, p);
    device_gaussian(om, p, fs.seeds[f]);
    XOperatorF64 xop(Xf, nf, p);
    SimplsBatch b;
    b.n = nf; b.p = p; b.m = m; b.F = 1; b.K = K;
    b.power_iters = opt.power_iters;
    b.X = &xop;
    b.Yg = Yf;
    b.S = S;
    b.omega = om;
    b.m1_mode = (m == 1);
    b.R = R; b.Q = Q; b.V = V; b.tnorm = tn; b.ncomp_done = ncd; b.status = st;
    simpls_batch_run(b);
    // Compact class prediction of the test rows (pls_predict_classes_compact_cuda).
    d2h(Qh.data(), Q, (size_t)m * K * sizeof(double));
    ctx.sync();
    std::fill(Wh.begin(), Wh.end(), 0.0);
    for (int s = 0; s < L; ++s)
      for (int a = 0; a < ncomp[s]; ++a)
        for (int j = 0; j < m; ++j) Wh[a + (size_t)j * K + (size_t)s * K * m] = Qh[j + (size_t)a * m];
    h2d(W, Wh.data(), Wh.size() * sizeof(double));
    h2d(d_idx, trows.data(), nt * sizeof(int));
    gather_rows_kernel<<<2 * ctx.sm_count, 256, 0, ctx.stream>>>(X, n, p, d_idx, nt, Xt); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    center_scale(Xt, nt, p, nt, mX, opt.scaling == 2 ? vX : nullptr);
    lowrank_predict(Xt, nt, p, R, K, W, m, ncomp, L, mY, T, Yp);
    for (int s = 0; s < L; ++s) row_argmax(Yp + (size_t)s * nt * m, nt, m, nullptr, lab + (size_t)s * nt);
    scatter_pred_kernel<<<ceil_div((long long)nt * L, 256), 256, 0, ctx.stream>>>(lab, nt, L, d_idx, n, fs.group[f], res.d_pred); ::fpls::note_launch();
    FPLS_CHECK_LAUNCH();
    if (res.d_score) {
      scatter_score_kernel<<<ceil_div((long long)nt * m * L, 256), 256, 0, ctx.stream>>>(Yp, nt, m, L, d_idx, n,
                                                                                          fs.group[f], res.d_score);
      ::fpls::note_launch();
      FPLS_CHECK_LAUNCH();
    }
  }
}

}  // namespace

void cv_grid_classify(const CvFitSet& fs, const double* x64, const float* x32,
                      const int* labels_host, const int* ncomp, int L,
                      const CvGridOptions& opt, CvGridResult& res, const void* x_host, CvPreparedX* prep) {
  Context& ctx = Context::get();
  PhaseTimer pt("CV grid set-up");
  FPLS_REQUIRE(L >= 1, "ncomp must contain at least one value");
  for (int s = 0; s < L; ++s) FPLS_REQUIRE(ncomp[s] >= 1, "ncomp values must be >= 1");
  for (int i = 0; i < fs.n; ++i)
    FPLS_REQUIRE(labels_host[i] >= 1 && labels_host[i] <= fs.m, "labels must be in 1..n_classes");
  FPLS_REQUIRE(fs.p > 5 || fs.m == 1, "CV with <= 5 predictors is not supported on the GPU path");
  std::vector<int> status, fallback;
  std::vector<double> counts;
  classify_fits(fs, labels_host, status, fallback, counts);
  res.status = status;
  const bool batched = opt.batched && opt.scaling != 2;
  // The X-side work (and a host X's upload) first, unless the caller enqueued it.
  std::unique_ptr<CvPreparedX> own;
  if (batched && !prep) {
    own = cv_prepare_x(x64, x32, fs.n, fs.p, fs.m, *std::max_element(ncomp, ncomp + L), opt, x_host);
    prep = own.get();
  }
  // The per-fit sketches are drawn on the side stream, overlapping every
  // device step below until the SIMPLS loop needs them.
  double* d_om = nullptr;
  if (batched) {
    std::vector<unsigned> seeds;
    for (int f = 0; f < fs.F; ++f)
      if (status[f] == 1) seeds.push_back(fs.seeds[f]);
    if (!seeds.empty()) {
      unsigned int* d_seeds = ctx.arena.alloc_n<unsigned int>(seeds.size());
      d_om = ctx.arena.alloc_n<double>(seeds.size() * (size_t)fs.p);
      // The sketch buffers are fresh arena memory of this call, so the side
      // stream only follows the work of earlier calls (the call's start event),
      // not the X-side work of this call enqueued before it.
      if (ctx.call_started) {
        FPLS_CUDA(cudaStreamWaitEvent(ctx.side, ctx.call_start, 0));
      } else {
        FPLS_CUDA(cudaEventRecord(ctx.side_done, ctx.stream));
        FPLS_CUDA(cudaStreamWaitEvent(ctx.side, ctx.side_done, 0));
      }
      FPLS_CUDA(cudaMemcpyAsync(d_seeds, seeds.data(), seeds.size() * sizeof(unsigned), cudaMemcpyHostToDevice,
                                ctx.side));
      device_gaussian_streams(d_om, fs.p, fs.p, d_seeds, static_cast<int>(seeds.size()), ctx.side);
      if (prep->dual) {
        // X Omega of the row-space loop also on the side stream: it needs only
        // the operator of X and the sketches, so it overlaps the row Gram.
        FPLS_CUDA(cudaStreamWaitEvent(ctx.side, ctx.planes_ready, 0));
        prep->XOm = ctx.arena.alloc_n<double>((size_t)fs.n * seeds.size());
        StreamSwap on_side(ctx, ctx.side);
        prep->xop->times(d_om, static_cast<int>(seeds.size()), prep->XOm);
      }
      FPLS_CUDA(cudaEventRecord(ctx.side_done, ctx.side));
    }
  }
  pt.mark("classify + sketches");
  const size_t npred = (size_t)fs.G * L * fs.n;
  res.d_pred = ctx.arena.alloc_n<int>(npred);
  bool special = false;
  for (int f = 0; f < fs.F; ++f) special |= (status[f] == 3 || status[f] == 4);
  if (special) {
    std::vector<int> pred(npred, 0);
    fill_special_predictions(fs, labels_host, status, fallback, L, pred);
    h2d(res.d_pred, pred.data(), npred * sizeof(int));
    ctx.sync();
  } else {
    dzero(res.d_pred, npred * sizeof(int));
  }
  if (opt.want_scores) {
    const size_t nscore = npred * (size_t)fs.m;
    res.d_score = ctx.arena.alloc_n<double>(nscore);
    dzero(res.d_score, nscore * sizeof(double));
  }
  pt.mark("prediction buffers");
  pt.report();
  if (batched) {
    run_batched(fs, labels_host, ncomp, L, opt, status, counts, d_om, res, *prep);
    return;
  }
  if (x_host) {
    if (x64) h2d(const_cast<double*>(x64), x_host, (size_t)fs.n * fs.p * sizeof(double));
    else h2d(const_cast<float*>(x32), x_host, (size_t)fs.n * fs.p * sizeof(float));
  }
  // The per-fit path reads X in FP64 (widened once when the caller's is FP32).
  const double* X = x64;
  if (!X) {
    double* w = ctx.arena.alloc_n<double>((size_t)fs.n * fs.p);
    load_centered(nullptr, x32, fs.n, fs.p, nullptr, w);
    X = w;
  }
  run_sequential(fs, X, labels_host, ncomp, L, opt, status, res);
}

long long* cv_prediction_counts_device(const int* d_pred, int G, int L, int n, const int* d_labels,
                                      const int* d_exclude) {
  Context& ctx = Context::get();
  long long* d_counts = ctx.arena.alloc_n<long long>(2 * (size_t)G * L);
  pred_counts_kernel<<<G * L, 256, 0, ctx.stream>>>(d_pred, L, n, d_labels, d_exclude, d_counts); ::fpls::note_launch();
  FPLS_CHECK_LAUNCH();
  return d_counts;
}

void cv_prediction_counts(const int* d_pred, int G, int L, int n, const int* d_labels,
                          const int* d_exclude, std::vector<long long>& counts) {
  Context& ctx = Context::get();
  long long* d_counts = cv_prediction_counts_device(d_pred, G, L, n, d_labels, d_exclude);
  counts.assign(2 * (size_t)G * L, 0);
  d2h(counts.data(), d_counts, counts.size() * sizeof(long long));
  ctx.sync();
}

}  // namespace fpls
