// Process-wide device context: one stream, a scratch arena and a few device
// scalars.  Replaces the reference's thread_local CudaRSVDWorkspace
// (src/svd_cuda_rsvd.cpp:271-2092); like it, it is used from a single host
// thread and released by fpls_reset_workspace().
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

namespace fpls {

class Arena {
 public:
  ~Arena();
  // Returns 256-byte aligned device memory valid until reset().
  void* alloc(size_t bytes);
  template <typename T>
  T* alloc_n(size_t n) { return static_cast<T*>(alloc(n * sizeof(T))); }
  // Drops every allocation; consolidates the blocks into one of the total size.
  void reset();
  void release();
  size_t capacity() const;

 private:
  struct Block { char* base; size_t size; size_t used; };
  std::vector<Block> blocks_;
  size_t high_water_ = 0;
};

// Device-resident predictor matrices registered by the caller (kept across calls).
struct ResidentX {
  void* ptr = nullptr;
  int n = 0, p = 0;
  bool f32 = false;
};

struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;   // second stream for work that overlaps `stream` (joined by events)
  cudaEvent_t side_done = nullptr;
  cudaEvent_t planes_ready = nullptr;   // the operator of a CV grid's X is complete on `stream`
  cudaStream_t copy = nullptr;   // host-to-device copies that overlap `stream` (joined by copy_event(i))
  std::vector<cudaEvent_t> copy_events;
  cudaEvent_t copy_event(int i);   // i-th event of the copy stream (created on first use)
  Arena arena;
  int* d_status = nullptr;     // device-side failure flag (0 = ok)
  int sm_count = kSMCount;
  int precision = 0;           // session precision of single fits: 0 FP64, 1 BF16x3 (predictor GEMMs)
  // Timing of the last ABI call (events on `stream`, bracketing the whole call).
  cudaEvent_t call_start = nullptr, call_stop = nullptr;
  bool call_started = false;
  double last_call_ms = 0.0;
  // Optional profiling window: CUDA events around the launches of the main
  // kernels, grouped by kernel class, with each launch's algorithmic bytes and
  // flops (the figures a roofline divides by the measured time).
  bool profile = false;
  struct ProfClass {
    std::string name;
    std::vector<cudaEvent_t> events;      // start/stop pairs
    double bytes = 0.0, flops = 0.0;
  };
  std::vector<ProfClass> prof_classes;
  // Records the start event of one launch of `cls` on `st` (no-op unless
  // profiling); prof_end() records the stop event and adds bytes / flops.
  int prof_begin(const char* cls, cudaStream_t st);
  void prof_end(int slot, cudaStream_t st, double bytes, double flops);
  std::vector<ResidentX> resident;
  // Split-K partials of the FP64 products, one buffer per stream (grown on
  // demand, kept across calls): partial sums are added in K-range order
  // instead of by atomics, so FP64 results repeat bit for bit.
  struct StreamBuffer { cudaStream_t stream; double* ptr; size_t cap; };
  std::vector<StreamBuffer> splitk;
  double* splitk_workspace(cudaStream_t st, size_t elems);
  // Page-locked host staging for the small results of a call (grown on
  // demand, kept across calls): copies into it stay asynchronous, so a call
  // gathers its results with one synchronisation instead of one per copy.
  char* staging = nullptr;
  size_t staging_cap = 0;
  char* host_staging(size_t bytes);

  // Row-sharded fit in progress (null otherwise): the caller's all-reduce
  // and the row count over all ranks.
  struct RowShards {
    int (*fn)(double* buf, long long count, void* stream, void* user) = nullptr;
    void* user = nullptr;
    long long n_total = 0;
  };
  RowShards* shards = nullptr;

  static Context& get();       // initialises the device on first use
  void begin_call();           // resets the arena and the status flag, starts the call timer
  void end_call();             // stops the call timer (after the final synchronisation)
  int read_status();           // synchronises the stream and reads the flag
  void sync();
  void release();
};

// Opt-in phase timer (FASTPLS_TRACE=1): CUDA events on the context stream
// between named marks; the sums per name are printed to stderr by report().
// Makes the launches of a scope go to another stream of the context (every
// launch site uses ctx.stream), e.g. the side stream; restores the main one.
struct StreamSwap {
  Context& ctx;
  cudaStream_t saved;
  StreamSwap(Context& c, cudaStream_t s) : ctx(c), saved(c.stream) { c.stream = s; }
  ~StreamSwap() { ctx.stream = saved; }
  StreamSwap(const StreamSwap&) = delete;
  StreamSwap& operator=(const StreamSwap&) = delete;
};

class PhaseTimer {
 public:
  explicit PhaseTimer(const char* title);
  ~PhaseTimer();
  void mark(const char* name);
  void report();
  bool enabled() const { return on_; }

 private:
  const char* title_;
  bool on_ = false;
  bool reported_ = false;
  std::vector<std::pair<const char*, cudaEvent_t>> marks_;
};

// Row-sharded fits: each rank holds a block of the rows of X and Y, and every
// sum over rows (column sums, X^T Y, X^T t, t^T t, Y^T t, T^T T, residual sums)
// is completed by the caller's all-reduce.  shard_sum() sums a device buffer
// over the ranks in place, ordered on the context stream; it does nothing when
// no sharded fit is active.  Every rank makes the same calls in the same order.
void shard_sum(double* buf, size_t count);
// Rows over all ranks (the local count when not sharded).
long long shard_rows(long long n_local);
bool sharded();
struct RowShardScope {
  Context::RowShards rs;
  Context& ctx;
  // Sets the callback and sums the local row count over the ranks (the first
  // all-reduce of every sharded fit).
  RowShardScope(Context& c, int (*fn)(double*, long long, void*, void*), void* user, long long n_local);
  ~RowShardScope() { ctx.shards = nullptr; }
  RowShardScope(const RowShardScope&) = delete;
  RowShardScope& operator=(const RowShardScope&) = delete;
};

// Host <-> device copies on the context stream (synchronous w.r.t. the caller
// once sync() is called).
void h2d(void* dst, const void* src, size_t bytes);
void d2h(void* dst, const void* src, size_t bytes);
void d2d(void* dst, const void* src, size_t bytes);
void dzero(void* dst, size_t bytes);

}  // namespace fpls
