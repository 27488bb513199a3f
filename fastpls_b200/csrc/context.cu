#include "context.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace fpls {

Arena::~Arena() {}

void* Arena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  if (bytes == 0) bytes = 256;
  for (auto& b : blocks_) {
    if (b.size - b.used >= bytes) {
      void* p = b.base + b.used;
      b.used += bytes;
      return p;
    }
  }
  size_t want = std::max<size_t>(bytes, size_t(64) << 20);
  char* base = nullptr;
  FPLS_CUDA(cudaMalloc(&base, want));
  blocks_.push_back({base, want, bytes});
  return base;
}

size_t Arena::capacity() const {
  size_t c = 0;
  for (auto& b : blocks_) c += b.size;
  return c;
}

void Arena::reset() {
  size_t used = 0;
  for (auto& b : blocks_) used += b.used;
  high_water_ = std::max(high_water_, used);
  if (blocks_.size() > 1) {
    size_t total = capacity();
    for (auto& b : blocks_) cudaFree(b.base);
    blocks_.clear();
    char* base = nullptr;
    FPLS_CUDA(cudaMalloc(&base, total));
    blocks_.push_back({base, total, 0});
  } else {
    for (auto& b : blocks_) b.used = 0;
  }
}

void Arena::release() {
  for (auto& b : blocks_) cudaFree(b.base);
  blocks_.clear();
}

Context& Context::get() {
  static Context ctx;
  if (ctx.device < 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n < 1) {
      throw Error(kErrNoDevice, "fastpls_b200: no CUDA device is available");
    }
    int dev = 0;
    // One process per GPU: FASTPLS_DEVICE selects the ordinal (default: current device).
    if (const char* e = std::getenv("FASTPLS_DEVICE")) {
      char* endp = nullptr;
      const long v = std::strtol(e, &endp, 10);
      if (endp != e && v >= 0 && v < n) FPLS_CUDA(cudaSetDevice(static_cast<int>(v)));
    }
    FPLS_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    FPLS_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) {
      throw Error(kErrNoDevice, std::string("fastpls_b200 is built for sm_100a (B200); device is ") +
                                    prop.name);
    }
    ctx.sm_count = prop.multiProcessorCount;
    FPLS_CUDA(cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
    FPLS_CUDA(cudaStreamCreateWithFlags(&ctx.side, cudaStreamNonBlocking));
    FPLS_CUDA(cudaEventCreateWithFlags(&ctx.side_done, cudaEventDisableTiming));
    FPLS_CUDA(cudaEventCreateWithFlags(&ctx.planes_ready, cudaEventDisableTiming));
    FPLS_CUDA(cudaStreamCreateWithFlags(&ctx.copy, cudaStreamNonBlocking));
    FPLS_CUDA(cudaMalloc(&ctx.d_status, 64 * sizeof(int)));
    FPLS_CUDA(cudaMemset(ctx.d_status, 0, 64 * sizeof(int)));
    ctx.device = dev;
  }
  return ctx;
}

namespace {
long long g_launches = 0;
}

void note_launch() { ++g_launches; }
long long launch_count() { return g_launches; }

void Context::begin_call() {
  arena.reset();
  if (!call_start) {
    FPLS_CUDA(cudaEventCreate(&call_start));
    FPLS_CUDA(cudaEventCreate(&call_stop));
  }
  FPLS_CUDA(cudaEventRecord(call_start, stream));
  call_started = true;
  FPLS_CUDA(cudaMemsetAsync(d_status, 0, 64 * sizeof(int), stream));
}

void Context::end_call() {
  if (!call_started) return;
  call_started = false;
  FPLS_CUDA(cudaEventRecord(call_stop, stream));
  FPLS_CUDA(cudaEventSynchronize(call_stop));
  float ms = 0.f;
  FPLS_CUDA(cudaEventElapsedTime(&ms, call_start, call_stop));
  last_call_ms = ms;
}

int Context::read_status() {
  int s = 0;
  FPLS_CUDA(cudaMemcpyAsync(&s, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
  FPLS_CUDA(cudaStreamSynchronize(stream));
  return s;
}

void Context::sync() { FPLS_CUDA(cudaStreamSynchronize(stream)); }

cudaEvent_t Context::copy_event(int i) {
  while (static_cast<int>(copy_events.size()) <= i) {
    cudaEvent_t ev;
    FPLS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    copy_events.push_back(ev);
  }
  return copy_events[i];
}

void Context::release() {
  if (device < 0) return;
  cudaStreamSynchronize(side);
  if (copy) cudaStreamSynchronize(copy);
  cudaStreamSynchronize(stream);
  arena.release();
  for (auto& b : splitk) cudaFree(b.ptr);
  splitk.clear();
  if (staging) cudaFreeHost(staging);
  staging = nullptr;
  staging_cap = 0;
}

char* Context::host_staging(size_t bytes) {
  if (bytes <= staging_cap) return staging;
  // grow: earlier copies into the old buffer must have landed
  FPLS_CUDA(cudaStreamSynchronize(stream));
  if (staging) FPLS_CUDA(cudaFreeHost(staging));
  staging = nullptr;
  staging_cap = std::max(bytes, std::max<size_t>(2 * staging_cap, 1 << 16));
  FPLS_CUDA(cudaMallocHost(&staging, staging_cap));
  return staging;
}

double* Context::splitk_workspace(cudaStream_t st, size_t elems) {
  for (auto& b : splitk) {
    if (b.stream != st) continue;
    if (b.cap >= elems) return b.ptr;
    // grow: earlier products on this stream may still read the old buffer
    FPLS_CUDA(cudaStreamSynchronize(st));
    FPLS_CUDA(cudaFree(b.ptr));
    b.cap = std::max(elems, 2 * b.cap);
    FPLS_CUDA(cudaMalloc(&b.ptr, b.cap * sizeof(double)));
    return b.ptr;
  }
  StreamBuffer b{st, nullptr, std::max<size_t>(elems, 1 << 20)};
  FPLS_CUDA(cudaMalloc(&b.ptr, b.cap * sizeof(double)));
  splitk.push_back(b);
  return b.ptr;
}

// The caller's side of a copy may be host or device memory (unified
// addressing tells them apart): a caller that already holds its matrices in
// HBM passes device pointers and the copy stays on the device.
void h2d(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  FPLS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, Context::get().stream));
}
void d2h(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  FPLS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, Context::get().stream));
}
void d2d(void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  FPLS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, Context::get().stream));
}
void dzero(void* dst, size_t bytes) {
  if (bytes == 0) return;
  FPLS_CUDA(cudaMemsetAsync(dst, 0, bytes, Context::get().stream));
}

void shard_sum(double* buf, size_t count) {
  Context& ctx = Context::get();
  if (!ctx.shards || count == 0) return;
  const int rc = ctx.shards->fn(buf, static_cast<long long>(count), static_cast<void*>(ctx.stream),
                                ctx.shards->user);
  if (rc != 0)
    throw Error(kErrCuda, "row-sharded fit: the all-reduce callback returned " + std::to_string(rc));
}

long long shard_rows(long long n_local) {
  const Context& ctx = Context::get();
  return ctx.shards ? ctx.shards->n_total : n_local;
}

bool sharded() { return Context::get().shards != nullptr; }

RowShardScope::RowShardScope(Context& c, int (*fn)(double*, long long, void*, void*), void* user,
                             long long n_local)
    : ctx(c) {
  FPLS_REQUIRE(fn != nullptr, "row-sharded fit: the all-reduce callback is null");
  rs.fn = fn;
  rs.user = user;
  rs.n_total = n_local;
  ctx.shards = &rs;
  try {
    double nd = static_cast<double>(n_local);
    double* d = ctx.arena.alloc_n<double>(1);
    h2d(d, &nd, sizeof(double));
    shard_sum(d, 1);
    d2h(&nd, d, sizeof(double));
    ctx.sync();
    rs.n_total = static_cast<long long>(nd + 0.5);
    FPLS_REQUIRE(rs.n_total >= n_local, "row-sharded fit: the all-reduce did not sum the row counts");
  } catch (...) {
    ctx.shards = nullptr;   // the destructor does not run when the constructor throws
    throw;
  }
}

}  // namespace fpls

namespace fpls {

PhaseTimer::PhaseTimer(const char* title) : title_(title) {
  const char* e = std::getenv("FASTPLS_TRACE");
  on_ = e && e[0] == '1';
  mark("start");
}

PhaseTimer::~PhaseTimer() {
  if (on_ && !reported_) {
    try {
      report();
    } catch (...) {
    }
  }
  for (auto& m : marks_) cudaEventDestroy(m.second);
}

void PhaseTimer::mark(const char* name) {
  if (!on_) return;
  cudaEvent_t ev;
  FPLS_CUDA(cudaEventCreate(&ev));
  FPLS_CUDA(cudaEventRecord(ev, Context::get().stream));
  marks_.emplace_back(name, ev);
}

void PhaseTimer::report() {
  if (!on_ || reported_) return;
  reported_ = true;
  FPLS_CUDA(cudaStreamSynchronize(Context::get().stream));
  std::vector<std::pair<std::string, double>> acc;
  double total = 0.0;
  for (size_t k = 1; k < marks_.size(); ++k) {
    float ms = 0.f;
    FPLS_CUDA(cudaEventElapsedTime(&ms, marks_[k - 1].second, marks_[k].second));
    total += ms;
    bool found = false;
    for (auto& a : acc)
      if (a.first == marks_[k].first) { a.second += ms; found = true; }
    if (!found) acc.emplace_back(marks_[k].first, ms);
  }
  std::fprintf(stderr, "[fastpls trace] %s: %.3f ms\n", title_, total);
  for (auto& a : acc) std::fprintf(stderr, "  %-14s %8.3f ms\n", a.first.c_str(), a.second);
}

}  // namespace fpls

namespace fpls {

int Context::prof_begin(const char* cls, cudaStream_t st) {
  if (!profile) return -1;
  int slot = -1;
  for (size_t i = 0; i < prof_classes.size(); ++i)
    if (prof_classes[i].name == cls) slot = static_cast<int>(i);
  if (slot < 0) {
    prof_classes.push_back(ProfClass{});
    prof_classes.back().name = cls;
    slot = static_cast<int>(prof_classes.size()) - 1;
  }
  cudaEvent_t ev;
  FPLS_CUDA(cudaEventCreate(&ev));
  FPLS_CUDA(cudaEventRecord(ev, st));
  prof_classes[slot].events.push_back(ev);
  return slot;
}

void Context::prof_end(int slot, cudaStream_t st, double bytes, double flops) {
  if (slot < 0 || !profile) return;
  cudaEvent_t ev;
  FPLS_CUDA(cudaEventCreate(&ev));
  FPLS_CUDA(cudaEventRecord(ev, st));
  ProfClass& c = prof_classes[slot];
  c.events.push_back(ev);
  c.bytes += bytes;
  c.flops += flops;
}

}  // namespace fpls
