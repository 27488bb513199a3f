// Shared helpers of the extern "C" entry points: error capture (C++ exceptions
// become a status code plus a message in the caller's buffer) and host<->device
// staging through the context arena.
#pragma once

#include <cstring>
#include <exception>

#include "common.cuh"
#include "context.cuh"

namespace fpls {
namespace capi {

inline void set_err(char* err, size_t errlen, const char* msg) {
  if (!err || errlen == 0) return;
  std::strncpy(err, msg, errlen - 1);
  err[errlen - 1] = '\0';
}

template <typename Fn>
int guarded(char* err, size_t errlen, Fn&& fn) {
  if (err && errlen) err[0] = '\0';
  try {
    fn();
    Context::get().end_call();
    return FPLS_OK;
  } catch (const Error& e) {
    set_err(err, errlen, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return FPLS_ERR_INTERNAL;
  } catch (...) {
    set_err(err, errlen, "fastpls_b200: unknown internal error");
    return FPLS_ERR_INTERNAL;
  }
}

template <typename T>
T* upload(const T* host, size_t n) {
  T* d = Context::get().arena.alloc_n<T>(n ? n : 1);
  if (n) h2d(d, host, n * sizeof(T));
  return d;
}

template <typename T>
void download(T* host, const T* dev, size_t n) {
  if (host && n) d2h(host, dev, n * sizeof(T));
}

// A copy of a caller's matrix (host or device) on the copy stream, queued
// behind the work the main stream has enqueued so far (so that an earlier
// upload keeps the whole link), for a later step of the same call; wait()
// makes the main stream wait for it.  A call that leaves early (an error)
// waits for the copy on the host, so that no copy still writes into arena
// memory the next call reuses.  Uses copy events 0 and 1 of the context.
struct SideUpload {
  void* dst = nullptr;
  bool pending = false;
  SideUpload(const void* src, size_t bytes) {
    if (!bytes) return;
    Context& ctx = Context::get();
    dst = ctx.arena.alloc_n<char>(bytes);
    FPLS_CUDA(cudaEventRecord(ctx.copy_event(0), ctx.stream));
    FPLS_CUDA(cudaStreamWaitEvent(ctx.copy, ctx.copy_event(0), 0));
    FPLS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx.copy));
    FPLS_CUDA(cudaEventRecord(ctx.copy_event(1), ctx.copy));
    pending = true;
  }
  SideUpload(const SideUpload&) = delete;
  SideUpload& operator=(const SideUpload&) = delete;
  void wait() {
    if (!pending) return;
    Context& ctx = Context::get();
    FPLS_CUDA(cudaStreamWaitEvent(ctx.stream, ctx.copy_event(1), 0));
    pending = false;
  }
  ~SideUpload() {
    if (pending) cudaEventSynchronize(Context::get().copy_event(1));
  }
};

}  // namespace capi
}  // namespace fpls
