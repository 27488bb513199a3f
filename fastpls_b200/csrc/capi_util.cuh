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

}  // namespace capi
}  // namespace fpls
