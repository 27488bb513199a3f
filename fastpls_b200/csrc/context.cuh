// Process-wide device context: one stream, a scratch arena and a few device
// scalars.  Replaces the reference's thread_local CudaRSVDWorkspace
// (src/svd_cuda_rsvd.cpp:271-2092); like it, it is used from a single host
// thread and released by fpls_reset_workspace().
#pragma once

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

struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  Arena arena;
  int* d_status = nullptr;     // device-side failure flag (0 = ok)
  int sm_count = kSMCount;

  static Context& get();       // initialises the device on first use
  void begin_call();           // resets the arena and the status flag
  int read_status();           // synchronises the stream and reads the flag
  void sync();
  void release();
};

// Host <-> device copies on the context stream (synchronous w.r.t. the caller
// once sync() is called).
void h2d(void* dst, const void* src, size_t bytes);
void d2h(void* dst, const void* src, size_t bytes);
void d2d(void* dst, const void* src, size_t bytes);
void dzero(void* dst, size_t bytes);

}  // namespace fpls
