// fpls_bf16x3_gemm_noalloc: the tensor-core split GEMM for callers that cannot
// allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc at the point where they
// need a product: code running while another framework owns the device memory
// budget (a fixed pool handed out by an embedding runtime), code inside a
// stream callback or a region being recorded by someone else, or an
// allocation-free real-time loop.  They already hold device buffers for their
// inputs and outputs; this entry point needs nothing else.  Every temporary of
// the kernel (the BF16 hi/lo copies of both operands, the stream-K work tables
// and the FP32 partials) lives in one file-scope device array of fixed size,
// which every GPU that loads the library keeps until the process exits.
#include "../../include/fastpls_b200.h"

#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "xop_split.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(16) << 20;  // 16 MiB per device
constexpr size_t kErrSlotBytes = 256;                                    // error flag at the front

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct DeviceSetup {
  bool ready = false;
  void* ptr = nullptr;  // device address of g_noalloc_scratch on this device
  int sms = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;  // first calls from several host threads set up once

// Once per device, on the caller's current device (the call never changes it):
// resolve the array's device address there.
DeviceSetup& setup_device(int dev) {
  if (dev < 0 || dev >= kMaxDevices) throw fpls::Error(fpls::kErrArgument, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (!s.ready) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw fpls::Error(fpls::kErrCuda, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    int sms = 0;
    FPLS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    s.ptr = p;
    s.sms = sms;
    s.ready = true;
  }
  return s;
}

// A, B and C must be memory of the current device (device or managed memory):
// a host pointer, or another GPU's buffer, would fault inside the kernels, so
// it is refused before anything is launched.
void require_device_pointer(const void* ptr, int dev, const char* name) {
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, ptr);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // the failed query's error is not a device fault: clear it
    throw fpls::Error(fpls::kErrArgument, std::string("bf16x3_gemm_noalloc: ") + name + " is not a device pointer");
  }
  const bool on_device = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
  if (!on_device || (a.type == cudaMemoryTypeDevice && a.device != dev))
    throw fpls::Error(fpls::kErrArgument, std::string("bf16x3_gemm_noalloc: ") + name +
                                              " must be device memory of the current device");
}

void put_err(char* err, size_t errlen, const char* msg) {
  if (!err || errlen == 0) return;
  std::strncpy(err, msg, errlen - 1);
  err[errlen - 1] = '\0';
}

}  // namespace

extern "C" int fpls_bf16x3_gemm_noalloc(const double* A, int M, int K, const double* B, int N,
                                        double* C, char* err, size_t errlen) {
  if (err && errlen) err[0] = '\0';
  try {
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C)
      throw fpls::Error(fpls::kErrArgument, "bf16x3_gemm_noalloc: dimensions must be positive and pointers set");
    int dev = 0;
    FPLS_CUDA(cudaGetDevice(&dev));
    require_device_pointer(A, dev, "A");
    require_device_pointer(B, dev, "B");
    require_device_pointer(C, dev, "C");
    DeviceSetup& s = setup_device(dev);
    const size_t need = fpls::split_gemm_scratch_need(M, N, K, s.sms);
    if (need + kErrSlotBytes > kNoAllocScratchBytes) {
      throw fpls::Error(fpls::kErrArgument,
                        "bf16x3_gemm_noalloc: shape needs " + std::to_string(need) +
                            " bytes of scratch, more than the fixed 16 MiB");
    }
    cudaStream_t st = 0;  // the legacy default stream of the calling thread
    int* flag = static_cast<int*>(s.ptr);
    FPLS_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
    char* work = static_cast<char*>(s.ptr) + kErrSlotBytes;
    fpls::split_gemm_in_scratch(A, B, M, N, K, C, work, kNoAllocScratchBytes - kErrSlotBytes, flag,
                                st, s.sms);
    int h = 0;
    FPLS_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    FPLS_CUDA(cudaStreamSynchronize(st));
    if (h) throw fpls::Error(fpls::kErrCuda, "tensor-core pipeline wait timed out");
    return FPLS_OK;
  } catch (const fpls::Error& e) {
    put_err(err, errlen, e.what());
    return e.code;
  } catch (const std::exception& e) {
    put_err(err, errlen, e.what());
    return FPLS_ERR_INTERNAL;
  }
}
