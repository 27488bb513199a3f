// Shared sm_100a building blocks of the tensor-core kernels: mbarriers with
// bounded waits, 2-D TMA tile loads (no cluster multicast), the K-major
// SWIZZLE_128B shared-memory descriptor of tcgen05.mma, tcgen05.commit and
// tcgen05.ld, and the driver's tensor-map encoder.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "context.cuh"

namespace fpls {
namespace tc {

// Clock budget of every mbarrier wait (~4 s at 2 GHz); a wait that runs out
// raises the kernel's error flag and returns instead of spinning on.
constexpr long long kWaitBudget = 1ll << 33;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// Bounded parity wait: returns false (and raises *err) when the budget runs out
// or, with stop_on_error, when another thread already raised the flag.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err,
                                          bool stop_on_error = true) {
  const long long t0 = clock64();
  for (uint32_t spin = 0;; ++spin) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (stop_on_error && (spin & 63) == 63 && *(volatile int*)err) return false;
    if (clock64() - t0 > kWaitBudget) {
      atomicExch(err, 1);
      return false;
    }
  }
}

// 2-D tiled TMA load into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint32_t dst, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// UMMA shared-memory descriptor: K-major, SWIZZLE_128B (128-byte rows), 8-row
// core groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1) << 16;              // leading byte offset (unused for SW128 K-major)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;      // stride byte offset
  d |= static_cast<uint64_t>(1) << 46;              // descriptor version for sm_100
  d |= static_cast<uint64_t>(2) << 61;              // SWIZZLE_128B
  return d;
}

// Arrives on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 16 consecutive 32-bit TMEM columns of this warp's lane quarter (one value per
// lane and column); the caller issues tcgen05.wait::ld before reading r.
__device__ __forceinline__ void tmem_ld16_raw(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Programmatic dependent launch: wait until the grid this one depends on has
// completed and its writes are visible (a no-op for a grid launched without
// programmatic stream serialisation), and allow the next grid on the stream to
// be scheduled.  Every kernel chained this way fits on the GPU in one wave, so
// a dependent waiting early never holds an SM its predecessor still needs.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Launch attribute for programmatic stream serialisation (FASTPLS_PDL=0 turns
// it off).
inline bool pdl_enabled() {
  const char* e = std::getenv("FASTPLS_PDL");
  return !(e && e[0] == '0');
}

// cuTensorMapEncodeTiled through the runtime's driver entry point.
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    FPLS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      throw Error(kErrCuda, "cuTensorMapEncodeTiled is unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace tc
}  // namespace fpls
