// tma.cuh — Tensor Memory Accelerator tile loads (cp.async.bulk.tensor with a tensor map,
// completing on an mbarrier), per-thread cp.async copies, mbarrier helpers and programmatic
// dependent launch, inline PTX for sm_100a.  No multicast form is used anywhere.  Every wait
// is bounded: after kMaxPolls unsuccessful polls it gives up and reports false, so a kernel
// can flag PIC_ST_TIMEOUT and leave.
#pragma once
#include <cstdint>

namespace tma {

constexpr uint32_t kMaxPolls = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Arrive on m (count 1) and add `bytes` to the transaction count the phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity) {
  for (uint32_t k = 0; k < kMaxPolls; ++k)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

// 2-D tensor-map tile load (cp.async.bulk.tensor, tile mode, this CTA only) of the box whose
// first element is at column x (a multiple of 16 bytes) and row y of the map's tensor,
// completing on mbarrier m.  Columns and rows outside the tensor read as zero.
__device__ __forceinline__ void tensor_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* m) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(m))
      : "memory");
}

// Per-thread asynchronous global -> shared copy of 4 or 8 bytes (cp.async): nothing is held
// in registers while the copy is in flight.  valid = false reads no global memory and writes
// zeros (src must still be a valid address: callers pass the array base).
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
// Wait for every cp.async this thread issued (a block barrier must follow before other
// threads read the data).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Programmatic dependent launch.  A kernel launched with programmatic stream serialisation may
// start while its predecessor in the stream is still running: it must call pdl_wait() before
// reading anything the predecessor writes.  pdl_trigger() lets the successor launch once every
// CTA of this kernel has called it (or exited).  Both are no-ops for ordinary launches.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace tma
