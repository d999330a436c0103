// dev_util.cuh -- sm_100a PTX helpers: mbarriers, 2-D TMA loads, bounded
// waits, and the status word kernels use to report a failure instead of
// hanging.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpc {

// Status bits a kernel can raise (OR-ed into the context's status word).
enum : unsigned {
  ST_WAIT_TIMEOUT = 1u,   // an mbarrier / flag wait ran past its limit
  ST_NONFINITE = 2u,      // the state norm became NaN/Inf/0
  ST_BAD_LAUNCH = 4u,     // a kernel saw an inconsistent launch shape
};

// Upper bound on a TMA ring (mbarrier) wait, in nanoseconds of %globaltimer,
// and the default bound on a grid-barrier wait (the persistent kernels take
// theirs from the launch arguments: a per-context setting).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint: a thread whose phase is not complete
// sleeps (instead of polling) until it completes or about hint_ns pass.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity,
                                                    uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Waits for phase `parity` of `bar` to complete, for at most kWaitLimitNs.
// Returns false (and raises ST_WAIT_TIMEOUT in *status) if the limit passed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 255u && globaltimer_ns() - t0 > kWaitLimitNs) {
      atomicOr(status, ST_WAIT_TIMEOUT);
      return false;
    }
  }
}

// 2-D tiled TMA load global -> shared, completing on `bar` (tx bytes).
// The x coordinate (innermost, in elements) must be a multiple of 2 for
// 8-byte elements: callers pass multiples of the 256-column strip width.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const void* tmap, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// 3-D tiled TMA load global -> shared, completing on `bar` (tx bytes); the
// innermost coordinate x follows the same 16-byte rule.
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const void* tmap, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Same load with an L2 cache-policy hint (see make_evict_first_policy).
__device__ __forceinline__ void tma_load_2d_hint(void* smem_dst, const void* tmap, uint64_t* bar,
                                                 int x, int y, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

// 1-D bulk copy global -> shared completing on `bar`.  Both addresses must
// be 16-byte aligned and `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// An L2 policy that marks lines to be kept over normal and evict-first ones:
// for the part of the dipole blocks that stays in L2 from one pass to the next.
__device__ __forceinline__ uint64_t make_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// An L2 policy that marks lines for early eviction: for data streamed once
// per pass (the dipole blocks), so that the small, reused vectors stay.
__device__ __forceinline__ uint64_t make_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ void prefetch_tmap(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// Programmatic dependent launch: pdl_trigger lets the next kernel on the
// stream be scheduled now; pdl_wait blocks until every earlier kernel on the
// stream has completed and its writes are visible.  Everything a kernel reads
// or writes that an earlier kernel touches must come after pdl_wait.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Bulk (TMA engine) store shared -> global of `bytes` (16-byte aligned
// addresses, a multiple of 16 bytes), in this thread's bulk group.  The
// threads that wrote the shared data first order their writes for the async
// proxy (fence_proxy_async_smem) and meet the issuing thread at a barrier.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(ssrc)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// until at most N of this thread's bulk groups still read shared memory
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// until at most N of this thread's bulk groups are incomplete
template <int N>
__device__ __forceinline__ void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// Grid-barrier arrival and wait for thread 0 of a CTA: the e-th barrier of a
// launch waits until the monotonic 64-bit counter (cleared before the launch)
// reaches target = e x gridDim.x.  The acquire-release add publishes this
// CTA's writes (ordered before it by the CTA's own barrier) and, for the last
// arrival, already sees every other CTA's; the others poll with acquire
// loads.  Returns false (and raises ST_WAIT_TIMEOUT) if the wait passed
// limit_ns.
__device__ __forceinline__ bool grid_arrive_wait(unsigned long long* ctr, unsigned long long target,
                                                 unsigned* status,
                                                 unsigned long long limit_ns = kWaitLimitNs) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;"
               : "=l"(old)
               : "l"(ctr), "l"(1ull)
               : "memory");
  if (old + 1 >= target) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (unsigned it = 0;; ++it) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ctr) : "memory");
    if (v >= target) return true;
    if ((it & 1023u) == 1023u && globaltimer_ns() - t0 > limit_ns) {
      atomicOr(status, ST_WAIT_TIMEOUT);
      return false;
    }
  }
}

// The grid-barrier settings of one persistent launch: the wait limit and an
// extra arrival count added to every target (0; 1 only when a test injects a
// barrier that cannot complete, so that the bounded wait runs out).
struct BarrierCfg {
  unsigned long long wait_ns;
  unsigned long long skew;
};

// Named barrier among `nthreads` threads (ids 1..15; 0 is __syncthreads).
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

}  // namespace mpc
