// Bulk copies between this GPU's global memory and a CTA's shared memory
// (cp.async.bulk, the non-tensor TMA path): global -> shared with completion
// counted on an mbarrier, shared -> global as a bulk group.  Every copy is
// issued by one thread of the CTA into (or out of) its own shared memory,
// with no multicast, and every source or destination in global memory is
// this GPU's own.  Addresses are 16-byte aligned and sizes multiples of 16.
#pragma once

namespace nc {
namespace {

#define NC_BULK_CHUNK 32768u   /* bytes per bulk copy instruction */

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One global -> shared (or shared -> global) region.
struct BulkJob {
    void* smem;         // this CTA's shared memory
    const void* global; // this GPU's global memory
    uint32_t bytes;     // a multiple of 16
};

// Load `count` regions into shared memory and wait for them.  The wait is
// bounded: past the limit the CTA raises TIMEOUT and the abort flag and
// returns false after a second bounded wait for its copies.
__device__ bool bulk_load(const DeviceCloth& d, const BulkJob* jobs, uint32_t count) {
    __shared__ __align__(8) unsigned long long s_bar;
    const uint32_t bar = smem_addr(&s_bar);
    uint32_t total = 0u;
    for (uint32_t j = 0; j < count; ++j) total += jobs[j].bytes;
    if (total == 0u) return true;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total) : "memory");
        for (uint32_t j = 0; j < count; ++j) {
            const char* src = static_cast<const char*>(jobs[j].global);
            char* dst = static_cast<char*>(jobs[j].smem);
            for (uint32_t at = 0; at < jobs[j].bytes; at += NC_BULK_CHUNK) {
                const uint32_t len = min(NC_BULK_CHUNK, jobs[j].bytes - at);
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_addr(dst + at)),
                    "l"(src + at), "r"(len), "r"(bar)
                    : "memory");
            }
        }
    }
    __syncthreads();
    // every thread waits for the copies (phase 0 of the barrier)
    const unsigned limit = d.spin_limit != 0u ? d.spin_limit : NC_BARRIER_SPIN_LIMIT;
    uint32_t done = 0u;
    for (unsigned spin = 0; spin <= 2u * limit && !done; ++spin) {
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done)
                     : "r"(bar)
                     : "memory");
        if (!done && spin == limit && threadIdx.x == 0) {
            atomicOr(d.failure, NUMI_CLOTH_FAILURE_TIMEOUT);
            atomicExch(d.abort_flag, 1u);
        }
    }
    const bool all = __syncthreads_and(done != 0u) != 0;
    // a completed barrier is invalidated so the next load may initialise it
    if (all && threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
    __syncthreads();
    return all;
}

// Store `count` regions of shared memory to global memory and wait until
// the writes are done.  Every thread of the CTA calls it after its last
// write to those regions (the proxy fence makes them visible to the copy).
__device__ void bulk_store(const BulkJob* jobs, uint32_t count) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t j = 0; j < count; ++j) {
            char* dst = static_cast<char*>(const_cast<void*>(jobs[j].global));
            const char* src = static_cast<const char*>(jobs[j].smem);
            for (uint32_t at = 0; at < jobs[j].bytes; at += NC_BULK_CHUNK) {
                const uint32_t len = min(NC_BULK_CHUNK, jobs[j].bytes - at);
                asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst + at),
                             "r"(smem_addr(src + at)), "r"(len)
                             : "memory");
            }
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
}

}  // namespace
}  // namespace nc
