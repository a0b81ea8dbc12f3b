// tma.cuh -- the Tensor Memory Accelerator on sm_100a: 2D tiled bulk copies
// from global into shared memory, completed on an mbarrier (PTX ISA:
// cp.async.bulk.tensor, mbarrier.*), plus the host side that encodes tensor maps
// through the driver entry point (no link against libcuda).
//
// Only loads into this CTA's own shared memory are issued: no multicast, no
// cluster destination other than the CTA itself.  Every wait is bounded.
#pragma once

#include <cuda.h>

#include "device.cuh"

namespace qed2d {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the async proxy (the TMA unit)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory"); }

// order this thread's earlier accesses and those it has synchronised with
// (generic proxy) before its later async-proxy operations: global (other
// blocks' stores seen through a grid barrier, before the TMA copies read them)
// and shared (a stage's reads, before the copies that overwrite it)
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" : : : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" : : : "memory");
}

// one arrival that also announces `bytes` of transactions for the current phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" : : "r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of an mbarrier: false after `limit` tries
// (each try_wait itself suspends the thread for a while), raising
// QED2D_ERR_TIMEOUT in *err.  It does not give up when another block has
// failed: the copies it waits for are this block's own and complete in
// microseconds, and a block leaves only with none of them in flight.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err,
                                          unsigned long long limit = 1ULL << 22) {
    unsigned long long tries = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++tries > limit) {
            atomicExch(err, 2 /* QED2D_ERR_TIMEOUT */);
            return false;
        }
    }
    return true;
}

// 2D tile load: the box of `map` at element coordinates (x, y) into dst (this
// CTA's shared memory, 128-byte aligned), completing `bytes` on bar.  The
// caller keeps x * element size a multiple of 16 bytes and the box inside the
// tensor.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :
        : "r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// host: a 2D float32 tensor map of dims (nx, ny) elements, row pitch `pitch`
// bytes, box (bx, by); no swizzle, no interleave, zero fill (never used: every
// box the kernels load lies inside the tensor)
int encode_map_2d(CUtensorMap* map, const void* base, unsigned long long nx, unsigned long long ny,
                  unsigned long long pitch, unsigned bx, unsigned by);

}  // namespace qed2d
