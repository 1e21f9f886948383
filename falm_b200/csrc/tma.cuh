// TMA plane streaming for the 2.5D stencil kernels (sm_100a).
//
// A field is described to the Tensor Memory Accelerator as a 4D tensor
// (x = sx, y = sy, z = sz, c = components) in the reference's SoA layout.  A
// kernel marches a tile column along z: one elected thread issues
// cp.async.bulk.tensor loads of (tile + halo) x/y boxes of the next planes
// into a ring of shared-memory slots, each slot guarded by an mbarrier that
// completes on the transferred byte count.  No multicast is used: every CTA
// loads its own boxes from this GPU's memory.
//
// Every wait is bounded (about one second of clock64 time): a wait that gives
// up records an error in the context's device error word and returns false,
// and the kernel drains its own copies (again bounded) before it returns.
// Warp 0 of a block polls the barriers; a block barrier then publishes the
// landed data to the other warps.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace fb {

constexpr unsigned kWaitLimit = 1u << 28;   // polls of try_wait (the clock64 bound of ~1 s normally ends a wait first)
constexpr unsigned kSuspendNs = 200000;     // suspend-time hint of one try_wait (ns): the thread sleeps until the phase
                                            // completes or this much time has passed

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}

constexpr long long kWaitCycles = 2000000000LL;   // clock64 bound of one wait: about one second

// bounded wait: try_wait suspends the thread in hardware until the phase
// completes or the suspend-time hint passes; poll it, checking clock64 every
// 4 polls, and give up after `cycles` clock64 cycles (or kWaitLimit polls):
// false (and *err set to FALM_ERR_TIMEOUT) then
__device__ __forceinline__ bool mbar_wait_cycles(uint64_t *bar, uint32_t parity, int *err, long long cycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    for (unsigned it = 1; it < kWaitLimit; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 3u) == 0 && clock64() - t0 > cycles) break;
    }
    if (err) atomicExch(err, FALM_ERR_TIMEOUT);
    return false;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
    return mbar_wait_cycles(bar, parity, err, kWaitCycles);
}

// origin of a box of width `box` (elements) inside an axis of `dim` elements:
// the wanted origin, moved back so the box does not run past the end when the
// axis is at least one box long, kept on a multiple of `align` elements
__device__ __forceinline__ int box_origin(int want, int box, int dim, int align) {
    if (dim < box) return want;
    int last = (dim - box) / align * align;
    return want < last ? want : last;
}

// 4D tiled load of box (bx, by, 1, bc) at coordinates (x, y, z, c) into smem
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int c, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_addr(dst)), "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Self-check of a load request: the x coordinate must start on a 16-byte
// boundary, the destination on a 128-byte one, and x, y, z must lie inside the
// tensor (x, y may run past the upper end: those elements are zero-filled).
// A kernel sends a slot's loads only when every request passes; otherwise it
// records 200 + site in the error word and completes the slot's barrier with
// a plain arrive, so no wait is left pending and nothing faults.
__device__ __forceinline__ bool tma_ok(const void *dst, int x, int y, int z, int esize, int xdim, int ydim, int zdim) {
    return ((x * esize) & 15) == 0 && (smem_addr(dst) & 127) == 0 && x >= 0 && x < xdim && y >= 0 && y < ydim && z >= 0 &&
           z < zdim;
}

__device__ __forceinline__ void tma_reject(uint64_t *bar, int *err, int site) {
    if (err) atomicExch(err, 200 + site);
    mbar_arrive(bar);
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

}  // namespace fb
