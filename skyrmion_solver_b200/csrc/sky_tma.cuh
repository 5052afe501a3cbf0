// Tensor-memory-accelerator (TMA) staging of haloed x-planes.
//
// A marching tile needs, per x-plane and per source array, the box
//   z = z0 - 4 .. z0 + 35,  y = y0 - 2 .. y0 + BY + 1,  x = q,  components 0 .. C-1
// of a lattice array in the reference layout (index a*N + x*Y*Z + y*Z + z).
// Seen as a rank-4 tensor with dimensions (Z, Y, X, C) (innermost first) that box
// is one cp.async.bulk.tensor tile copy: one thread issues it, the copy engine
// writes the box into shared memory as [c][y][z] rows of 40 values (the marching
// kernels' wide-row plane layout) and fills every point outside the lattice with
// zeros, and an mbarrier counts the bytes that have landed.  The per-thread
// address arithmetic and copy instructions of cp.async staging disappear.
//
// Alignment (checked when the maps are encoded): the array base is 16-byte
// aligned (cudaMalloc), the row pitch Z * sizeof(T) and the component pitch
// N * sizeof(T) are multiples of 16 bytes, the box's inner extent (40 values) is
// a multiple of 16 bytes, and the innermost start coordinate z0 - 4 (z0 a
// multiple of 32) is a multiple of 4 values.  Plain loads only, each of this
// GPU's own memory into the issuing CTA's own shared memory.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace sky {

// Tensor maps of one array per role; one per array the stage kernels stage.
struct alignas(64) TmaMap {
    CUtensorMap m;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the copy engine
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Arrive (one of the barrier's expected arrivals) and add `bytes` to the
// transaction count the current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete, giving up after
// kMbarSpins unsuccessful polls (each poll itself may suspend the thread for a
// short hardware-chosen time); returns false when it gave up.
constexpr int kMbarSpins = 1 << 21;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kMbarSpins; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Order this thread's earlier generic-proxy accesses of shared memory before
// its later async-proxy (copy engine) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the previous kernel of the stream finishes.  Before it
// reads anything that kernel wrote it waits for its completion (and memory flush);
// without the launch attribute the wait returns at once.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// This block has done the work the next kernel may overlap: once every block of the
// grid has signalled (or exited), the dependent kernel may be scheduled.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void prefetch_tmap(const TmaMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(&map->m) : "memory");
}

// One tile copy of the box at (z, y, x, c) of `map` into shared memory at dst,
// completing on `bar`; the destination is the issuing CTA's own shared memory.
__device__ __forceinline__ void tma_load_plane(void* dst, const TmaMap* map, int z, int y, int x, int c,
                                               uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(&map->m), "r"(z), "r"(y), "r"(x), "r"(c), "r"(smem_addr(bar))
        : "memory");
}

// Host: encode the plane-box map of a C-component lattice array of element size
// `esize` (4 or 8) with dimensions (X, Y, Z): box (hz, hy, 1, C).  Returns 0 on
// success, else a sky_status (invalid argument when an alignment rule fails).
int encode_plane_map(TmaMap* out, const void* base, int esize, int X, int Y, int Z, int C, int hz, int hy);

}  // namespace sky
