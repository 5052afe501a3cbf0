// Marching stencil kernels ("2.5-D" x-march).
//
// A thread block owns a BY x 32 (y, z) tile of one lattice and walks along x
// over a chunk [xa, xe).  The haloed input planes (BY+4) x 36 of all C
// components pass through a ring of five shared-memory slots (planes x-2 ..
// x+2 of the site being finished); the next plane is copied from global memory
// with cp.async into a staging area while the current one is computed, so the
// global-load latency overlaps the stencil and point arithmetic.
//
// Per thread and component two register queues hold, for planes x-2 .. x+2 at
// the thread's own (y, z), the raw first-difference sums
//   uy = f[y-2] - 8 f[y-1] + 8 f[y+1] - f[y+2]   and   uz (same along z),
// so the mixed derivatives d_x d_y and d_x d_z come from five registers
// instead of sixteen shared-memory taps each:
//   sum_{m,n} c_m c_n f[x+m, y+n] = sum_m c_m uy(x+m),  c = (1, -8, 0, 8, -1),
// which is the reference's 5x5 outer-product stencil (core/derivatives.py:121-173)
// regrouped; only the rounding order differs.  d_y d_z uses the 16 in-plane taps.
//
// The stage input is X = F + a V + b L (the RK4 stage fields of
// core/integrator.py:50-92, built on the fly), so a stage reads each input
// array once per site plus the halo.
#pragma once

#include <type_traits>

#include "sky_kernels.cuh"
#include "sky_tma.cuh"

namespace sky {

// A row of a staged plane holds z = z0 - ZOFF .. z0 - ZOFF + HZ - 1.  Narrow rows
// (36 values: z0-2 .. z0+33) are filled element by element; wide rows (40 values:
// z0-4 .. z0+35) are filled with 16-byte copies, which needs Z to be a multiple of
// 16 / sizeof(T) so that every 16-byte chunk of a row starts on a 16-byte boundary
// and lies wholly inside or (as the first chunk at z0 = 0) wholly outside the lattice
// in z; a chunk crossing z = Z copies its in-lattice part and zero-fills the rest.
constexpr size_t kMaxSmemPerBlock = 232448;  // 227 KB of dynamic shared memory per block

template <int C_, int BY_, bool WIDE_ = false>
struct MarchShape {
    static constexpr int C = C_, BY = BY_, BZ = 32;
    static constexpr bool WIDE = WIDE_;
    static constexpr int HY = BY + 4, HZ = WIDE ? BZ + 8 : BZ + 4;
    static constexpr int ZOFF = WIDE ? 4 : 2;
    static constexpr int PLANE = HY * HZ;  // one component of one plane, with halo
    static constexpr int SLOT = C * PLANE;  // all components of one plane
    static constexpr int RING = 5;
    static constexpr int NTHREADS = BZ * BY;
    static constexpr int NPER = (SLOT + NTHREADS - 1) / NTHREADS;  // plane elements per thread
    // Sources staged through shared memory: all nsrc, or only the first two when
    // three would not fit in one block's 227 KB (FP64 rho); the third source is
    // then read from global memory while the plane is combined.
    template <typename T, typename S = T>
    static constexpr int staged(int nsrc) {
        return (nsrc == 3 && size_t(RING) * SLOT * sizeof(T) + 3 * size_t(SLOT) * sizeof(S) > kMaxSmemPerBlock) ? 2
                                                                                                            : nsrc;
    }
    // ring + staging (+ a second ring for the low parts of a compensated field);
    // the staging area holds values of the source type S
    template <typename T, typename S = T>
    static constexpr size_t smem_bytes(int nsrc, bool lo = false) {
        return size_t(RING) * (lo ? 2 : 1) * SLOT * sizeof(T) + size_t(staged<T, S>(nsrc)) * SLOT * sizeof(S);
    }
    // TMA staging (wide rows): a ring into which the copy engine writes the first
    // source (5 + LA slots for LA planes in flight; a compensated field's low parts
    // get a second ring), plus LA staging slots for each further source.
    // kTmaPlanesInFlight planes are kept in flight when that fits one block's shared
    // memory.  One is the default: on the omega 128^3 FP32 stages two planes in flight
    // measured no faster for stages 2 and 3 (80.5 against 79.5 us, 80.8 against 82.3 us)
    // and slower for stage 4 (152 against 140 us), whose larger shared-memory share
    // leaves less L1 for the update's global loads.
    static constexpr int kTmaPlanesInFlight = 1;
    static constexpr size_t tma_slots(int nsrc, bool lo, int la) {
        return lo ? 2 * size_t(RING + la) : size_t(RING + la) + size_t(la) * size_t(nsrc - 1);
    }
    template <typename T>
    static constexpr int tma_lookahead(int nsrc, bool lo = false) {
        return (kTmaPlanesInFlight > 1 && !lo && tma_slots(nsrc, lo, 2) * SLOT * sizeof(T) + 128 <= kMaxSmemPerBlock)
                   ? 2
                   : 1;
    }
    template <typename T>
    static constexpr size_t smem_bytes_tma(int nsrc, bool lo = false) {
        return tma_slots(nsrc, lo, tma_lookahead<T>(nsrc, lo)) * size_t(SLOT) * sizeof(T);
    }
};

// Whether an epilogue wants a call at the start of each site (before the stencil
// arithmetic), e.g. to issue the global loads its operator() will consume.
// plane_begin(x): called by every thread once per computed plane x, right after the
// plane barrier (TMA staging only).
template <class E, class = void>
struct HasPlaneBegin : std::false_type {};
template <class E>
struct HasPlaneBegin<E, std::void_t<decltype(std::declval<E&>().plane_begin(0))>> : std::true_type {};

// begin_site(s, N, next): s is the site about to be computed and next the same
// thread's site on the following plane of the tile (-1 on the tile's last plane).
template <class E, class = void>
struct HasBeginSite : std::false_type {};
template <class E>
struct HasBeginSite<E, std::void_t<decltype(std::declval<E&>().begin_site(int64_t(0), int64_t(0), int64_t(0)))>>
    : std::true_type {};

// Per-tile TMA state of a marching kernel: the kernel's two mbarriers
// (initialised once per launch; planes alternate between them when two are in
// flight), the parity bit of the phase each one completes next, the maps of the
// tile's sources (null: the source reads as zero) and the launch-wide error word
// that a timed-out wait sets.
struct TmaTile {
    uint64_t* bar;
    uint32_t phase;
    const TmaMap* map[3];
    int* status;
};

// ---------------------------------------------------------------------------
// cp.async (sm_80+ asynchronous global -> shared copies; zero-fill when the
// source size is 0, so out-of-lattice halo points read as 0 without a load).
// ---------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, bool valid) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    const int n = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(BYTES), "r"(n)
                 : "memory");
}
// 16-byte copy of `nbytes` (0..16) bytes, zero-filling the rest of the 16.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int nbytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Per-thread element offsets of the haloed plane: element k of thread tid is
// idx = tid + k*NTHREADS of the slot, i.e. (c, yy, zz) = decompose(idx); its
// global offset within the x-plane is c*N + gy*Z + gz (int32), or -1 when the
// point lies outside the lattice in y or z (or idx is past the slot).  The
// host guarantees C*N < 2^31 for marching launches.
template <class M>
struct PlaneOffsets {
    int off[M::NPER];
    __device__ __forceinline__ void init(const Params& p, int64_t N, int y0, int z0) {
        const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
        for (int k = 0; k < M::NPER; ++k) {
            const int idx = tid + k * M::NTHREADS;
            const int row = idx / M::HZ;
            const int zz = idx - row * M::HZ;
            const int c = row / M::HY;
            const int yy = row - c * M::HY;
            const int gy = y0 - 2 + yy, gz = z0 - M::ZOFF + zz;
            const bool ok = idx < M::SLOT && gy >= 0 && gy < p.Y && gz >= 0 && gz < p.Z;
            off[k] = ok ? static_cast<int>(c * N + (int64_t)gy * p.Z + gz) : -1;
        }
    }
};

// Wide rows: per-thread 16-byte chunks of the haloed plane.  Chunk k of thread tid
// is ci = tid + k*NTHREADS; its global element offset within the x-plane and the
// number of its bytes inside the lattice (0 when outside or past the slot).
template <class M, typename T>
struct PlaneChunks {
    static constexpr int VW = 16 / int(sizeof(T));
    static constexpr int CPR = M::HZ / VW;
    static constexpr int NCHS = M::C * M::HY * CPR;
    static constexpr int NCH = (NCHS + M::NTHREADS - 1) / M::NTHREADS;
    int off[NCH];
    int nb[NCH];
    __device__ __forceinline__ void init(const Params& p, int64_t N, int y0, int z0) {
        static_assert(M::WIDE && M::HZ % VW == 0, "16-byte chunks need the wide row layout");
        const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
        for (int k = 0; k < NCH; ++k) {
            const int ci = tid + k * M::NTHREADS;
            const int row = ci / CPR;
            const int cz = ci - row * CPR;
            const int c = row / M::HY;
            const int yy = row - c * M::HY;
            const int gy = y0 - 2 + yy, gz0 = z0 - M::ZOFF + cz * VW;
            const bool ok = ci < NCHS && gy >= 0 && gy < p.Y && gz0 >= 0 && gz0 < p.Z;
            off[k] = ok ? static_cast<int>(c * N + (int64_t)gy * p.Z + gz0) : 0;
            nb[k] = ok ? int(sizeof(T)) * min(VW, p.Z - gz0) : 0;
        }
    }
};

// Source s of a plane lands at stage + s * DST (DST = M::SLOT: consecutive staging
// slots; a ring of R slots per source when the plane goes straight into the ring).
template <class M, int NSRC, typename T, int DST = M::SLOT>
__device__ __forceinline__ void plane_issue_wide(T* __restrict__ stage, const PlaneChunks<M, T>& pc,
                                                 const T* const (&src)[3], int64_t plane_base, bool xok) {
    using PC = PlaneChunks<M, T>;
    const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
    for (int k = 0; k < PC::NCH; ++k) {
        const int ci = tid + k * M::NTHREADS;
        if (PC::NCHS % M::NTHREADS == 0 || ci < PC::NCHS) {
#pragma unroll
            for (int s = 0; s < NSRC; ++s) {
                const T* g = src[s];
                const int n = (xok && g != nullptr) ? pc.nb[k] : 0;
                cp_async16(stage + s * DST + ci * PC::VW, n ? (const void*)(g + plane_base + pc.off[k])
                                                                : (const void*)src[0], n);
            }
        }
    }
    cp_async_commit();
}

template <class M, int NSRC, typename T, typename S = T>
__device__ __forceinline__ void plane_combine_wide(T* __restrict__ slot, const S* __restrict__ stage, T a, T b) {
    using PC = PlaneChunks<M, S>;
    const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
    for (int k = 0; k < PC::NCH; ++k) {
        const int ci = tid + k * M::NTHREADS;
        if (PC::NCHS % M::NTHREADS == 0 || ci < PC::NCHS) {
            T v[PC::VW];
#pragma unroll
            for (int e = 0; e < PC::VW; ++e) v[e] = T(stage[ci * PC::VW + e]);
            if (NSRC > 1) {
#pragma unroll
                for (int e = 0; e < PC::VW; ++e) v[e] += a * T(stage[M::SLOT + ci * PC::VW + e]);
            }
            if (NSRC > 2) {
#pragma unroll
                for (int e = 0; e < PC::VW; ++e) v[e] += b * T(stage[2 * M::SLOT + ci * PC::VW + e]);
            }
#pragma unroll
            for (int e = 0; e < PC::VW; ++e) slot[ci * PC::VW + e] = v[e];
        }
    }
}

// Issue the cp.async copies of one x-plane (element offset plane_base) of the
// NSRC source arrays into the staging slots; a null source reads as zero.
template <class M, int NSRC, typename T, int DST = M::SLOT>
__device__ __forceinline__ void plane_issue(T* __restrict__ stage, const PlaneOffsets<M>& po, const T* const (&src)[3],
                                            int64_t plane_base, bool xok) {
    // T here is the source (staging) type
    const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
    for (int k = 0; k < M::NPER; ++k) {
        const int idx = tid + k * M::NTHREADS;
        if (M::SLOT % M::NTHREADS == 0 || idx < M::SLOT) {
            const bool ok = xok && po.off[k] >= 0;
#pragma unroll
            for (int s = 0; s < NSRC; ++s) {
                const T* g = src[s];
                const bool v = ok && g != nullptr;
                cp_async<sizeof(T)>(stage + s * DST + idx,
                                    v ? (const void*)(g + plane_base + po.off[k]) : (const void*)src[0], v);
            }
        }
    }
    cp_async_commit();
}

// Combine the thread's own staged elements (source type S) into a ring slot of
// type T: X = F + a V + b L.
template <class M, int NSRC, typename T, typename S = T>
__device__ __forceinline__ void plane_combine(T* __restrict__ slot, const S* __restrict__ stage, T a, T b) {
    const int tid = threadIdx.x + M::BZ * threadIdx.y;
#pragma unroll
    for (int k = 0; k < M::NPER; ++k) {
        const int idx = tid + k * M::NTHREADS;
        if (M::SLOT % M::NTHREADS == 0 || idx < M::SLOT) {
            T v = T(stage[idx]);
            if (NSRC > 1) v += a * T(stage[M::SLOT + idx]);
            if (NSRC > 2) v += b * T(stage[2 * M::SLOT + idx]);
            slot[idx] = v;
        }
    }
}

// As plane_combine for three sources of which only the first two were staged:
// the third (src2, element offsets of the plane at plane_base) is read from
// global memory here, in groups of eight loads issued back to back (one memory
// latency per group); plane_prefetch_l2 brought its lines into L2 one plane
// earlier.
template <class M, typename T, typename S = T>
__device__ __forceinline__ void plane_combine_g(T* __restrict__ slot, const S* __restrict__ stage, T a, T b,
                                                const PlaneOffsets<M>& po, const S* __restrict__ src2,
                                                int64_t plane_base, bool xok) {
    constexpr int G = 8;
    const int tid = threadIdx.x + M::BZ * threadIdx.y;
    const bool any = xok && src2 != nullptr;
#pragma unroll
    for (int k0 = 0; k0 < M::NPER; k0 += G) {
        T l[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const int k = k0 + j;
            l[j] = T(0);
            if (k < M::NPER && any && po.off[k] >= 0) l[j] = T(__ldg(src2 + plane_base + po.off[k]));
        }
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const int k = k0 + j;
            const int idx = tid + k * M::NTHREADS;
            if (k < M::NPER && (M::SLOT % M::NTHREADS == 0 || idx < M::SLOT))
                slot[idx] = T(stage[idx]) + a * T(stage[M::SLOT + idx]) + b * l[j];
        }
    }
}

// L2 prefetch of the thread's elements of one plane of src (narrow-row offsets).
template <class M, typename S>
__device__ __forceinline__ void plane_prefetch_l2(const PlaneOffsets<M>& po, const S* src, int64_t plane_base,
                                                  bool xok) {
    if (!xok || src == nullptr) return;
#pragma unroll
    for (int k = 0; k < M::NPER; ++k)
        if (po.off[k] >= 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(src + plane_base + po.off[k]));
}

// Raw first-difference sum c_m f[m*st], c = (1, -8, 0, 8, -1) for m = -2..2.
template <typename T>
__device__ __forceinline__ T diff5(const T* f, int st) {
    return (f[-2 * st] - f[2 * st]) + T(8) * (f[st] - f[-st]);
}

// ---------------------------------------------------------------------------
// One tile: planes xa-2 .. xe+1 of lattice p through the ring; the point
// physics Th<T> and the epilogue Epi run at every in-lattice site with x in
// [xa, xe).  DENS adds the FP64 energy / baryon densities of the stage input
// to esum / bsum (compensated).  LO (with DENS, NSRC = 2): src[1] holds the low
// parts of a compensated field; the stencils see the high parts and the FP64
// densities use hi + lo (a null src[1] reads as zero).
// When the stage input is the field itself (NSRC = 1, or the hi / lo pair of LO,
// with S = T) the planes are copied straight into a six-slot ring, whose sixth
// slot takes the plane in flight: no staging copy and one barrier per plane.
// ---------------------------------------------------------------------------
// S: type of the source arrays and of the staging area (S = T, or float sources
// staged for an FP64 ring).
// GRAD = false: density-only walk (no second derivatives, no gradient, no
// epilogue); the ring may then hold just the first M::C <= Th::C components
// (the baryon density needs phi_0..3 only) and each site's FP64 density (the
// potential of the RK4 dynamics when DENS & 4, else energy when DENS & 1, else
// baryon) is passed to epi.density(s, value); with DENS & 16 the site's FP64
// field values and first derivatives go to epi.site(s, phi, D) instead.
// TMA: the planes are copied by the tensor-memory accelerator (one thread issues
// one box copy per source and plane; sky_tma.cuh) instead of per-thread cp.async;
// wide rows and S = T only.  The first source goes straight into a six-slot ring,
// further sources into staging slots that are added into the ring slot, and one
// barrier per plane orders the copies with the readers.  Returns false (every
// thread of the block) when a wait for a copy gave up (the block's error bit is
// then set in tma->status).
template <template <typename> class Th, class M, typename T, int NSRC, int DENS, class Epi, bool LO = false,
          typename S = T, bool GRAD = true, bool TMA = false>
__device__ __forceinline__ bool march_tile(T* __restrict__ sm, const Params& p, const S* const (&src)[3], T a, T b,
                                           int xa, int xe, int y0, int z0, Epi& epi, KSum& esum, KSum& bsum,
                                           TmaTile* tma = nullptr) {
    constexpr int C = M::C;
    constexpr int CT = Th<double>::C;  // components of the theory
    // register queues of the y / z first-difference sums for C <= 5; with more
    // components (rho, C = 13) they would not fit the registers, and the mixed
    // derivatives d_x d_y, d_x d_z take 16 taps across the ring planes instead
    constexpr bool QUEUE = GRAD && C <= 5;
    static_assert(GRAD ? Th<T>::C == C : C <= CT, "component count mismatch");
    static_assert(!LO || (DENS != 0 && NSRC == 2), "low-part ring only for the stage-1 density");
    static_assert(!LO || (std::is_same<S, T>::value && sizeof(T) == 4), "low-part ring needs FP32 sources");
    constexpr bool DIRECT = (NSRC == 1 || LO) && std::is_same<S, T>::value;
    constexpr int NST = M::template staged<T, S>(NSRC);  // sources staged in shared memory
    static_assert(NST == NSRC || !M::WIDE, "the unstaged third source is read with narrow-row offsets");
    static_assert(!TMA || (M::WIDE && std::is_same<S, T>::value && NST == NSRC), "TMA staging: wide rows, S = T");
    // planes in flight ahead of the one being consumed (TMA), and ring slots
    constexpr int LA = TMA ? M::template tma_lookahead<T>(NSRC, LO) : 1;
    constexpr int R = TMA ? M::RING + LA : (DIRECT ? M::RING + 1 : M::RING);
    constexpr int DST = DIRECT ? R * M::SLOT : M::SLOT;  // distance between the sources' copies
    // shared memory: DIRECT: ring (R slots) [+ low-part ring (R slots)];
    // TMA: ring (R slots) + LA buffers of NSRC - 1 staging slots;
    // otherwise: ring (5 slots) + NSRC staging slots of S
    T* ring = sm;
    S* stage = reinterpret_cast<S*>(sm + (TMA ? R : M::RING) * M::SLOT);
    T* ring_lo = sm + R * M::SLOT;

    const int64_t N = n_sites(p);
    const int64_t YZ = (int64_t)p.Y * p.Z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int y = y0 + ty, z = z0 + tx;
    const bool own = (y < p.Y) && (z < p.Z);
    StencilCoef<T> k;
    k.init(p);
    // element offsets (narrow rows) or 16-byte chunks (wide rows) of the haloed plane
    using PO = typename std::conditional<M::WIDE, PlaneChunks<M, S>, PlaneOffsets<M>>::type;
    PO po;
    po.init(p, N, y0, z0);
    constexpr int CQ = QUEUE ? C : 1;
    T uq[CQ][5], wq[CQ][5];  // uy / uz queues for planes x-2 .. x+2
#pragma unroll
    for (int c = 0; c < CQ; ++c)
#pragma unroll
        for (int m = 0; m < 5; ++m) uq[c][m] = wq[c][m] = T(0);
    const int q0 = xa - 2, q1 = xe + 1;
    const int lofs = (ty + 2) * M::HZ + (tx + M::ZOFF);  // thread's site within a component plane
    auto issue = [&](int64_t base, bool xok, int dslot) {
        S* dst = DIRECT ? reinterpret_cast<S*>(ring + dslot * M::SLOT) : stage;
        if constexpr (M::WIDE) {
            plane_issue_wide<M, NST, S, DST>(dst, po, src, base, xok);
        } else {
            plane_issue<M, NST, S, DST>(dst, po, src, base, xok);
            if constexpr (NST < NSRC) plane_prefetch_l2<M, S>(po, src[2], base, xok);
        }
    };
    // TMA: thread 0 copies plane qq of every present source (a plane outside the
    // lattice arrives as zeros); source 0 into ring slot dslot, the low parts into the
    // low-part ring, further sources into the staging slots
    const int tid0 = threadIdx.x + M::BZ * threadIdx.y;
    // buffer nb (mbarrier nb, staging buffer nb) carries planes q0 + nb, q0 + nb + LA, ...
    // (named apart from the combine weight b of the third source)
    auto issue_tma = [&](int qq, int dslot, int nb) {
        if (tid0 != 0) return;
        constexpr uint32_t box = uint32_t(M::SLOT * sizeof(T));
        uint32_t n = 1;
#pragma unroll
        for (int k = 1; k < NSRC; ++k) n += tma->map[k] != nullptr ? 1u : 0u;
        uint64_t* bar = tma->bar + nb;
        T* stg = reinterpret_cast<T*>(stage) + nb * (NSRC - 1) * M::SLOT;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, n * box);
        const int zc = z0 - M::ZOFF, yc = y0 - 2;
        tma_load_plane(ring + dslot * M::SLOT, tma->map[0], zc, yc, qq, 0, bar);
#pragma unroll
        for (int k = 1; k < NSRC; ++k) {
            if (tma->map[k] == nullptr) continue;
            T* dst = LO ? ring_lo + dslot * M::SLOT : stg + (k - 1) * M::SLOT;
            tma_load_plane(dst, tma->map[k], zc, yc, qq, 0, bar);
        }
    };
    __syncthreads();
    if constexpr (TMA) {
        issue_tma(q0, 0, 0);
        if (LA > 1 && q0 + 1 <= q1) issue_tma(q0 + 1, 1, 1);
    } else {
        issue((int64_t)q0 * YZ, q0 >= 0 && q0 < p.X, 0);
    }
    int slot = 0;  // ring slot of plane q
    for (int q = q0; q <= q1; ++q) {
        if constexpr (TMA) {
            // plane q has landed; for further sources, add a V + b L into the ring slot
            const int nb = LA > 1 ? ((q - q0) & 1) : 0;
            const bool ok = mbar_wait_bounded(tma->bar + nb, (tma->phase >> nb) & 1u);
            tma->phase ^= 1u << nb;
            if constexpr (!DIRECT) {
                using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
                constexpr int VW = 16 / int(sizeof(T));
                constexpr int NV = M::SLOT / VW;
                static_assert(M::SLOT % VW == 0, "slot of whole 16-byte vectors");
                V4* dstv = reinterpret_cast<V4*>(ring + slot * M::SLOT);
                const V4* s1 = reinterpret_cast<const V4*>(stage) + nb * (NSRC - 1) * NV;
                const V4* s2 = s1 + NV;
                const bool h1 = tma->map[1] != nullptr;
                const bool h2 = NSRC > 2 && tma->map[2] != nullptr;
                if (h1 || h2) {
                    for (int i = tid0; i < NV; i += M::NTHREADS) {
                        V4 v = dstv[i];
                        T* e = reinterpret_cast<T*>(&v);
                        if (h1) {
                            const V4 u = s1[i];
                            const T* f = reinterpret_cast<const T*>(&u);
#pragma unroll
                            for (int j = 0; j < VW; ++j) e[j] += a * f[j];
                        }
                        if (h2) {
                            const V4 u = s2[i];
                            const T* f = reinterpret_cast<const T*>(&u);
#pragma unroll
                            for (int j = 0; j < VW; ++j) e[j] += b * f[j];
                        }
                        dstv[i] = v;
                    }
                }
            }
            // the ring slots are written by ordinary stores (the combine above) and read by
            // ordinary loads, and later overwritten by the copy engine: every thread orders
            // its own generic accesses before those async-proxy writes, and the barrier
            // then orders all threads' accesses before the next copy is issued
            fence_proxy_async_smem();
            // every thread has its plane q (and finished the centre of plane q - 1): the
            // ring slot of plane q - 5 and staging buffer nb are free for plane q + LA
            if (__syncthreads_or(ok ? 0 : 1)) {
                if (tid0 == 0) {
                    atomicOr(tma->status, 1);
                    // let late copies land before the block exits
                    for (int k = 0; k < LA; ++k) mbar_wait_bounded(tma->bar + k, (tma->phase >> k) & 1u);
                }
                return false;
            }
            if (q + LA <= q1) issue_tma(q + LA, (slot + LA) % R, nb);
            if constexpr (HasPlaneBegin<Epi>::value) {
                if (q - 2 >= xa) epi.plane_begin(q - 2);
            }
        } else if constexpr (DIRECT) {
            cp_async_wait_all();
            // (A) plane q has landed for every thread, and every thread finished the
            // previous centre: the slot of plane q - 5 (staging: the staging area) is free
            __syncthreads();
            if (q < q1) issue((int64_t)(q + 1) * YZ, q + 1 >= 0 && q + 1 < p.X, slot + 1 == R ? 0 : slot + 1);
        } else {
            cp_async_wait_all();
            __syncthreads();  // (A), as above
            if constexpr (NST < NSRC) {
                if constexpr (!M::WIDE)
                    plane_combine_g<M, T, S>(ring + slot * M::SLOT, stage, a, b, po, src[2], (int64_t)q * YZ,
                                             q >= 0 && q < p.X);
            } else if constexpr (M::WIDE) {
                plane_combine_wide<M, NSRC, T, S>(ring + slot * M::SLOT, stage, a, b);
            } else {
                plane_combine<M, NSRC, T, S>(ring + slot * M::SLOT, stage, a, b);
            }
            if (q < q1) issue((int64_t)(q + 1) * YZ, q + 1 >= 0 && q + 1 < p.X, 0);
            __syncthreads();  // (B) slot complete
        }
        // arrival: first-difference sums of plane q at (y, z)
        if constexpr (QUEUE) {
            const T* P = ring + slot * M::SLOT + lofs;
#pragma unroll
            for (int c = 0; c < C; ++c) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    uq[c][m] = uq[c][m + 1];
                    wq[c][m] = wq[c][m + 1];
                }
                uq[c][4] = diff5<T>(P + c * M::PLANE, M::HZ);
                wq[c][4] = diff5<T>(P + c * M::PLANE, 1);
            }
        }
        const int x = q - 2;
        if (x >= xa && own) {
            // plane q-j sits in slot (slot + R - j) % R: x-2 = q-4, ..., x+2 = q
            const T* Pm2 = ring + ((slot + R - 4) % R) * M::SLOT + lofs;
            const T* Pm1 = ring + ((slot + R - 3) % R) * M::SLOT + lofs;
            const T* P0 = ring + ((slot + R - 2) % R) * M::SLOT + lofs;
            const T* Pp1 = ring + ((slot + R - 1) % R) * M::SLOT + lofs;
            const T* Pp2 = ring + slot * M::SLOT + lofs;
            const Mask mk = site_mask(p, x, y, z);
            const int64_t s = (int64_t)x * YZ + (int64_t)y * p.Z + z;
            // baryon density of an FP32 stage input, from the FP32 derivatives the gradient uses
            // (its FP64 sum needs no more than FP32 per-site accuracy; only the energy, which
            // decides the arrest, is evaluated in FP64)
            [[maybe_unused]] double b32 = 0.0;
            if constexpr (HasBeginSite<Epi>::value) epi.begin_site(s, N, x + 1 < xe ? s + YZ : int64_t(-1));
            if constexpr (GRAD) {
            T phi[C], D[3][C], Sd[6][C], g[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int co = c * M::PLANE;
                const T* f = P0 + co;
                const T f0 = f[0];
                phi[c] = f0;
                {
                    const T fm2 = Pm2[co], fm1 = Pm1[co], fp1 = Pp1[co], fp2 = Pp2[co];
                    D[0][c] = mk.px ? k.d1a[0] * (fp1 - fm1) - k.d1b[0] * (fp2 - fm2) : T(0);
                    Sd[0][c] = mk.px ? k.d2a[0] * (fp1 + fm1) - k.d2b[0] * (fp2 + fm2) - k.d2c[0] * f0 : T(0);
                }
                {
                    const T fm2 = f[-2 * M::HZ], fm1 = f[-M::HZ], fp1 = f[M::HZ], fp2 = f[2 * M::HZ];
                    D[1][c] = mk.py ? k.d1a[1] * (fp1 - fm1) - k.d1b[1] * (fp2 - fm2) : T(0);
                    Sd[1][c] = mk.py ? k.d2a[1] * (fp1 + fm1) - k.d2b[1] * (fp2 + fm2) - k.d2c[1] * f0 : T(0);
                }
                {
                    const T fm2 = f[-2], fm1 = f[-1], fp1 = f[1], fp2 = f[2];
                    D[2][c] = mk.pz ? k.d1a[2] * (fp1 - fm1) - k.d1b[2] * (fp2 - fm2) : T(0);
                    Sd[2][c] = mk.pz ? k.d2a[2] * (fp1 + fm1) - k.d2b[2] * (fp2 + fm2) - k.d2c[2] * f0 : T(0);
                }
                T sxy, sxz;
                if constexpr (QUEUE) {
                    sxy = (uq[c][0] - uq[c][4]) + T(8) * (uq[c][3] - uq[c][1]);
                    sxz = (wq[c][0] - wq[c][4]) + T(8) * (wq[c][3] - wq[c][1]);
                } else {
                    sxy = (diff5<T>(Pm2 + co, M::HZ) - diff5<T>(Pp2 + co, M::HZ)) +
                          T(8) * (diff5<T>(Pp1 + co, M::HZ) - diff5<T>(Pm1 + co, M::HZ));
                    sxz = (diff5<T>(Pm2 + co, 1) - diff5<T>(Pp2 + co, 1)) +
                          T(8) * (diff5<T>(Pp1 + co, 1) - diff5<T>(Pm1 + co, 1));
                }
                Sd[3][c] = (mk.mx && mk.my) ? k.mix[0] * sxy : T(0);
                Sd[4][c] = (mk.mx && mk.mz) ? k.mix[1] * sxz : T(0);
                Sd[5][c] = (mk.my && mk.mz) ? k.mix[2] * mixed16<T>(f, M::HZ, 1) : T(0);
            }
            Th<T>::gradient(phi, D, Sd, p, g);
            if constexpr (DENS != 0 && sizeof(T) == 4) b32 = double(Th<T>::baryon(phi, D, p));
            epi(s, N, phi, g);
            }
            if (DENS) {
                // FP64 energy and baryon densities of the stage input (stage 1: the field itself),
                // evaluated after the gradient so their registers do not overlap
                StencilCoef<double> kd;
                kd.init(p);
                double phd[CT], Dd[3][CT];
#pragma unroll
                for (int c = C; c < CT; ++c) phd[c] = Dd[0][c] = Dd[1][c] = Dd[2][c] = 0.0;
                // difference of two tap values in FP64.  Compensated field: the
                // difference of the high parts is split exactly into s + e (Knuth's
                // TwoSum, FP32), e absorbs the difference of the low parts, and only s
                // and that remainder are converted: two conversions instead of four,
                // with an error below 2^-47 of the field's magnitude
                const ptrdiff_t dlo = ring_lo - ring;
                auto dif = [&](const T* u, const T* v) -> double {
                    if constexpr (LO) {
                        const T ua = u[0], vb = -v[0];
                        const T s = ua + vb, bb = s - ua;
                        const T e = (ua - (s - bb)) + (vb - bb);
                        return double(s) + double(e + (u[dlo] - v[dlo]));
                    } else {
                        return double(u[0]) - double(v[0]);
                    }
                };
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const int co = c * M::PLANE;
                    const T* f = P0 + co;
                    phd[c] = LO ? double(f[0]) + double(f[dlo]) : double(f[0]);
                    const double xd = dif(Pp1 + co, Pm1 + co), xd2 = dif(Pp2 + co, Pm2 + co);
                    const double yd = dif(f + M::HZ, f - M::HZ), yd2 = dif(f + 2 * M::HZ, f - 2 * M::HZ);
                    const double zd = dif(f + 1, f - 1), zd2 = dif(f + 2, f - 2);
                    Dd[0][c] = mk.px ? kd.d1a[0] * xd - kd.d1b[0] * xd2 : 0.0;
                    Dd[1][c] = mk.py ? kd.d1a[1] * yd - kd.d1b[1] * yd2 : 0.0;
                    Dd[2][c] = mk.pz ? kd.d1a[2] * zd - kd.d1b[2] * zd2 : 0.0;
                }
                if constexpr (GRAD) {
                    ksum_add(esum, Th<double>::energy(phd, Dd, p));
                    if constexpr (sizeof(T) == 4)
                        ksum_add(bsum, b32);
                    else
                        ksum_add(bsum, Th<double>::baryon(phd, Dd, p));
                } else if constexpr ((DENS & 16) != 0) {
                    epi.site(s, phd, Dd);  // the epilogue reads the FP64 field and first derivatives
                } else {
                    double v;
                    if constexpr ((DENS & 4) != 0)
                        v = Dynamics<Th>::potential(phd, Dd, p);  // potential of the RK4 dynamics
                    else
                        v = (DENS & 1) ? Th<double>::energy(phd, Dd, p) : Th<double>::baryon(phd, Dd, p);
                    ksum_add(esum, v);
                    epi.density(s, v);
                }
            }
        }
        slot = (slot + 1) % R;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Tiling of one lattice into (x-chunk, 8-row y, 32-column z) tiles.
// ---------------------------------------------------------------------------
struct MarchGrid {
    int nz, ny, nx, xc;
    __host__ __device__ int count() const { return nz * ny * nx; }
};

template <class M>
__host__ __device__ inline MarchGrid march_grid(const Params& p, int xc) {
    MarchGrid g;
    g.xc = xc;
    g.nz = (p.Z + M::BZ - 1) / M::BZ;
    g.ny = (p.Y + M::BY - 1) / M::BY;
    g.nx = (p.X + xc - 1) / xc;
    return g;
}

__device__ __forceinline__ void march_origin(const MarchGrid& g, int t, int by, int& xa, int& xe, int& y0, int& z0,
                                             int X) {
    const int iz = t % g.nz;
    const int r = t / g.nz;
    const int iy = r % g.ny;
    const int ix = r / g.ny;
    z0 = iz * 32;
    y0 = iy * by;
    xa = ix * g.xc;
    xe = min(xa + g.xc, X);
}

// ---------------------------------------------------------------------------
// Plain reference-layout gradient (drop-in for do_gradient_step_kernel):
// EG = projected gradient of `field`, l = -dt EG.
// ---------------------------------------------------------------------------
template <typename T>
struct PlainEpi {
    T* eg;
    T* l;
    T mdt;
    template <int C>
    __device__ __forceinline__ void operator()(int64_t s, int64_t N, const T (&)[C], const T (&g)[C]) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
            eg[c * N + s] = g[c];
            l[c * N + s] = mdt * g[c];
        }
    }
};

// ---------------------------------------------------------------------------
// Reference-layout FP64 density (drop-in for compute_energy_kernel /
// compute_skyrmion_number_kernel): per-site e h^3 or b h^3 (optional) and its
// compensated sum finished by the last block (deterministic for a given grid).
// MODE 0: energy (all components), 1: baryon (phi_0..3; M::C = 4).
// ---------------------------------------------------------------------------
struct DensEpi {
    double* dens;
    __device__ __forceinline__ void density(int64_t s, double v) {
        if (dens) dens[s] = v;
    }
};

template <template <typename> class Th, class M, int MODE>
__global__ void __launch_bounds__(M::NTHREADS) k_march_density(Params p, MarchGrid mg, const double* __restrict__ field,
                                                               double* __restrict__ dens, double* __restrict__ scratch,
                                                               double* __restrict__ out_dev) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    __shared__ KSum shk[32];
    DensEpi epi{dens};
    const double* const src[3] = {field, nullptr, nullptr};
    KSum es{0.0, 0.0}, unused{0.0, 0.0};
    for (int t = blockIdx.x; t < mg.count(); t += gridDim.x) {
        int xa, xe, y0, z0;
        march_origin(mg, t, M::BY, xa, xe, y0, z0, p.X);
        march_tile<Th, M, double, 1, (MODE == 0 ? 1 : 2), DensEpi, false, double, false>(sm, p, src, 0.0, 0.0, xa, xe,
                                                                                         y0, z0, epi, es, unused);
    }
    if (scratch) finish_ksum(es, scratch, out_dev, shk);
}

// ---------------------------------------------------------------------------
// Baryon moments of a reference-layout FP64 field, for the centre of mass and
// the RMS radius (compute_center_of_mass_kernel / compute_rms_radius_kernel,
// th/nuclear_skyrme/kernels.py:678-758, and their host sums,
// th/nuclear_skyrme/observables.py:182-270): with b the baryon density of a
// site (h^3 included) and r = (h_x i, h_y j, h_z k) its grid point
// (create_grid_kernel), the nine sums of b, b r, |b|, |b| r and |b| |r|^2.
// Each block writes its compensated partials to parts[18 * block + 2 q].
// ---------------------------------------------------------------------------
constexpr int kMoments = 9;

struct MomentEpi {
    Params p;
    KSum m[kMoments];
    __device__ __forceinline__ void density(int64_t s, double b) {
        const int64_t YZ = (int64_t)p.Y * p.Z;
        const int ix = (int)(s / YZ);
        const int64_t r = s - (int64_t)ix * YZ;
        const int iy = (int)(r / p.Z);
        const int iz = (int)(r - (int64_t)iy * p.Z);
        const double x = p.hx * ix, y = p.hy * iy, z = p.hz * iz;
        const double a = fabs(b);
        ksum_add(m[0], b);
        ksum_add(m[1], b * x);
        ksum_add(m[2], b * y);
        ksum_add(m[3], b * z);
        ksum_add(m[4], a);
        ksum_add(m[5], a * x);
        ksum_add(m[6], a * y);
        ksum_add(m[7], a * z);
        ksum_add(m[8], a * (x * x + y * y + z * z));
    }
};

template <template <typename> class Th, class M>
__global__ void __launch_bounds__(M::NTHREADS) k_march_moments(Params p, MarchGrid mg, const double* __restrict__ field,
                                                               double* __restrict__ parts) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    __shared__ KSum shk[M::NTHREADS / 32];
    MomentEpi epi;
    epi.p = p;
#pragma unroll
    for (int q = 0; q < kMoments; ++q) epi.m[q] = KSum{0.0, 0.0};
    const double* const src[3] = {field, nullptr, nullptr};
    KSum es{0.0, 0.0}, unused{0.0, 0.0};
    for (int t = blockIdx.x; t < mg.count(); t += gridDim.x) {
        int xa, xe, y0, z0;
        march_origin(mg, t, M::BY, xa, xe, y0, z0, p.X);
        march_tile<Th, M, double, 1, 2, MomentEpi, false, double, false>(sm, p, src, 0.0, 0.0, xa, xe, y0, z0, epi,
                                                                         es, unused);
    }
#pragma unroll
    for (int q = 0; q < kMoments; ++q) {
        const KSum b = block_ksum(epi.m[q], shk);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            parts[2 * kMoments * blockIdx.x + 2 * q] = b.s;
            parts[2 * kMoments * blockIdx.x + 2 * q + 1] = b.c;
        }
    }
}

// ---------------------------------------------------------------------------
// Nuclear-model diagnostics in one FP64 pass (th/nuclear_skyrme/kernels.py:
// 484-1033 and observables.py:273-487): per site the left currents L_k and
// isorotation currents T_i, their Gram matrices LL, TT, LT, and with
// r = grid point - centre of mass (grid point = (h_x i, h_y j, h_z k)):
//   U  += 2 h^3 U0,  U0 = TT + kappa^2 (TT tr LL - LT LT^T)          (symmetric)
//   V  += 2 h^3 r x (r x A),  A = LL + kappa^2 (LL tr LL - LL LL)   (symmetric)
//   W  += 2 h^3 r x B_i,      B = LT + kappa^2 (LT tr LL - LT LL)
//   Q  += (3 r r^T - r^2) b / 2                                      (symmetric)
//   D  += h^3 (r^T S r - r^2 tr S / 3),  S the stress tensor
// (V_ij = eps_ilm eps_jnp r_l r_n A_mp and W_ij = eps_jlm r_l B_im, written as
// cross products).  28 sums, accumulated per thread and reduced per block with
// compensation; parts[56 * block + 2 q].
// ---------------------------------------------------------------------------
constexpr int kDiag = 28;  // U(6) V(6) W(9) Q(6) D(1)

struct DiagEpi {
    Params p;
    double com[3];
    double acc[kDiag];
    __device__ __forceinline__ static void cross3(const double* a, const double* b, double* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    }
    __device__ __forceinline__ void site(int64_t s, const double* phi, const double (&D)[3][4]) {
        const double k2 = p.c1 * p.c1, m2 = p.c0 * p.c0, vol = p.vol;
        const double sg = phi[0];
        const double pi[3] = {phi[1], phi[2], phi[3]};
        double L[3][3], T[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double ds = D[k][0];
            const double dp[3] = {D[k][1], D[k][2], D[k][3]};
            double cr[3];
            cross3(pi, dp, cr);
#pragma unroll
            for (int a = 0; a < 3; ++a) L[k][a] = sg * dp[a] - pi[a] * ds + cr[a];
        }
        const double pi2 = pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                double e = 0.0;
#pragma unroll
                for (int b = 0; b < 3; ++b) e += double(eps3(i, a, b)) * pi[b];
                T[i][a] = pi[i] * pi[a] - (i == a ? pi2 : 0.0) + sg * e;
            }
        double LL[3][3], TT[3][3], LT[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                LL[i][j] = L[i][0] * L[j][0] + L[i][1] * L[j][1] + L[i][2] * L[j][2];
                TT[i][j] = T[i][0] * T[j][0] + T[i][1] * T[j][1] + T[i][2] * T[j][2];
                LT[i][j] = T[i][0] * L[j][0] + T[i][1] * L[j][1] + T[i][2] * L[j][2];
            }
        const double tr = LL[0][0] + LL[1][1] + LL[2][2];
        // grid point relative to the centre of mass
        const int64_t YZ = (int64_t)p.Y * p.Z;
        const int ix = (int)(s / YZ);
        const int64_t rem = s - (int64_t)ix * YZ;
        const int iy = (int)(rem / p.Z);
        const int iz = (int)(rem - (int64_t)iy * p.Z);
        const double r[3] = {p.hx * ix - com[0], p.hy * iy - com[1], p.hz * iz - com[2]};
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const int si[6] = {0, 0, 0, 1, 1, 2}, sj[6] = {0, 1, 2, 1, 2, 2};
        // U
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int i = si[q], j = sj[q];
            const double u = TT[i][j] + k2 * (TT[i][j] * tr - (LT[i][0] * LT[j][0] + LT[i][1] * LT[j][1] +
                                                                 LT[i][2] * LT[j][2]));
            acc[q] += 2.0 * vol * u;
        }
        // V = r x (r x A): X[:, p] = r x A[:, p], then V[i, :] = r x X[i, :]
        double A[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                A[i][j] = LL[i][j] + k2 * (LL[i][j] * tr - (LL[i][0] * LL[j][0] + LL[i][1] * LL[j][1] +
                                                             LL[i][2] * LL[j][2]));
        double X[3][3];
#pragma unroll
        for (int pp = 0; pp < 3; ++pp) {
            const double col[3] = {A[0][pp], A[1][pp], A[2][pp]};
            double o[3];
            cross3(r, col, o);
#pragma unroll
            for (int i = 0; i < 3; ++i) X[i][pp] = o[i];
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int i = si[q], j = sj[q];
            double o[3];
            cross3(r, X[i], o);
            acc[6 + q] += 2.0 * vol * o[j];
        }
        // W[i, :] = r x B[i, :]
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double Bi[3];
#pragma unroll
            for (int m = 0; m < 3; ++m)
                Bi[m] = LT[i][m] + k2 * (LT[i][m] * tr - (LT[i][0] * LL[m][0] + LT[i][1] * LL[m][1] +
                                                           LT[i][2] * LL[m][2]));
            double o[3];
            cross3(r, Bi, o);
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[12 + 3 * i + j] += 2.0 * vol * o[j];
        }
        // Q
        const double rho = 0.5 * Nuclear<double>::baryon(phi, D, p);
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int i = si[q], j = sj[q];
            acc[21 + q] += (3.0 * r[i] * r[j] - (i == j ? r2 : 0.0)) * rho;
        }
        // D-term integrand: S = LL + kappa^2 (tr LL - LL LL) - e 1
        double quartic = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i + 1; j < 3; ++j) quartic += LL[i][i] * LL[j][j] - LL[i][j] * LL[i][j];
        const double e = 0.5 * tr + 0.5 * k2 * quartic + m2 * (1.0 - sg);
        double rSr = 0.0, trS = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double d2 = LL[i][0] * LL[0][j] + LL[i][1] * LL[1][j] + LL[i][2] * LL[2][j];
                const double Sij = LL[i][j] + k2 * (tr * LL[i][j] - d2) - (i == j ? e : 0.0);
                rSr += r[i] * r[j] * Sij;
                if (i == j) trS += Sij;
            }
        acc[27] += (rSr - r2 * trS / 3.0) * vol;
    }
};

template <class M>
__global__ void __launch_bounds__(M::NTHREADS) k_march_diag(Params p, MarchGrid mg, const double* __restrict__ field,
                                                            double cx, double cy, double cz,
                                                            double* __restrict__ parts) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    __shared__ KSum shk[M::NTHREADS / 32];
    DiagEpi epi;
    epi.p = p;
    epi.com[0] = cx;
    epi.com[1] = cy;
    epi.com[2] = cz;
#pragma unroll
    for (int q = 0; q < kDiag; ++q) epi.acc[q] = 0.0;
    const double* const src[3] = {field, nullptr, nullptr};
    KSum es{0.0, 0.0}, unused{0.0, 0.0};
    for (int t = blockIdx.x; t < mg.count(); t += gridDim.x) {
        int xa, xe, y0, z0;
        march_origin(mg, t, M::BY, xa, xe, y0, z0, p.X);
        march_tile<Nuclear, M, double, 1, 16, DiagEpi, false, double, false>(sm, p, src, 0.0, 0.0, xa, xe, y0, z0,
                                                                             epi, es, unused);
    }
    for (int q = 0; q < kDiag; ++q) {
        const KSum b = block_ksum(KSum{epi.acc[q], 0.0}, shk);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            parts[2 * kDiag * blockIdx.x + 2 * q] = b.s;
            parts[2 * kDiag * blockIdx.x + 2 * q + 1] = b.c;
        }
    }
}

template <template <typename> class Th, class M, typename T>
__global__ void __launch_bounds__(M::NTHREADS) k_march_plain(Params p, MarchGrid mg, const T* __restrict__ field,
                                                             T* __restrict__ eg, T* __restrict__ l) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    PlainEpi<T> epi{eg, l, T(-p.dt)};
    const T* const src[3] = {field, nullptr, nullptr};
    KSum es{0.0, 0.0}, bs{0.0, 0.0};
    for (int t = blockIdx.x; t < mg.count(); t += gridDim.x) {
        int xa, xe, y0, z0;
        march_origin(mg, t, M::BY, xa, xe, y0, z0, p.X);
        march_tile<Th, M, T, 1, false>(sm, p, src, T(0), T(0), xa, xe, y0, z0, epi, es, bs);
    }
}

}  // namespace sky
