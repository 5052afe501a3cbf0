// Lattice kernels shared by the reference-layout C ABI and the resident engine.
//
// Storage type S (what lives in HBM) and arithmetic type T (what the stencil
// and the point physics compute in) are template parameters: S = T = double is
// the plain FP64 path; S = T = float is the mixed-precision engine's stage
// arithmetic.  Energies and baryon numbers are always evaluated in FP64 and
// summed with compensated FP64 accumulation.
#pragma once

#include "sky_common.cuh"
#include "sky_stencil.cuh"
#include "sky_theories.cuh"

namespace sky {

// Largest grid of the tile-looping reduction kernels; bounds the scratch the
// reductions need (2 doubles per block + result + counter).
constexpr int kMaxRedBlocks = 1184;  // 148 SMs x 8
constexpr int64_t kScratchDoubles = 2 * kMaxRedBlocks + 8;

// Tile shapes per (theory, arithmetic type).  Shared memory per block is
// C * (TX+4)(BY+4)(BZ+4) * sizeof(T).
template <int C, typename T>
struct GradTile {
    using type = TileShape<C, 32, 8, 4>;
};
template <>
struct GradTile<13, double> {
    using type = TileShape<13, 32, 4, 1>;
};
template <>
struct GradTile<13, float> {
    using type = TileShape<13, 32, 4, 2>;
};
template <int C>
struct DensTile {  // first derivatives only, FP64 arithmetic
    using type = TileShape<C, 32, (C > 5 ? 4 : 8), (C > 5 ? 1 : 2)>;
};

struct TileGrid {
    int nz, ny, nx;
    __host__ __device__ int count() const { return nz * ny * nx; }
};

template <class Shape>
__host__ __device__ inline TileGrid tile_grid(const Params& p) {
    TileGrid g;
    g.nz = (p.Z + Shape::BZ - 1) / Shape::BZ;
    g.ny = (p.Y + Shape::BY - 1) / Shape::BY;
    g.nx = (p.X + Shape::TX - 1) / Shape::TX;
    return g;
}

__device__ __forceinline__ void tile_origin(const TileGrid& g, int t, int bz, int by, int tx, int& x0, int& y0,
                                            int& z0) {
    const int iz = t % g.nz;
    const int r = t / g.nz;
    const int iy = r % g.ny;
    const int ix = r / g.ny;
    z0 = iz * bz;
    y0 = iy * by;
    x0 = ix * tx;
}

// ---------------------------------------------------------------------------
// Energy gradient: EG = projected gradient of `field`, l = -dt * EG.
// One tile per block iteration; grid-stride over tiles.
// ---------------------------------------------------------------------------
template <template <typename> class Th, class Shape, typename T, typename S>
__global__ void __launch_bounds__(Shape::NTHREADS) k_gradient(Params p, const S* __restrict__ field,
                                                              S* __restrict__ eg, S* __restrict__ lout) {
    constexpr int C = Th<T>::C;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int64_t N = n_sites(p);
    const TileGrid tg = tile_grid<Shape>(p);
    StencilCoef<T> k;
    k.init(p);
    const T mdt = T(-p.dt);
    for (int t = blockIdx.x; t < tg.count(); t += gridDim.x) {
        int x0, y0, z0;
        tile_origin(tg, t, Shape::BZ, Shape::BY, Shape::TX, x0, y0, z0);
        __syncthreads();
        load_tile<Shape>(sm, field, p, N, x0, y0, z0);
        __syncthreads();
        const int z = z0 + threadIdx.x, y = y0 + threadIdx.y;
        if (z >= p.Z || y >= p.Y) continue;
#pragma unroll 1
        for (int i = 0; i < Shape::TX; ++i) {
            const int x = x0 + i;
            if (x >= p.X) break;
            const Mask m = site_mask(p, x, y, z);
            T phi[C], D[3][C], Sd[6][C], g[C];
#pragma unroll
            for (int c = 0; c < C; ++c)
                site_derivs<Shape, T, C>(sm, c, i + 2, threadIdx.y + 2, threadIdx.x + 2, k, m, D, Sd, phi[c]);
            Th<T>::gradient(phi, D, Sd, p, g);
            const int64_t s = ((int64_t)x * p.Y + y) * p.Z + z;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                eg[c * N + s] = S(g[c]);
                lout[c * N + s] = S(mdt * g[c]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Last-block-done finish of a per-block KSum: deterministic (fixed partition
// and fixed combine order for a given grid size).
// scratch layout: [0, 2*gridDim) partial (s, c); [2*kMaxRedBlocks] result;
// [2*kMaxRedBlocks + 1] counter (uint32 in the low bytes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void finish_ksum(KSum v, double* __restrict__ scratch, double* __restrict__ out_dev,
                                            KSum* shk) {
    __shared__ bool am_last;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    KSum b = block_ksum(v, shk);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + 2 * kMaxRedBlocks + 1);
    if (tid == 0) {
        scratch[2 * blockIdx.x] = b.s;
        scratch[2 * blockIdx.x + 1] = b.c;
        __threadfence();
        const unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const int nthreads = blockDim.x * blockDim.y;
    KSum acc{0.0, 0.0};
    for (int i = tid; i < (int)gridDim.x; i += nthreads) {
        KSum o{__ldcg(scratch + 2 * i), __ldcg(scratch + 2 * i + 1)};
        ksum_merge(acc, o);
    }
    KSum r = block_ksum(acc, shk);
    if (tid == 0) {
        const double res = r.s + r.c;
        scratch[2 * kMaxRedBlocks] = res;
        if (out_dev) *out_dev = res;
        *counter = 0u;
    }
}

// Block maxima, then the last block to finish reduces them; the result, times `sign`,
// goes to scratch[2 kMaxRedBlocks] and *out_dev (sign -1 turns a maximum of negated
// values into a minimum).
__device__ __forceinline__ void finish_max(double v, double* __restrict__ scratch, double* __restrict__ out_dev,
                                           double* shm, double sign = 1.0) {
    __shared__ bool am_last;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    double b = block_max(v, shm);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + 2 * kMaxRedBlocks + 1);
    if (tid == 0) {
        scratch[2 * blockIdx.x] = b;
        __threadfence();
        const unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    const int nthreads = blockDim.x * blockDim.y;
    double acc = -1.0e300;
    for (int i = tid; i < (int)gridDim.x; i += nthreads) acc = fmax(acc, __ldcg(scratch + 2 * i));
    const double r = sign * block_max(acc, shm);
    if (tid == 0) {
        scratch[2 * kMaxRedBlocks] = r;
        if (out_dev) *out_dev = r;
        *counter = 0u;
    }
}

// ---------------------------------------------------------------------------
// Per-site energy (MODE 0) or baryon (MODE 1) density in FP64 from a field of
// storage type S; optionally written to `dens` and/or summed into scratch.
// ---------------------------------------------------------------------------
template <template <typename> class Th, class Shape, int MODE, typename S>
__global__ void __launch_bounds__(Shape::NTHREADS) k_density(Params p, const S* __restrict__ field,
                                                             double* __restrict__ dens, double* __restrict__ scratch,
                                                             double* __restrict__ out_dev) {
    constexpr int C = Th<double>::C;
    constexpr int CL = (MODE == 0) ? C : 4;  // baryon density needs phi0..3 only
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    __shared__ KSum shk[32];
    const int64_t N = n_sites(p);
    const TileGrid tg = tile_grid<Shape>(p);
    StencilCoef<double> k;
    k.init(p);
    KSum acc{0.0, 0.0};
    for (int t = blockIdx.x; t < tg.count(); t += gridDim.x) {
        int x0, y0, z0;
        tile_origin(tg, t, Shape::BZ, Shape::BY, Shape::TX, x0, y0, z0);
        __syncthreads();
        load_tile<Shape>(sm, field, p, N, x0, y0, z0, CL);
        __syncthreads();
        const int z = z0 + threadIdx.x, y = y0 + threadIdx.y;
        if (z >= p.Z || y >= p.Y) continue;
        for (int i = 0; i < Shape::TX; ++i) {
            const int x = x0 + i;
            if (x >= p.X) break;
            const Mask m = site_mask(p, x, y, z);
            double phi[C], D[3][C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (c < CL) {
                    site_first<Shape, double, C>(sm, c, i + 2, threadIdx.y + 2, threadIdx.x + 2, k, m, D, phi[c]);
                } else {
                    phi[c] = 0.0;
                    D[0][c] = D[1][c] = D[2][c] = 0.0;
                }
            }
            const double e = (MODE == 0) ? Th<double>::energy(phi, D, p) : Th<double>::baryon(phi, D, p);
            const int64_t s = ((int64_t)x * p.Y + y) * p.Z + z;
            if (dens) dens[s] = e;
            ksum_add(acc, e);
        }
    }
    if (scratch) finish_ksum(acc, scratch, out_dev, shk);
}

}  // namespace sky
