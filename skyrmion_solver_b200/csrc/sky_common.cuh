// Shared definitions for the skyrmion_b200 lattice engine (sm_100a).
//
// Lattice layout (the reference's flattened SoA, skyrmion_solver core/utils.py:21-48):
//   field[a * N + x * Y * Z + y * Z + z], z fastest, N = X * Y * Z.
// Every kernel in this library maps threadIdx.x to z so warp accesses are
// contiguous in memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/skyrmion_b200.h"

namespace sky {

// Runtime description of one lattice instance, unpacked from the reference's
// positional p_i / p_f arrays (core/params.py:227-267 and th/*/params.py).
struct Params {
    int X, Y, Z;        // p_i[0..2]
    int halo;           // p_i[3]
    int C;              // p_i[5]: number of field components
    int nsky;           // components normalised / projected (p_i[5], p_i[11] or 4)
    int killkinen;      // p_i[8]
    int unit_length;    // p_i[10]
    double hx, hy, hz;  // p_f[3..5]
    double vol;         // p_f[6] (cell volume)
    double dt;          // p_f[7]
    double c0, c1, c2;  // theory couplings (see sky_pack_params)
};

__host__ __device__ inline int64_t n_sites(const Params& p) {
    return (int64_t)p.X * p.Y * p.Z;
}

// ---------------------------------------------------------------------------
// Compensated (Neumaier / TwoSum) FP64 accumulation.  Used for every energy,
// baryon-number and arrest reduction so the result does not depend on the
// grid size's rounding drift.
// ---------------------------------------------------------------------------
struct KSum {
    double s, c;
};

__device__ __forceinline__ void ksum_add(KSum& a, double v) {
    double t = a.s + v;
    double e = (fabs(a.s) >= fabs(v)) ? ((a.s - t) + v) : ((v - t) + a.s);
    a.s = t;
    a.c += e;
}

__device__ __forceinline__ void ksum_merge(KSum& a, const KSum& b) {
    ksum_add(a, b.s);
    a.c += b.c;
}

__device__ __forceinline__ KSum ksum_shfl_down(const KSum& a, int off) {
    KSum r;
    r.s = __shfl_down_sync(0xffffffffu, a.s, off);
    r.c = __shfl_down_sync(0xffffffffu, a.c, off);
    return r;
}

// Block-wide deterministic reduction of a KSum (fixed tree order); result valid
// in thread 0.  `sh` must hold blockDim/32 entries.
__device__ __forceinline__ KSum block_ksum(KSum v, KSum* sh) {
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int warp = tid >> 5;
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    // lane index within the warp follows the linear thread id
    (void)lane;
    const int l = tid & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        KSum o = ksum_shfl_down(v, off);
        if (l + off < 32) ksum_merge(v, o);
    }
    if (l == 0) sh[warp] = v;
    __syncthreads();
    KSum r{0.0, 0.0};
    if (tid == 0) {
        const int nw = (nthreads + 31) >> 5;
        for (int w = 0; w < nw; ++w) ksum_merge(r, sh[w]);
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int l = tid & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double o = __shfl_down_sync(0xffffffffu, v, off);
        if (l + off < 32) v = fmax(v, o);
    }
    if (l == 0) sh[tid >> 5] = v;
    __syncthreads();
    double r = -1.0e300;
    if (tid == 0) {
        const int nw = (nthreads + 31) >> 5;
        for (int w = 0; w < nw; ++w) r = fmax(r, sh[w]);
    }
    __syncthreads();
    return r;
}

}  // namespace sky
