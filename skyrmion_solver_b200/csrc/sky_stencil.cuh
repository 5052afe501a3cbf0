// Haloed 3-D tile staging and fourth-order stencils.
//
// A thread block covers a tile of TX x BY x BZ sites (x, y, z) with blockDim =
// (BZ, BY); thread (tz, ty) owns the TX sites (x0 + i, y0 + ty, z0 + tz).  The
// tile plus a 2-site halo on every side is staged in shared memory for all C
// components, so every stencil tap is a shared-memory read.
//
// Stencils restate core/derivatives.py:18-173:
//   first   d_i f  = ( f[-2]/12 - 2 f[-1]/3 + 2 f[+1]/3 - f[+2]/12 ) / h_i
//   second  d_ii f = (-f[-2]/12 + 4 f[-1]/3 - 5 f[0]/2 + 4 f[+1]/3 - f[+2]/12) / h_i^2
//   mixed   d_ij f = sum_{m,n} c_m c_n f[m,n] / (144 h_i h_j),  c = (1,-8,0,8,-1)
// with the reference's masks: pure derivatives are zero unless
// halo <= idx < L-halo on that axis; mixed derivatives are zero unless
// halo < idx < L-halo on both axes (strict on the low side, core/derivatives.py:121).
#pragma once

#include "sky_common.cuh"

namespace sky {

template <int C_, int BZ_, int BY_, int TX_>
struct TileShape {
    static constexpr int C = C_, BZ = BZ_, BY = BY_, TX = TX_;
    static constexpr int HZ = BZ + 4, HY = BY + 4, HX = TX + 4;
    static constexpr int PLANE = HY * HZ;
    static constexpr int VOL = HX * PLANE;
    static constexpr int NTHREADS = BZ * BY;
    template <typename T>
    static constexpr size_t smem_bytes() { return size_t(C) * VOL * sizeof(T); }
};

// Per-axis stencil validity for one site (reference masks).
struct Mask {
    bool px, py, pz;  // pure (first / second) derivative
    bool mx, my, mz;  // mixed derivative participation
};

__device__ __forceinline__ Mask site_mask(const Params& p, int x, int y, int z) {
    Mask m;
    const int h = p.halo;
    m.px = (x >= h) && (x < p.X - h);
    m.py = (y >= h) && (y < p.Y - h);
    m.pz = (z >= h) && (z < p.Z - h);
    m.mx = (x > h) && (x < p.X - h);
    m.my = (y > h) && (y < p.Y - h);
    m.mz = (z > h) && (z < p.Z - h);
    return m;
}

// Load the haloed tile of `ncomp` components of a reference-layout buffer
// (component stride N) into shared memory; points outside the lattice read 0.
// Element type of the source S may differ from the shared-memory type T.
template <class Shape, typename T, typename S>
__device__ __forceinline__ void load_tile(T* __restrict__ sm, const S* __restrict__ src, const Params& p, int64_t N,
                                          int x0, int y0, int z0, int ncomp = Shape::C) {
    const int tid = threadIdx.x + Shape::BZ * threadIdx.y;
    const int64_t YZ = (int64_t)p.Y * p.Z;
    // one "row" = HZ consecutive z values for fixed (c, xx, yy)
    const int nrows = ncomp * Shape::HX * Shape::HY;
    for (int row = threadIdx.y; row < nrows; row += Shape::BY) {
        const int c = row / (Shape::HX * Shape::HY);
        const int r = row - c * (Shape::HX * Shape::HY);
        const int xx = r / Shape::HY;
        const int yy = r - xx * Shape::HY;
        const int gx = x0 - 2 + xx;
        const int gy = y0 - 2 + yy;
        const bool rowok = (gx >= 0) && (gx < p.X) && (gy >= 0) && (gy < p.Y);
        const S* base = src + (int64_t)c * N + gx * YZ + (int64_t)gy * p.Z;
        T* dst = sm + c * Shape::VOL + xx * Shape::PLANE + yy * Shape::HZ;
        for (int zz = threadIdx.x; zz < Shape::HZ; zz += Shape::BZ) {
            const int gz = z0 - 2 + zz;
            T v = T(0);
            if (rowok && gz >= 0 && gz < p.Z) v = T(base[gz]);
            dst[zz] = v;
        }
    }
    (void)tid;
}

// Stencil coefficients, pre-divided by the spacing.
template <typename T>
struct StencilCoef {
    T d1a[3], d1b[3];      // first:  d1a*(f+1 - f-1) + d1b*(f+2 - f-2)  ... see below
    T d2a[3], d2b[3], d2c[3];
    T mix[3];              // 1 / (144 h_i h_j) for xy, xz, yz
    __device__ __forceinline__ void init(const Params& p) {
        const double h[3] = {p.hx, p.hy, p.hz};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            d1a[i] = T((2.0 / 3.0) / h[i]);
            d1b[i] = T((1.0 / 12.0) / h[i]);
            d2a[i] = T((4.0 / 3.0) / (h[i] * h[i]));
            d2b[i] = T((1.0 / 12.0) / (h[i] * h[i]));
            d2c[i] = T((5.0 / 2.0) / (h[i] * h[i]));
        }
        mix[0] = T(1.0 / (144.0 * p.hx * p.hy));
        mix[1] = T(1.0 / (144.0 * p.hx * p.hz));
        mix[2] = T(1.0 / (144.0 * p.hy * p.hz));
    }
};

// 16-tap mixed stencil sum over the (a, b) plane: sum_{m,n in {-2,-1,1,2}} c_m c_n f(m, n)
// with c = (1, -8, 8, -1) for offsets (-2, -1, 1, 2).
template <typename T>
__device__ __forceinline__ T mixed16(const T* __restrict__ f, int sa, int sb) {
    // inner differences along b for each a offset
    const int offs[4] = {-2, -1, 1, 2};
    const T cs[4] = {T(1), T(-8), T(8), T(-1)};
    T acc = T(0);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const T* r = f + offs[m] * sa;
        const T inner = (r[-2 * sb] - r[2 * sb]) + T(8) * (r[sb] - r[-sb]);
        acc += cs[m] * inner;
    }
    return acc;
}

// All first and second derivatives of component c at the site whose tile
// coordinate is (xx, yy, zz) (interior offsets, i.e. including +2 halo).
template <class Shape, typename T, int CD>
__device__ __forceinline__ void site_derivs(const T* __restrict__ sm, int c, int xx, int yy, int zz,
                                            const StencilCoef<T>& k, const Mask& m, T (&D)[3][CD],
                                            T (&Sd)[6][CD], T& f0out) {
    const T* f = sm + c * Shape::VOL + xx * Shape::PLANE + yy * Shape::HZ + zz;
    const int sx = Shape::PLANE, sy = Shape::HZ, sz = 1;
    const T f0 = f[0];
    f0out = f0;
    const int st[3] = {sx, sy, sz};
    const bool pm[3] = {m.px, m.py, m.pz};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T fm2 = f[-2 * st[i]], fm1 = f[-st[i]], fp1 = f[st[i]], fp2 = f[2 * st[i]];
        const T d1 = k.d1a[i] * (fp1 - fm1) - k.d1b[i] * (fp2 - fm2);
        const T d2 = k.d2a[i] * (fp1 + fm1) - k.d2b[i] * (fp2 + fm2) - k.d2c[i] * f0;
        D[i][c] = pm[i] ? d1 : T(0);
        Sd[i][c] = pm[i] ? d2 : T(0);
    }
    Sd[3][c] = (m.mx && m.my) ? k.mix[0] * mixed16<T>(f, sx, sy) : T(0);
    Sd[4][c] = (m.mx && m.mz) ? k.mix[1] * mixed16<T>(f, sx, sz) : T(0);
    Sd[5][c] = (m.my && m.mz) ? k.mix[2] * mixed16<T>(f, sy, sz) : T(0);
}

// First derivatives only (energy / baryon kernels).
template <class Shape, typename T, int CD>
__device__ __forceinline__ void site_first(const T* __restrict__ sm, int c, int xx, int yy, int zz,
                                           const StencilCoef<T>& k, const Mask& m, T (&D)[3][CD], T& f0out) {
    const T* f = sm + c * Shape::VOL + xx * Shape::PLANE + yy * Shape::HZ + zz;
    const int st[3] = {Shape::PLANE, Shape::HZ, 1};
    const bool pm[3] = {m.px, m.py, m.pz};
    f0out = f[0];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T d1 = k.d1a[i] * (f[st[i]] - f[-st[i]]) - k.d1b[i] * (f[2 * st[i]] - f[-2 * st[i]]);
        D[i][c] = pm[i] ? d1 : T(0);
    }
}

}  // namespace sky
