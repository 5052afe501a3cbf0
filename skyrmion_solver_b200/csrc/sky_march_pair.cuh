// Z-pair marching tile: the FP32 engine stages with two adjacent z-sites per thread.
//
// The tile, the haloed plane layout, the TMA plane pipeline and the stage input
// X = F + a V + b L are those of march_tile (sky_march.cuh); only the thread
// mapping and the arithmetic differ.  A block of 16 x BY threads covers the
// 32 x BY (z, y) tile; thread (tx, ty) owns the sites z0 + 2 tx and z0 + 2 tx + 1
// of row y0 + ty.  Every stencil tap is one 8-byte shared-memory load of the two
// sites' values, and every FP32 operation of the stencils and of the theory's
// point arithmetic is one packed FP32x2 instruction for both sites (sky_pair.cuh).
// The FP64 energy density of stage 1 and the FP64 update of stage 4 stay per site.
//
// For theories whose gradient needs no mixed second derivatives (Th<T>::kMixed is
// false): the mixed derivatives are not formed.
#pragma once

#include "sky_march.cuh"
#include "sky_pair.cuh"

namespace sky {

template <class M>
struct PairShape {
    static constexpr int TZ = M::BZ / 2;            // threads along z
    static constexpr int NT = TZ * M::BY;           // threads per block
};

// Stencil derivatives of one component for the two sites: first derivatives D[i]
// and pure second derivatives S[i] (i = x, y, z), with the reference's masks per site.
// Pointers address the pair's first site in the ring slots of planes x-2 .. x+2.
template <class M>
__device__ __forceinline__ void pair_derivs(const float* Pm2, const float* Pm1, const float* P0, const float* Pp1,
                                            const float* Pp2, const StencilCoef<float>& k, const Mask& m0,
                                            const Mask& m1, P2& f0, P2 (&D)[3], P2 (&S)[3]) {
    const P2 d1a[3] = {P2(k.d1a[0]), P2(k.d1a[1]), P2(k.d1a[2])};
    const P2 d1b[3] = {P2(k.d1b[0]), P2(k.d1b[1]), P2(k.d1b[2])};
    const P2 d2a[3] = {P2(k.d2a[0]), P2(k.d2a[1]), P2(k.d2a[2])};
    const P2 d2b[3] = {P2(k.d2b[0]), P2(k.d2b[1]), P2(k.d2b[2])};
    const P2 d2c[3] = {P2(k.d2c[0]), P2(k.d2c[1]), P2(k.d2c[2])};
    f0 = p2_load(P0);
    {
        const P2 fm2 = p2_load(Pm2), fm1 = p2_load(Pm1), fp1 = p2_load(Pp1), fp2 = p2_load(Pp2);
        D[0] = p2_mask(d1a[0] * (fp1 - fm1) - d1b[0] * (fp2 - fm2), m0.px, m1.px);
        S[0] = p2_mask(d2a[0] * (fp1 + fm1) - d2b[0] * (fp2 + fm2) - d2c[0] * f0, m0.px, m1.px);
    }
    {
        const P2 fm2 = p2_load(P0 - 2 * M::HZ), fm1 = p2_load(P0 - M::HZ), fp1 = p2_load(P0 + M::HZ),
                 fp2 = p2_load(P0 + 2 * M::HZ);
        D[1] = p2_mask(d1a[1] * (fp1 - fm1) - d1b[1] * (fp2 - fm2), m0.py, m1.py);
        S[1] = p2_mask(d2a[1] * (fp1 + fm1) - d2b[1] * (fp2 + fm2) - d2c[1] * f0, m0.py, m1.py);
    }
    {
        // z - 2 .. z + 3 as three aligned pairs: (z-2, z-1), (z, z+1) = f0, (z+2, z+3)
        const P2 a = p2_load(P0 - 2), c = p2_load(P0 + 2);
        const P2 fm2 = a, fp2 = c;
        const P2 fm1(a.v.y, f0.v.x), fp1(f0.v.y, c.v.x);
        D[2] = p2_mask(d1a[2] * (fp1 - fm1) - d1b[2] * (fp2 - fm2), m0.pz, m1.pz);
        S[2] = p2_mask(d2a[2] * (fp1 + fm1) - d2b[2] * (fp2 + fm2) - d2c[2] * f0, m0.pz, m1.pz);
    }
}

// One tile of an FP32 engine stage with z-pairs (TMA staging; see march_tile for
// the pipeline and the meaning of NSRC, DENS, LO).  The epilogue is called once per
// site with lane l = 0, 1: epi(s, N, phi, g, l).
template <template <typename> class Th, class M, int NSRC, int DENS, class Epi, bool LO = false>
__device__ __forceinline__ bool march_tile_pair(float* __restrict__ sm, const Params& p, float a, float b, int xa,
                                                int xe, int y0, int z0, Epi& epi, KSum& esum, KSum& bsum,
                                                TmaTile* tma) {
    using T = float;
    constexpr int C = M::C;
    constexpr int NT = PairShape<M>::NT;
    static_assert(M::WIDE, "z-pair tiles use the wide-row plane layout");
    static_assert(!Th<float>::kMixed, "z-pair tiles form no mixed second derivatives");
    static_assert(!LO || (DENS != 0 && NSRC == 2), "low-part ring only for the stage-1 density");
    constexpr bool DIRECT = (NSRC == 1 || LO);
    constexpr int LA = M::template tma_lookahead<T>(NSRC, LO);
    constexpr int R = M::RING + LA;
    T* ring = sm;
    T* stage = sm + R * M::SLOT;
    T* ring_lo = sm + R * M::SLOT;

    const int64_t N = n_sites(p);
    const int64_t YZ = (int64_t)p.Y * p.Z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int y = y0 + ty, z = z0 + 2 * tx;
    const bool own0 = (y < p.Y) && (z < p.Z), own1 = (y < p.Y) && (z + 1 < p.Z);
    StencilCoef<T> k;
    k.init(p);
    const int q0 = xa - 2, q1 = xe + 1;
    const int lofs = (ty + 2) * M::HZ + (2 * tx + M::ZOFF);
    const int tid0 = threadIdx.x + PairShape<M>::TZ * threadIdx.y;
    auto issue_tma = [&](int qq, int dslot, int nb) {
        if (tid0 != 0) return;
        constexpr uint32_t box = uint32_t(M::SLOT * sizeof(T));
        uint32_t n = 1;
#pragma unroll
        for (int kk = 1; kk < NSRC; ++kk) n += tma->map[kk] != nullptr ? 1u : 0u;
        uint64_t* bar = tma->bar + nb;
        T* stg = stage + nb * (NSRC - 1) * M::SLOT;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, n * box);
        const int zc = z0 - M::ZOFF, yc = y0 - 2;
        tma_load_plane(ring + dslot * M::SLOT, tma->map[0], zc, yc, qq, 0, bar);
#pragma unroll
        for (int kk = 1; kk < NSRC; ++kk) {
            if (tma->map[kk] == nullptr) continue;
            T* dst = LO ? ring_lo + dslot * M::SLOT : stg + (kk - 1) * M::SLOT;
            tma_load_plane(dst, tma->map[kk], zc, yc, qq, 0, bar);
        }
    };
    __syncthreads();
    issue_tma(q0, 0, 0);
    if (LA > 1 && q0 + 1 <= q1) issue_tma(q0 + 1, 1, 1);
    int slot = 0;
    for (int q = q0; q <= q1; ++q) {
        const int nb = LA > 1 ? ((q - q0) & 1) : 0;
        const bool ok = mbar_wait_bounded(tma->bar + nb, (tma->phase >> nb) & 1u);
        tma->phase ^= 1u << nb;
        if constexpr (!DIRECT) {
            constexpr int NV = M::SLOT / 4;
            float4* dstv = reinterpret_cast<float4*>(ring + slot * M::SLOT);
            const float4* s1 = reinterpret_cast<const float4*>(stage) + nb * (NSRC - 1) * NV;
            const float4* s2 = s1 + NV;
            const bool h1 = tma->map[1] != nullptr;
            const bool h2 = NSRC > 2 && tma->map[2] != nullptr;
            if (h1 || h2) {
                const float2 av = make_float2(a, a), bv = make_float2(b, b);
                for (int i = tid0; i < NV; i += NT) {
                    float4 v = dstv[i];
                    float2 lo2 = make_float2(v.x, v.y), hi2 = make_float2(v.z, v.w);
                    if (h1) {
                        const float4 u = s1[i];
                        lo2 = __ffma2_rn(av, make_float2(u.x, u.y), lo2);
                        hi2 = __ffma2_rn(av, make_float2(u.z, u.w), hi2);
                    }
                    if (h2) {
                        const float4 u = s2[i];
                        lo2 = __ffma2_rn(bv, make_float2(u.x, u.y), lo2);
                        hi2 = __ffma2_rn(bv, make_float2(u.z, u.w), hi2);
                    }
                    dstv[i] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
                }
            }
        }
        fence_proxy_async_smem();
        if (__syncthreads_or(ok ? 0 : 1)) {
            if (tid0 == 0) {
                atomicOr(tma->status, 1);
                for (int kk = 0; kk < LA; ++kk) mbar_wait_bounded(tma->bar + kk, (tma->phase >> kk) & 1u);
            }
            return false;
        }
        if (q + LA <= q1) issue_tma(q + LA, (slot + LA) % R, nb);
        if constexpr (HasPlaneBegin<Epi>::value) {
            if (q - 2 >= xa) epi.plane_begin(q - 2);
        }
        const int x = q - 2;
        if (x >= xa && own0) {
            const T* Pm2 = ring + ((slot + R - 4) % R) * M::SLOT + lofs;
            const T* Pm1 = ring + ((slot + R - 3) % R) * M::SLOT + lofs;
            const T* P0 = ring + ((slot + R - 2) % R) * M::SLOT + lofs;
            const T* Pp1 = ring + ((slot + R - 1) % R) * M::SLOT + lofs;
            const T* Pp2 = ring + slot * M::SLOT + lofs;
            const Mask mk0 = site_mask(p, x, y, z), mk1 = site_mask(p, x, y, z + 1);
            const int64_t s = (int64_t)x * YZ + (int64_t)y * p.Z + z;
            const int64_t nx = x + 1 < xe ? s + YZ : int64_t(-1);
            if constexpr (HasBeginSite<Epi>::value) {
                epi.begin_site(s, N, nx, 0);
                if (own1) epi.begin_site(s + 1, N, nx >= 0 ? nx + 1 : int64_t(-1), 1);
            }
            P2 phi[C], D[3][C], Sd[6][C], g[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int co = c * M::PLANE;
                P2 d[3], sd[3];
                pair_derivs<M>(Pm2 + co, Pm1 + co, P0 + co, Pp1 + co, Pp2 + co, k, mk0, mk1, phi[c], d, sd);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    D[i][c] = d[i];
                    Sd[i][c] = sd[i];
                    Sd[3 + i][c] = P2(0.0f);  // mixed derivatives: not needed by the theory
                }
            }
            Th<P2>::gradient(phi, D, Sd, p, g);
            [[maybe_unused]] P2 b2 = P2(0.0f);
            if constexpr (DENS != 0) b2 = Th<P2>::baryon(phi, D, p);
            // the epilogue per site
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if (l == 1 && !own1) break;
                float ph[C], gg[C];
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    ph[c] = l ? phi[c].v.y : phi[c].v.x;
                    gg[c] = l ? g[c].v.y : g[c].v.x;
                }
                epi(s + l, N, ph, gg, l);
            }
            if constexpr (DENS != 0) {
                // FP64 energy density of each site (as march_tile's DENS block, per lane) and the
                // FP32 baryon density from the pair derivatives
                constexpr int CT = Th<double>::C;
                StencilCoef<double> kd;
                kd.init(p);
                const ptrdiff_t dlo = ring_lo - ring;
#pragma unroll
                for (int l = 0; l < 2; ++l) {
                    if (l == 1 && !own1) break;
                    const Mask& mk = l ? mk1 : mk0;
                    double phd[CT], Dd[3][CT];
                    auto dif = [&](const T* u, const T* v) -> double {
                        if constexpr (LO) {
                            const T ua = u[0], vb = -v[0];
                            const T ss = ua + vb, bb = ss - ua;
                            const T e = (ua - (ss - bb)) + (vb - bb);
                            return double(ss) + double(e + (u[dlo] - v[dlo]));
                        } else {
                            return double(u[0]) - double(v[0]);
                        }
                    };
#pragma unroll
                    for (int c = 0; c < C; ++c) {
                        const int co = c * M::PLANE + l;
                        const T* f = P0 + co;
                        phd[c] = LO ? double(f[0]) + double(f[dlo]) : double(f[0]);
                        const double xd = dif(Pp1 + co, Pm1 + co), xd2 = dif(Pp2 + co, Pm2 + co);
                        const double yd = dif(f + M::HZ, f - M::HZ), yd2 = dif(f + 2 * M::HZ, f - 2 * M::HZ);
                        const double zd = dif(f + 1, f - 1), zd2 = dif(f + 2, f - 2);
                        Dd[0][c] = mk.px ? kd.d1a[0] * xd - kd.d1b[0] * xd2 : 0.0;
                        Dd[1][c] = mk.py ? kd.d1a[1] * yd - kd.d1b[1] * yd2 : 0.0;
                        Dd[2][c] = mk.pz ? kd.d1a[2] * zd - kd.d1b[2] * zd2 : 0.0;
                    }
                    ksum_add(esum, Th<double>::energy(phd, Dd, p));
                    ksum_add(bsum, double(l ? b2.v.y : b2.v.x));
                }
            }
        }
        slot = (slot + 1) % R;
    }
    return true;
}

}  // namespace sky
