// Resident engine kernels: the arrested-Newton / RK4 step of
// core/integrator.py:284-410 as fused stage launches plus a small control
// launch, for a batch of lattice instances at once.
//
// With k1 = dt V, k2 = dt (V + l1/2), k3 = dt (V + l2/2), k4 = dt (V + l3) the
// stage inputs of the reference schedule are
//   X1 = F,  X2 = F + (dt/2) V,  X3 = F + (dt/2)(V + l1/2),  X4 = F + dt (V + l2/2)
// and the update is
//   V' = V + (l1 + 2 l2 + 2 l3 + l4)/6,   F' = F + dt (V + (l1 + l2 + l3)/6)
// followed by the theory's normalisation of phi and projection of V'
// (core/integrator.py:163-175).  Stage s builds X_s for its haloed tile on the
// fly from F, V and the previous slope and writes only l_s; stage 4 applies the
// update into the other half of a ping-pong pair.
//
// One step is: stage 2, stage 3, stage 4 (+ update; its tail advances each instance),
// [the defect refresh,] stage 1 (its tail runs each instance's control).
// Stage 1 runs on the freshly updated field, so besides l1 (needed by the next
// step) it evaluates that field's energy and baryon density in FP64; the
// control launch reduces them (compensated, fixed order), records the step's
// (energy, err) exactly as do_arrested_newton_flow returns them, and takes the
// arrest decision for the next step: the velocity is treated as zero when
// killkinen is set and the energy rose (core/integrator.py:403-407).
#pragma once

#include "sky_kernels.cuh"
#include "sky_march.cuh"
#include "sky_march_pair.cuh"

namespace sky {

// Per-step statistics written by the control launch: record n describes the
// field after n steps (record 0: the admitted field).
struct StepStats {
    double energy;      // E after step n (FP64, compensated)
    double baryon;      // B after step n
    double err;         // signed max of step n's stage-4 gradient (reference `err`)
    double gabs;        // max |g| of step n's stage-4 gradient
    int arrested;       // velocity treated as zero in step n+1
    int step;           // n
    double kinetic;     // (1/2) h^3 sum |V'|^2 of the velocity step n produced (before any arrest)
    int status;         // the engine's error word when the record was written (0: no error)
    int reserved;
};

// Roles of an instance's TMA plane maps (InstDesc::tm).
// Plane maps (tm) cover a tile's haloed plane, centre maps (tmc) its BY x 32 sites
// (the stage-4 update's operands, which need no halo); the centre maps add the
// defect correction at kMapDlt.
enum { kMapF = 0, kMapFlo = 2, kMapV = 4, kMapL = 6, kNumMaps = 9, kMapDlt = 9, kNumCentreMaps = 10 };

// Device-resident state of one instance.
template <typename S>
struct InstDesc {
    TmaMap tm[kNumMaps];  // plane maps of F[0..1], Flo[0..1], V[0..1], L[0..2] (when tma is set)
    TmaMap tmc[kNumCentreMaps];  // centre maps of the same arrays and of Dlt (when tma is set)
    int tma;              // the stage kernels stage this instance's planes with TMA
    int* status;          // the engine's error word (bit 0: a wait for a TMA copy gave up)
    Params p;
    S* F[2];           // ping-pong field
    S* Flo[2];         // ping-pong low parts of a compensated FP32 field (null otherwise)
    S* Dlt;            // defect correction g64 - g32 of a defect-corrected FP32 instance (null otherwise)
    S* V[2];           // ping-pong velocity
    S* L[3];           // stage slopes l1, l2, l3
    KSum* epart;       // per-tile energy partials (stage 1)
    KSum* bpart;       // per-tile baryon partials (stage 1)
    double* gpart;     // per-tile [signed max, abs max of stage-4 g, kinetic KSum (s, c)] (4 doubles / tile)
    StepStats* stats;  // ring of per-step records
    int stats_cap;
    int tile_begin;    // first global tile index of this instance
    int ntiles;
    int tiles_nz, tiles_ny, tiles_nx;
    int xc;            // x-chunk of the marching kernels
    // control state (device-updated)
    double e_prev;     // energy entering the previous step
    int step;          // steps taken
    int arrested;      // arrest flag for the current step
    int active;        // 0 = skip (retired / paused)
    int cur;           // which half of the F / V ping-pong pairs is current
    int refresh;       // this step's stage 1 refreshes the defect correction
    int refresh_period;  // steps between refreshes of the defect correction
};

// RK4 update of one site (core/integrator.py:163-175): V' = V + (l1 + 2 l2 + 2 l3 + l4)/6,
// F' = F + (k1 + 2 k2 + 2 k3 + k4)/6 = F + dt (V + (l1 + l2 + l3)/6), then the theory's
// normalisation of the first nsky components and projection of V' orthogonal to them.
// With a compensated field (comp) F is the unevaluated sum hi + lo of two FP32
// values: the update, the normalisation and the projection run in FP64 and the result is
// split back into hi + lo, so increments far below one FP32 ulp of F still accumulate.
template <typename T, typename S, int C>
__device__ __forceinline__ void finalize_vals(int64_t s, int64_t N, const T (&f0)[C], const T (&flo)[C], bool comp,
                                              const T (&v0)[C], const T (&l1)[C], const T (&l2)[C],
                                              const T (&l3)[C], const T (&g)[C], T dtt, int nsky, int unit_length,
                                              S* __restrict__ Fo, S* __restrict__ Flo_out, S* __restrict__ Vo,
                                              T& v2) {
    T vv[C], inc[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const T l4 = -dtt * g[c];
        vv[c] = v0[c] + (l1[c] + T(2) * l2[c] + T(2) * l3[c] + l4) * T(1.0 / 6.0);
        inc[c] = dtt * (v0[c] + (l1[c] + l2[c] + l3[c]) * T(1.0 / 6.0));
    }
    if (!comp) {
        T fv[C];
#pragma unroll
        for (int c = 0; c < C; ++c) fv[c] = f0[c] + inc[c];
        if (unit_length) {
            // one reciprocal square root instead of a square root and nsky divisions
            // (within one unit in the last place of the quotients)
            T ss = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) ss += fv[c] * fv[c];
            if (ss != T(0)) {
                const T r = ss == T(1) ? T(1) : rsqrt(ss);  // unit fields (the vacuum shell) stay exact
#pragma unroll
                for (int c = 0; c < C; ++c)
                    if (c < nsky) fv[c] *= r;
            }
            T lm = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) lm += vv[c] * fv[c];
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) vv[c] -= lm * fv[c];
        }
        v2 = T(0);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            __stcg(Fo + c * N + s, S(fv[c]));
            __stcg(Vo + c * N + s, S(vv[c]));
            v2 += vv[c] * vv[c];
        }
    } else {
        // hi + lo + inc in FP64, with the two small terms summed in FP32 first: lo and the
        // increment are both far below hi, so their FP32 sum loses no more than the FP32
        // increment and the FP32 low part already do (about 2^-49 of the field).  One
        // reciprocal square root normalises.  The velocity is FP32 storage and is
        // projected in FP32 on the rounded field.
        double fd[C];
#pragma unroll
        for (int c = 0; c < C; ++c) fd[c] = double(f0[c]) + double(flo[c] + inc[c]);
        if (unit_length) {
            double ss = 0.0;
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) ss = fma(fd[c], fd[c], ss);
            if (ss != 0.0) {
                const double r = ss == 1.0 ? 1.0 : rsqrt(ss);  // unit fields (the vacuum shell) stay exact
#pragma unroll
                for (int c = 0; c < C; ++c)
                    if (c < nsky) fd[c] *= r;
            }
        }
        T hi[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            hi[c] = T(fd[c]);
            __stcg(Fo + c * N + s, S(hi[c]));
            __stcg(Flo_out + c * N + s, S(fd[c] - double(hi[c])));
        }
        if (unit_length) {
            T lm = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) lm += vv[c] * hi[c];
#pragma unroll
            for (int c = 0; c < C; ++c)
                if (c < nsky) vv[c] -= lm * hi[c];
        }
        v2 = T(0);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            __stcg(Vo + c * N + s, S(vv[c]));
            v2 += vv[c] * vv[c];
        }
    }
}

// finalize_vals with the inputs read from global memory (the stage-4 epilogue).
template <typename T, typename S, int C>
__device__ __forceinline__ void finalize_site(int64_t s, int64_t N, const S* __restrict__ F,
                                              const S* __restrict__ Flo_in, const S* __restrict__ V,
                                              const S* __restrict__ L1, const S* __restrict__ L2,
                                              const S* __restrict__ L3, const T (&g)[C], T dtt, int nsky,
                                              int unit_length, S* __restrict__ Fo, S* __restrict__ Flo_out,
                                              S* __restrict__ Vo, T& v2) {
    // the arrays are read-only during stage 4 (it writes the other halves of the
    // ping-pong pairs): non-coherent global loads (the pointers come from the
    // descriptor in global memory, so the compiler cannot infer the space itself)
    T f0[C], flo[C], v0[C], a1[C], a2[C], a3[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int64_t j = c * N + s;
        f0[c] = T(__ldg(F + j));
        flo[c] = Flo_in ? T(__ldg(Flo_in + j)) : T(0);
        v0[c] = V ? T(__ldg(V + j)) : T(0);
        a1[c] = T(__ldg(L1 + j));
        a2[c] = T(__ldg(L2 + j));
        a3[c] = T(__ldg(L3 + j));
    }
    finalize_vals<T, S, C>(s, N, f0, flo, Flo_in != nullptr, v0, a1, a2, a3, g, dtt, nsky, unit_length, Fo, Flo_out,
                           Vo, v2);
}

// ---------------------------------------------------------------------------
// Control of one instance: reduces the stage-1 partials (energy and baryon number
// of the field entering this step) and the previous step's stage-4 gradient
// partials, records StepStats and sets the arrest flag.
// ---------------------------------------------------------------------------
// mode 0: end of a step (arrest decision); 1: admission (step 0, no arrest);
// 2: resume after a precision change (keeps the pending arrest decision).
// The work is one warp's (the control kernel, or a warp of the last block to finish a
// stage-1 launch, one warp per instance): lane-strided compensated sums of
// the per-tile partials and a fixed shuffle tree, so the order depends on the tile count
// only.  The partials are read through L2: in the stage kernel they were written by
// other blocks of the same launch.
template <typename S>
__device__ __forceinline__ void engine_control_warp(InstDesc<S>& in, int mode) {
    const int lane = (threadIdx.x + blockDim.x * threadIdx.y) & 31;
    KSum e{0.0, 0.0}, b{0.0, 0.0}, kin{0.0, 0.0};
    double gm = -1.0e300, ga = 0.0;
    for (int t = lane; t < in.ntiles; t += 32) {
        ksum_merge(e, KSum{__ldcg(&in.epart[t].s), __ldcg(&in.epart[t].c)});
        ksum_merge(b, KSum{__ldcg(&in.bpart[t].s), __ldcg(&in.bpart[t].c)});
        gm = fmax(gm, __ldcg(&in.gpart[4 * t]));
        ga = fmax(ga, __ldcg(&in.gpart[4 * t + 1]));
        ksum_merge(kin, KSum{__ldcg(&in.gpart[4 * t + 2]), __ldcg(&in.gpart[4 * t + 3])});
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const KSum oe = ksum_shfl_down(e, off), ob = ksum_shfl_down(b, off), ok = ksum_shfl_down(kin, off);
        const double om = __shfl_down_sync(0xffffffffu, gm, off), oa = __shfl_down_sync(0xffffffffu, ga, off);
        if (lane + off < 32) {
            ksum_merge(e, oe);
            ksum_merge(b, ob);
            ksum_merge(kin, ok);
            gm = fmax(gm, om);
            ga = fmax(ga, oa);
        }
    }
    if (lane == 0) {
        const double en = e.s + e.c;
        if (mode == 1) in.step = 0;
        const int n = in.step;
        // arrest (core/integrator.py:403-407): the energy after step n exceeds the one after step n-1
        int arrest = in.arrested;
        if (mode == 0) arrest = (n > 0 && in.p.killkinen && en > in.e_prev) ? 1 : 0;
        if (mode == 1) arrest = 0;
        StepStats& st = in.stats[n % in.stats_cap];
        st.energy = en;
        st.baryon = b.s + b.c;
        if (mode != 2) {  // a resume keeps the step's gradient statistics
            st.err = (n > 0) ? gm : 0.0;
            st.kinetic = (n > 0) ? kin.s + kin.c : 0.0;
            st.gabs = (n > 0) ? ga : 0.0;
        }
        st.arrested = arrest;
        st.step = n;
        st.status = in.status ? *in.status : 0;
        in.arrested = arrest;
        in.e_prev = en;
    }
}

// ---------------------------------------------------------------------------
// Control: one block per instance.  Reduces the stage-1 partials (energy and
// baryon number of the field entering this step) and the previous step's
// stage-4 gradient partials, records StepStats and sets the arrest flag.
// ---------------------------------------------------------------------------
// mode 0: end of a step (arrest decision); 1: admission (step 0, no arrest);
// 2: resume after a precision change (keeps the pending arrest decision).
// (The steps themselves fold mode 0 into stage 1: k_march_stage with tail.)
template <typename S>
__global__ void __launch_bounds__(32) k_engine_control(InstDesc<S>* __restrict__ insts, int i_begin, int i_end,
                                                       int mode) {
    const int ii = i_begin + blockIdx.x;
    if (ii >= i_end) return;
    InstDesc<S>& in = insts[ii];
    if (!in.active) return;
    engine_control_warp(in, mode);
}

// Default number of steps between refreshes of the defect correction of an FP32
// instance (sky_engine_set_defect_period changes it per instance).
constexpr int kDefectRefresh = 16;

// Flip the ping-pong halves and advance the step counter (the tail of stage 4); flag
// the defect refresh of the step that now begins.
template <typename S>
__device__ __forceinline__ void engine_advance_one(InstDesc<S>& in) {
    in.step += 1;
    in.cur ^= 1;
    const int period = in.refresh_period > 0 ? in.refresh_period : kDefectRefresh;
    in.refresh = (in.Dlt != nullptr && in.step % period == 0) ? 1 : 0;
}



// ---------------------------------------------------------------------------
// Marching stage kernel (C <= 5 theories): the stage input is built while the
// x-planes are staged (sky_march.cuh); the epilogue writes l_s, or applies the
// RK4 update at stage 4.
// ---------------------------------------------------------------------------
// The stage-4 update's operands for one plane of a tile, staged by TMA centre-box
// copies into shared memory (k_march_stage with TMA; sky_march.cuh, the plane_begin
// hook): F, F_lo, V, l1, l2, l3 and the defect correction, each C x BY x 32 values in
// [c][y][z] order; a null map means the operand is absent (reads as zero).
template <typename T>
struct CentreStage {
    T* buf;                     // kCentreArrays boxes
    uint64_t* bar;              // the mbarrier the copies complete on
    const TmaMap* map[7];       // F, F_lo, V, l1, l2, l3, Dlt
    int* status;                // the engine's error word (bit 1: a centre-box wait gave up)
    int z0, y0, box;            // tile origin; values per box
    uint32_t phase;             // parity of the copies' next phase
    uint32_t pending;           // parity of the phase this plane's copies complete
};
constexpr int kCentreArrays = 7;

// CC: components of the theory.
// CENTRE: stage 4 reads the update's operands from shared memory (CentreStage).
// NL: sites per thread (2 for the z-pair tiles: lane l is the thread's site l).
template <typename T, int STAGE, int CC, bool CENTRE = false, int NL = 1>
struct EngineEpi {
    // the correction of the thread's next site is held in registers (prefetched a plane
    // ahead) for CC <= 5; with more components it is read at the site
    static constexpr bool kPrefetch = CC <= 5;
    // inputs of the stage-4 update, read from global memory at the site (prefetching them
    // into shared memory with cp.async measured slower: more instructions and shared memory)
    const T* fin_src[6];  // F, F_lo (null unless compensated), V (null when arrested), l1, l2, l3
    T* out0;              // l_STAGE (stages 1-3) or F' (stage 4)
    T* out1;              // V' (stage 4)
    T* Flo_out;           // compensated field: low parts out (stage 4)
    T dtt;
    int nsky;
    int unit_length;
    T gmx, gab;   // signed and absolute maxima of the thread's stage-4 gradients (exact in T)
    T hvol;       // h^3 / 2
    // (1/2) h^3 sum |V'|^2 over the thread's sites: compensated FP64 for an FP64 instance; an
    // FP32 instance's per-site |V'|^2 is an FP32 value and its thread partial (at most one
    // x-chunk of sites) is summed in FP32, then merged per block in FP64
    KSum kin;
    T kin_t;
    T* dlt;       // defect correction (null unless defect-corrected)
    int refresh;  // stage 1 of a refresh step: dlt holds g64 of the field; replace it by g64 - g32
    CentreStage<T>* cs = nullptr;  // CENTRE: the plane's staged operands
    int zbase = 0;                 // z of the thread's first site within the tile
    T d[NL][kPrefetch ? CC : 1];   // the site's correction
    T dn[NL][kPrefetch ? CC : 1];  // the correction of the thread's site on the next plane, in flight
    int64_t dn_tag[NL];            // 1 + the site dn belongs to (0: none; value-initialised)
    // CENTRE: thread 0 copies the update's operands of plane x (every thread calls this
    // right after the plane barrier, before the stencil arithmetic).
    __device__ __forceinline__ void plane_begin(int x) {
        if constexpr (CENTRE) {
            cs->pending = cs->phase;
            cs->phase ^= 1u;
            if (threadIdx.x == 0 && threadIdx.y == 0) {
                uint32_t n = 0;
#pragma unroll
                for (int k = 0; k < kCentreArrays; ++k) n += cs->map[k] != nullptr ? 1u : 0u;
                mbar_arrive_expect_tx(cs->bar, n * uint32_t(cs->box * sizeof(T)));
#pragma unroll
                for (int k = 0; k < kCentreArrays; ++k)
                    if (cs->map[k]) tma_load_plane(cs->buf + k * cs->box, cs->map[k], cs->z0, cs->y0, x, 0, cs->bar);
            }
        }
    }
    // A thread walks its (y, z) column along x.  The correction of the next plane's
    // site is loaded while this site is computed, so that its global-memory latency
    // overlaps a whole plane of stencil and point arithmetic.
    __device__ __forceinline__ void begin_site(int64_t s, int64_t N, int64_t next, int l = 0) {
        if constexpr (CENTRE) return;  // the correction comes with the staged operands
        if constexpr (kPrefetch) {
            if (dlt) {
                if (dn_tag[l] == s + 1) {
#pragma unroll
                    for (int c = 0; c < CC; ++c) d[l][c] = dn[l][c];
                } else {
#pragma unroll
                    for (int c = 0; c < CC; ++c) d[l][c] = __ldcg(dlt + c * N + s);
                }
                if (next >= 0) {
#pragma unroll
                    for (int c = 0; c < CC; ++c) dn[l][c] = __ldcg(dlt + c * N + next);
                }
                dn_tag[l] = next + 1;
            }
        }
    }
    template <int C>
    __device__ __forceinline__ void operator()(int64_t s, int64_t N, const T (&)[C], const T (&g32)[C], int l = 0) {
        static_assert(C == CC, "component count");
        T g[C];
#pragma unroll
        for (int c = 0; c < C; ++c) g[c] = g32[c];
        if constexpr (CENTRE) {
            static_assert(STAGE == 4, "staged operands are the stage-4 update's");
            if (!mbar_wait_bounded(cs->bar, cs->pending)) atomicOr(cs->status, 2);
            // the site within the staged boxes: [c][y - y0][z - z0]
            const int o = threadIdx.y * 32 + zbase + l;
            const int bx = cs->box / C;
            T f0[C], flo[C], v0[C], a1[C], a2[C], a3[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int j = c * bx + o;
                f0[c] = cs->buf[j];
                flo[c] = cs->map[1] ? cs->buf[cs->box + j] : T(0);
                v0[c] = cs->map[2] ? cs->buf[2 * cs->box + j] : T(0);
                a1[c] = cs->buf[3 * cs->box + j];
                a2[c] = cs->buf[4 * cs->box + j];
                a3[c] = cs->buf[5 * cs->box + j];
                if (cs->map[6]) g[c] += cs->buf[6 * cs->box + j];
            }
#pragma unroll
            for (int c = 0; c < C; ++c) {
                gmx = fmax(gmx, g[c]);
                gab = fmax(gab, fabs(g[c]));
            }
            T v2;
            finalize_vals<T, T, C>(s, N, f0, flo, cs->map[1] != nullptr, v0, a1, a2, a3, g, dtt, nsky, unit_length,
                                   out0, Flo_out, out1, v2);
            if constexpr (sizeof(T) == 8)
                ksum_add(kin, hvol * v2);
            else
                kin_t += hvol * v2;
            return;
        }
        if (dlt) {
            T dd[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if constexpr (kPrefetch)
                    dd[c] = d[l][c];
                else
                    dd[c] = __ldcg(dlt + c * N + s);
            }
            if (STAGE == 1 && refresh) {   // dd = g64(F): the correction becomes g64 - g32(F)
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    __stcg(dlt + c * N + s, dd[c] - g32[c]);
                    g[c] = dd[c];
                }
            } else {
#pragma unroll
                for (int c = 0; c < C; ++c) g[c] = g32[c] + dd[c];
            }
        }
        if (STAGE < 4) {
#pragma unroll
            for (int c = 0; c < C; ++c) __stcg(out0 + c * N + s, -dtt * g[c]);
            return;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            gmx = fmax(gmx, g[c]);
            gab = fmax(gab, fabs(g[c]));
        }
        T v2;
        finalize_site<T, T, C>(s, N, fin_src[0], fin_src[1], fin_src[2], fin_src[3], fin_src[4], fin_src[5], g, dtt,
                               nsky, unit_length, out0, Flo_out, out1, v2);
        if constexpr (sizeof(T) == 8)
            ksum_add(kin, hvol * v2);
        else
            kin_t += hvol * v2;
    }
    // the thread's kinetic partial as a compensated FP64 sum
    __device__ __forceinline__ KSum kinetic() const {
        if constexpr (sizeof(T) == 8)
            return kin;
        else
            return KSum{double(kin_t), 0.0};
    }
};

// Shared memory of a stage launch: the plane pipeline (sky_march.cuh), plus for a TMA
// stage 4 the staged update operands when they fit (two FP32 blocks per SM keep
// 2 x (dynamic + 1.3 KB) within the SM's 228 KB).
template <class M, typename T>
constexpr size_t centre_bytes() {
    return size_t(kCentreArrays) * M::C * M::BY * M::BZ * sizeof(T);
}
template <class M, typename T, int STAGE, int MINB, bool TMA>
constexpr bool stage_centre() {
    return STAGE == 4 && TMA &&
           M::template smem_bytes_tma<T>(3) + centre_bytes<M, T>() + 128 <= (MINB >= 2 ? 115000 : kMaxSmemPerBlock);
}
template <class M, typename T, int STAGE, int MINB, bool LO, bool TMA>
constexpr size_t stage_smem_bytes() {
    constexpr int nsrc = LO ? 2 : (STAGE == 1 ? 1 : (STAGE == 2 ? 2 : 3));
    return TMA ? M::template smem_bytes_tma<T>(nsrc, LO) + 128 +
                     (stage_centre<M, T, STAGE, MINB, TMA>() ? centre_bytes<M, T>() : 0)
               : M::template smem_bytes<T>(nsrc, LO);
}

// TMA: planes staged by tensor-memory-accelerator box copies (every instance of
// the launch has its maps encoded; wide rows), and for stage 4 the update's
// operands too when they fit (stage_centre).  PAIR: z-pair tiles (FP32, TMA,
// theories without mixed derivatives; sky_march_pair.cuh), 16 x BY threads.
template <class M, bool PAIR>
constexpr int stage_threads() {
    return PAIR ? PairShape<M>::NT : M::NTHREADS;
}

template <template <typename> class Th, class M, typename T, int STAGE, int MINB, bool LO = false, bool TMA = false,
          bool PAIR = false>
__global__ void __launch_bounds__(stage_threads<M, PAIR>(), MINB)
    k_march_stage(const InstDesc<T>* __restrict__ insts, InstDesc<T>* ctl, const int* __restrict__ tile_inst,
                  int t_begin, int t_end, int* done) {
    static_assert(!PAIR || (TMA && sizeof(T) == 4), "z-pair tiles: FP32 with TMA staging");
    constexpr int NSRC = STAGE == 1 ? (LO ? 2 : 1) : (STAGE == 2 ? 2 : 3);
    constexpr bool CENTRE = stage_centre<M, T, STAGE, MINB, TMA>();
    extern __shared__ __align__(128) unsigned char smraw[];
    // TMA box copies land on 128-byte boundaries: the launch adds 128 bytes of slack
    // and the ring starts at the first 128-byte boundary of the dynamic segment
    T* sm = reinterpret_cast<T*>(smraw + (TMA ? ((128u - (smem_addr(smraw) & 127u)) & 127u) : 0u));
    __shared__ KSum shk[M::NTHREADS / 32];  // one entry per warp (kept small: two blocks
    __shared__ double shm[M::NTHREADS / 32];  // per SM need all but 1 KB of shared memory)
    __shared__ uint64_t tma_bar[3];
    TmaTile tt{tma_bar, 0u, {nullptr, nullptr, nullptr}, nullptr};
    CentreStage<T> cst;
    if constexpr (TMA) {
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            mbar_init(&tma_bar[0], 1);
            mbar_init(&tma_bar[1], 1);
            if (CENTRE) mbar_init(&tma_bar[2], 1);
        }
        __syncthreads();
    }
    // the previous launch of the step (its tail writes the control state) must be complete
    grid_dep_wait();
    if constexpr (CENTRE) {
        cst.buf = sm + M::template smem_bytes_tma<T>(3) / sizeof(T);
        cst.bar = &tma_bar[2];
        cst.box = M::C * M::BY * M::BZ;
        cst.phase = 0u;
        cst.pending = 0u;
    }
    for (int t = t_begin + blockIdx.x; t < t_end; t += gridDim.x) {
        const int ii = __ldg(tile_inst + t);
        const InstDesc<T>& in = insts[ii];
        if (!in.active) continue;  // uniform across the block
        // An arrested step treats the velocity as zero, so its stage-2 input F + (dt/2) V is
        // the field itself: l2 = l1, and stage 2 has nothing to compute.  Stages 3 and 4 then
        // read l1 where they read l2.  Not after a defect refresh: that stage 1 formed l1 from
        // the FP64 gradient, and stage 2's FP32 gradient plus the new correction may differ
        // from it in the last bit.
        const bool l2_is_l1 = in.arrested && !in.refresh;
        if (STAGE == 2 && l2_is_l1) continue;
        const Params p = in.p;
        const int parity = in.cur;
        const int lt = t - in.tile_begin;
        const MarchGrid mg{in.tiles_nz, in.tiles_ny, in.tiles_nx, in.xc};
        int xa, xe, y0, z0;
        march_origin(mg, lt, M::BY, xa, xe, y0, z0, p.X);
        const T* F = in.F[parity];
        const T* V = in.arrested ? nullptr : in.V[parity];
        const T dtt = T(p.dt), hdt = T(0.5 * p.dt);
        T* const L2 = l2_is_l1 ? in.L[0] : in.L[1];  // the step's l2
        const T* const src[3] = {F, LO ? in.Flo[parity] : V, STAGE == 3 ? in.L[0] : L2};
        const T a = STAGE == 4 ? dtt : hdt;
        const T b = STAGE == 3 ? T(0.25) * dtt : T(0.5) * dtt;
        using Epi = EngineEpi<T, STAGE, M::C, CENTRE, PAIR ? 2 : 1>;
        Epi epi{{F, in.Flo[parity], V, in.L[0], L2, in.L[2]},
                                STAGE < 4 ? in.L[STAGE - 1] : in.F[parity ^ 1],
                                STAGE < 4 ? nullptr : in.V[parity ^ 1],
                                in.Flo[parity ^ 1],
                                dtt, p.nsky, p.unit_length, T(-INFINITY), T(0), T(0.5 * p.vol), KSum{0.0, 0.0},
                                T(0), in.Dlt, in.refresh};
        KSum es{0.0, 0.0}, bs{0.0, 0.0};
        if constexpr (TMA) {
            tt.map[0] = &in.tm[kMapF + parity];
            tt.map[1] = LO ? &in.tm[kMapFlo + parity] : (V != nullptr ? &in.tm[kMapV + parity] : nullptr);
            tt.map[2] = NSRC > 2 ? &in.tm[kMapL + (STAGE == 3 || l2_is_l1 ? 0 : 1)] : nullptr;
            tt.status = in.status;
        }
        if constexpr (CENTRE) {
            cst.map[0] = &in.tmc[kMapF + parity];
            cst.map[1] = in.Flo[parity] != nullptr ? &in.tmc[kMapFlo + parity] : nullptr;
            cst.map[2] = V != nullptr ? &in.tmc[kMapV + parity] : nullptr;
            cst.map[3] = &in.tmc[kMapL];
            cst.map[4] = &in.tmc[kMapL + (l2_is_l1 ? 0 : 1)];
            cst.map[5] = &in.tmc[kMapL + 2];
            cst.map[6] = in.Dlt != nullptr ? &in.tmc[kMapDlt] : nullptr;
            cst.status = in.status;
            cst.z0 = z0;
            cst.y0 = y0;
            epi.cs = &cst;
        }
        epi.zbase = PAIR ? 2 * int(threadIdx.x) : int(threadIdx.x);
        bool ok;
        if constexpr (PAIR)
            ok = march_tile_pair<Th, M, NSRC, STAGE == 1, Epi, LO>(sm, p, a, b, xa, xe, y0, z0, epi, es, bs, &tt);
        else
            ok = march_tile<Th, M, T, NSRC, STAGE == 1, Epi, LO, T, true, TMA>(sm, p, src, a, b, xa, xe, y0, z0, epi,
                                                                             es, bs, TMA ? &tt : nullptr);
        // !ok: a copy did not arrive; the block's error bit is set and its partials stay stale
        if (ok && STAGE == 1) {
            const KSum be = block_ksum(es, shk);
            const KSum bb = block_ksum(bs, shk);
            if (threadIdx.x == 0 && threadIdx.y == 0) {
                in.epart[lt] = be;
                in.bpart[lt] = bb;
            }
        }
        if (ok && STAGE == 4) {
            // a thread without sites keeps -inf, which block_max maps below every gradient
            const double ga = block_max(fmax(double(epi.gmx), -1.0e300), shm);
            const double gb = block_max(double(epi.gab), shm);
            const KSum kk = block_ksum(epi.kinetic(), shk);
            if (threadIdx.x == 0 && threadIdx.y == 0) {
                in.gpart[4 * lt] = ga;
                in.gpart[4 * lt + 1] = gb;
                in.gpart[4 * lt + 2] = kk.s;
                in.gpart[4 * lt + 3] = kk.c;
            }
        }
        if (!ok) break;
    }
    grid_dep_launch();  // the next launch may be scheduled while the last blocks finish
    // tail (done != null, stages 1 and 4): the last block of the launch to finish runs the
    // advance (stage 4) or the control (stage 1: reductions, statistics, arrest decision) of
    // every active instance of the launch, one warp per instance, so a step needs no separate
    // launches for them.  Each block publishes its partials (fence) before it is counted; the
    // counter returns to 0 for the next launch.  The tail sits after the tile loop so that its
    // registers do not add to the stencil loop's.
    if constexpr (STAGE == 1 || STAGE == 4) {
        if (done != nullptr) {
            __shared__ int last_block;
            const int ltid = threadIdx.x + blockDim.x * threadIdx.y;
            if (ltid == 0) {
                __threadfence();
                last_block = atomicAdd(done, 1) == int(gridDim.x) - 1 ? 1 : 0;
            }
            __syncthreads();
            if (last_block) {
                __threadfence();
                const int nw = int(blockDim.x * blockDim.y) >> 5;
                const int i1 = __ldg(tile_inst + t_end - 1) + 1;
                for (int i = __ldg(tile_inst + t_begin) + (ltid >> 5); i < i1; i += nw) {
                    if (!ctl[i].active) continue;
                    if constexpr (STAGE == 4) {
                        if ((ltid & 31) == 0) engine_advance_one(ctl[i]);
                    } else {
                        engine_control_warp(ctl[i], 0);
                    }
                }
                if (ltid == 0) *done = 0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Defect refresh: for every defect-corrected FP32 instance whose refresh flag is
// set, the FP64 gradient of its compensated field hi + lo (staged from the FP32
// arrays into an FP64 ring) is written to Dlt; the following stage 1 turns it
// into the correction g64 - g32.
// ---------------------------------------------------------------------------
struct DefectEpi {
    float* dlt;
    template <int C>
    __device__ __forceinline__ void operator()(int64_t s, int64_t N, const double (&)[C], const double (&g)[C]) {
#pragma unroll
        for (int c = 0; c < C; ++c) dlt[c * N + s] = float(g[c]);
    }
};

// TBY: rows of the engine's FP32 tiles; the FP64 ring walks each as TBY / M::BY sub-tiles
// (4-row sub-tiles for 13 components, whose FP64 ring of 8-row planes would not fit).
template <template <typename> class Th, class M, int TBY>
__global__ void __launch_bounds__(M::NTHREADS, 1)
    k_march_defect(InstDesc<float>* __restrict__ insts, const int* __restrict__ tile_inst, int t_begin, int t_end) {
    static_assert(TBY % M::BY == 0, "sub-tiles of the engine tile's rows");
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    grid_dep_wait();
    for (int t = t_begin + blockIdx.x; t < t_end; t += gridDim.x) {
        const int ii = __ldg(tile_inst + t);
        const InstDesc<float>& in = insts[ii];
        if (!in.active || !in.refresh || in.Dlt == nullptr) continue;  // uniform across the block
        const Params p = in.p;
        const int lt = t - in.tile_begin;
        const MarchGrid mg{in.tiles_nz, in.tiles_ny, in.tiles_nx, in.xc};
        int xa, xe, y0, z0;
        march_origin(mg, lt, TBY, xa, xe, y0, z0, p.X);
        const float* const src[3] = {in.F[in.cur], in.Flo[in.cur], nullptr};
        DefectEpi epi{in.Dlt};
        KSum es{0.0, 0.0}, bs{0.0, 0.0};
        for (int sy = 0; sy < TBY && y0 + sy < p.Y; sy += M::BY)
            march_tile<Th, M, double, 2, false, DefectEpi, false, float>(sm, p, src, 1.0, 0.0, xa, xe, y0 + sy, z0,
                                                                         epi, es, bs);
    }
}

// ---------------------------------------------------------------------------
// Energy audit of one instance's current state (F, V), in FP64: the potential
// Phi of the RK4 dynamics (sky_theories.cuh, Dynamics) and the signed kinetic
// term (1/2) h^3 sum_c s_c |V_c|^2, whose sum H the dynamics conserves.  The
// field is staged into an FP64 ring (hi + lo for a compensated field); each
// block writes its two compensated partial sums to parts[4 * block].
// ---------------------------------------------------------------------------
template <template <typename> class Th, typename S>
struct AuditEpi {
    const S* V;  // null: the velocity is zero (arrested)
    int64_t N;
    double hvol;  // h^3 / 2
    KSum kin;
    __device__ __forceinline__ void density(int64_t s, double) {
        if (!V) return;
        double k = 0.0;
#pragma unroll
        for (int c = 0; c < Th<double>::C; ++c) {
            const double v = double(V[c * N + s]);
            k += Dynamics<Th>::kinetic_sign(c) * v * v;
        }
        ksum_add(kin, hvol * k);
    }
};

template <template <typename> class Th, class M, typename S>
__global__ void __launch_bounds__(M::NTHREADS, 1)
    k_engine_audit(const InstDesc<S>* __restrict__ d, MarchGrid mg, double* __restrict__ parts) {
    constexpr int NSRC = std::is_same<S, double>::value ? 1 : 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    double* sm = reinterpret_cast<double*>(smraw);
    __shared__ KSum shk[M::NTHREADS / 32];
    const Params p = d->p;
    const int cur = d->cur;
    const S* const src[3] = {d->F[cur], NSRC == 2 ? d->Flo[cur] : nullptr, nullptr};
    AuditEpi<Th, S> epi{d->arrested ? nullptr : d->V[cur], n_sites(p), 0.5 * p.vol, KSum{0.0, 0.0}};
    KSum es{0.0, 0.0}, unused{0.0, 0.0};
    for (int t = blockIdx.x; t < mg.count(); t += gridDim.x) {
        int xa, xe, y0, z0;
        march_origin(mg, t, M::BY, xa, xe, y0, z0, p.X);
        march_tile<Th, M, double, NSRC, 4, AuditEpi<Th, S>, false, S, false>(sm, p, src, 1.0, 0.0, xa, xe, y0, z0,
                                                                             epi, es, unused);
    }
    const KSum pe = block_ksum(es, shk);
    const KSum pk = block_ksum(epi.kin, shk);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        parts[4 * blockIdx.x] = pe.s;
        parts[4 * blockIdx.x + 1] = pe.c;
        parts[4 * blockIdx.x + 2] = pk.s;
        parts[4 * blockIdx.x + 3] = pk.c;
    }
}

}  // namespace sky
