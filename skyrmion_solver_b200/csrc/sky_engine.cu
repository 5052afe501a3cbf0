// Resident batched engine (host side): owns device memory for a set of lattice
// instances, groups them by (theory, precision), launches the fused stage
// kernels of sky_engine.cuh over every instance of a group at once and replays
// the per-step launch sequence from CUDA graphs.
#include <stdio.h>
#include <string.h>

#include <cmath>
#include <map>
#include <vector>

#include "sky_engine.cuh"
#include "sky_host.h"

namespace sky {

constexpr int kStatsCap = 8192;
constexpr int kGraphSteps = 8;  // steps captured per graph replay

struct HostInst {
    int id = -1;
    int theory = 0;
    int prec = 0;  // storage: 0 = FP32 storage/arithmetic, 1 = FP64
    int comp = 0;    // FP32 storage with a compensated (hi + lo) field
    int defect = 0;  // ... and a defect-corrected gradient (precision 3)
    int defect_period = kDefectRefresh;  // steps between refreshes of the correction
    Params p{};
    int64_t N = 0;
    int C = 0;
    void* F[2] = {nullptr, nullptr};
    void* Flo[2] = {nullptr, nullptr};
    void* Dlt = nullptr;
    void* V[2] = {nullptr, nullptr};
    void* L[3] = {nullptr, nullptr, nullptr};
    KSum* epart = nullptr;
    KSum* bpart = nullptr;
    double* gpart = nullptr;
    StepStats* stats = nullptr;
    int ntiles = 0, tnz = 0, tny = 0, tnx = 0;
    int xc = 0;          // x-chunk of the marching kernels
    int xc_request = 0;  // x-chunk asked for by the caller (0: automatic)
    bool tma = false;    // the stage kernels stage this instance with TMA box copies
    bool pair = false;   // ... with z-pair tiles (FP32 theories without mixed derivatives, option 3)
    int group_slot = -1;
    int64_t steps = 0;  // host mirror of the device step counter
    bool active = true;
    size_t bytes = 0;
};

struct Group {
    int theory = 0, prec = 0;
    std::vector<int> members;  // instance ids in slot order
    void* d_desc = nullptr;    // InstDesc<S>[cap]
    int* d_tile_inst = nullptr;
    int* d_done = nullptr;     // blocks of the current tail stage launch finished (0 between launches)
    int desc_cap = 0, tile_cap = 0;
    int ntiles = 0;
    bool any_comp = false;  // holds a compensated-field instance (stage 1 stages the low parts too)
    bool all_wide = true;   // every member can use the wide-row (16-byte staged) kernels
    bool any_defect = false;  // holds a defect-corrected instance (launch the defect refresh)
    bool all_tma = false;     // every member has TMA plane maps (launch the TMA stage kernels)
    bool all_pair = false;    // ... and runs as z-pair tiles (option 3 at admission)
};

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::map<int, HostInst> insts;
    int next_id = 0;
    Group groups[6][2];
    cudaGraphExec_t graph = nullptr;   // kGraphSteps steps
    cudaGraphExec_t graph1 = nullptr;  // one step (the remainder of a step call)
    bool graph_valid = false;
    int graph_pdl = -1;                // option 4 when the graphs were captured
    int64_t bytes = 0;
    int* d_status = nullptr;  // device error word the stage kernels set (bit 0: a TMA wait gave up)
};

// ---------------------------------------------------------------------------
// shapes and launches per (theory, precision)
// ---------------------------------------------------------------------------
// Every theory runs the marching kernels (sky_march.cuh) in both precisions.
// Tiles are 8 rows x 32 columns, except for FP64 rho (13 components): its
// 4-row tiles keep the five-plane ring at 150 KB, narrow rows only, with two
// of stage 3/4's three sources staged (one block per SM).
constexpr int kMarchBY = 8;
template <template <typename> class Th, typename T>
constexpr int march_by() {
    return (Th<float>::C > 5 && sizeof(T) == 8) ? 4 : kMarchBY;
}
template <template <typename> class Th, typename T>
constexpr bool march_wide_allowed() {
    return !(Th<float>::C > 5 && sizeof(T) == 8);
}
// Wide-row (16-byte staged) or narrow-row march shape.
template <template <typename> class Th, typename T, bool WIDE>
using MShape = MarchShape<Th<T>::C, march_by<Th, T>(), WIDE && march_wide_allowed<Th, T>()>;

template <int STAGE>
constexpr int stage_nsrc() {
    return STAGE == 1 ? 1 : (STAGE == 2 ? 2 : 3);
}

// Resident blocks per SM the marching stages are compiled for (__launch_bounds__):
// two for FP32 (registers capped at 128, no spills for C = 5), one for FP64
// (whose shared memory allows no more).
template <template <typename> class Th, typename T>
constexpr int march_minb() {
    return (sizeof(T) == 4 && Th<float>::C <= 5) ? 2 : 1;
}

// Whether every instance of a group can use the wide-row kernels: Z a multiple of
// 16 / sizeof(T) (the buffers are cudaMalloc'd, hence 256-byte aligned).
static bool wide_ok(int prec, int Z) { return Z % (prec ? 2 : 4) == 0; }

// One-time kernel attribute setup (kept out of stream capture); returns the
// number of resident blocks per SM.
template <template <typename> class Th, typename T, int STAGE, bool WIDE, bool LO = false, bool TMA = false>
static size_t stage_smem() {
    using M = MShape<Th, T, WIDE>;
    return stage_smem_bytes<M, T, STAGE, march_minb<Th, T>(), LO, TMA>();
}

template <template <typename> class Th, typename T, int STAGE, bool WIDE, bool LO = false, bool TMA = false,
          bool PAIR = false>
static int stage_setup_w(int* per_sm_out) {
    static int per_sm = 0;
    if (per_sm == 0) {
        int rc, n = 0;
        using M = MShape<Th, T, WIDE>;
        auto kern = k_march_stage<Th, M, T, STAGE, march_minb<Th, T>(), LO, TMA, PAIR>;
        const size_t smem = stage_smem<Th, T, STAGE, WIDE, LO, TMA>();
        rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                        "cudaFuncSetAttribute(march stage)", __LINE__);
        if (rc) return rc;
        rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, stage_threads<M, PAIR>(), smem),
                        "occupancy query", __LINE__);
        if (rc) return rc;
        per_sm = n < 1 ? 1 : n;
    }
    *per_sm_out = per_sm;
    return SKY_OK;
}

template <template <typename> class Th, typename T, int STAGE>
static int stage_setup(int* per_sm_out) {
    return stage_setup_w<Th, T, STAGE, true>(per_sm_out);
}

template <template <typename> class Th, typename T, int STAGE, bool WIDE, bool LO = false, bool TMA = false,
          bool PAIR = false>
static int launch_stage_w(const Group& g, int t_begin, int t_end, cudaStream_t st, int tail) {
    int per_sm = 1;
    int rc = stage_setup_w<Th, T, STAGE, WIDE, LO, TMA, PAIR>(&per_sm);
    if (rc) return rc;
    int n = t_end - t_begin;
    if (n <= 0) return SKY_OK;
    const int blocks = n < num_sms() * per_sm ? n : num_sms() * per_sm;
    InstDesc<T>* d = reinterpret_cast<InstDesc<T>*>(g.d_desc);
    using M = MShape<Th, T, WIDE>;
    const size_t smem = stage_smem<Th, T, STAGE, WIDE, LO, TMA>();
    const dim3 block(PAIR ? PairShape<M>::TZ : M::BZ, M::BY);
    auto kern = k_march_stage<Th, M, T, STAGE, march_minb<Th, T>(), LO, TMA, PAIR>;
    int* done = tail ? g.d_done : nullptr;
    if (option(4) == 1) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = block;
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return check_cuda(cudaLaunchKernelEx(&cfg, kern, static_cast<const InstDesc<T>*>(d), d,
                                             static_cast<const int*>(g.d_tile_inst), t_begin, t_end, done),
                          "launch engine stage", __LINE__);
    }
    kern<<<blocks, block, smem, st>>>(d, d, g.d_tile_inst, t_begin, t_end, done);
    return check_cuda(cudaGetLastError(), "launch engine stage", __LINE__);
}

// Whether the FP32 stages of Th run as z-pair tiles (option 3, TMA groups, theories
// without mixed second derivatives).
template <template <typename> class Th, typename T>
constexpr bool pair_allowed() {
    return sizeof(T) == 4 && !Th<float>::kMixed && Th<float>::C <= 5;
}

// Whether the stage kernels of (Th, T) can stage with TMA: wide rows must be allowed.
template <template <typename> class Th, typename T>
constexpr bool tma_allowed() {
    return march_wide_allowed<Th, T>();
}

template <template <typename> class Th, typename T, int STAGE>
static int launch_stage(const Group& g, int t_begin, int t_end, cudaStream_t st, int tail) {
    if constexpr (tma_allowed<Th, T>()) {
        if (g.all_tma) {
            if constexpr (pair_allowed<Th, T>()) {
                if (g.all_pair) {
                    if constexpr (STAGE == 1) {
                        if (g.any_comp) return launch_stage_w<Th, T, 1, true, true, true, true>(g, t_begin, t_end, st, tail);
                    }
                    return launch_stage_w<Th, T, STAGE, true, false, true, true>(g, t_begin, t_end, st, tail);
                }
            }
            if constexpr (STAGE == 1 && sizeof(T) == 4 && Th<float>::C <= 5) {
                if (g.any_comp) return launch_stage_w<Th, T, 1, true, true, true>(g, t_begin, t_end, st, tail);
            }
            return launch_stage_w<Th, T, STAGE, true, false, true>(g, t_begin, t_end, st, tail);
        }
    }
    // stage 1 of a group with compensated-field instances stages the low parts too,
    // in wide rows when two blocks per SM still fit (the two six-slot rings take
    // 112.5 KB per block for C = 5), else in narrow rows; rho's 13 components leave
    // no room for the second ring at all: its FP64 densities use the high parts
    if constexpr (STAGE == 1 && sizeof(T) == 4 && Th<float>::C <= 5) {
        if (g.any_comp) {
            if (g.all_wide) {
                int n = 0;
                const int rc = stage_setup_w<Th, T, 1, true, true>(&n);
                if (rc) return rc;
                if (n >= 2) return launch_stage_w<Th, T, 1, true, true>(g, t_begin, t_end, st, tail);
            }
            return launch_stage_w<Th, T, 1, false, true>(g, t_begin, t_end, st, tail);
        }
    }
    if (g.all_wide) return launch_stage_w<Th, T, STAGE, true>(g, t_begin, t_end, st, tail);
    return launch_stage_w<Th, T, STAGE, false>(g, t_begin, t_end, st, tail);
}

template <template <typename> class Th, typename T>
static int launch_stage_any(int stage, const Group& g, int tb, int te, cudaStream_t st, int tail) {
    switch (stage) {
        case 1: return launch_stage<Th, T, 1>(g, tb, te, st, tail);
        case 2: return launch_stage<Th, T, 2>(g, tb, te, st, tail);
        case 3: return launch_stage<Th, T, 3>(g, tb, te, st, tail);
        default: return launch_stage<Th, T, 4>(g, tb, te, st, tail);
    }
}

template <template <typename> class Th>
static int stage_dispatch_prec(int prec, int stage, const Group& g, int tb, int te, cudaStream_t st, int tail) {
    return prec ? launch_stage_any<Th, double>(stage, g, tb, te, st, tail)
                : launch_stage_any<Th, float>(stage, g, tb, te, st, tail);
}

template <template <typename> class Th, typename T>
static int setup_all() {
    int n, rc;
    if ((rc = stage_setup<Th, T, 1>(&n)) || (rc = stage_setup<Th, T, 2>(&n)) || (rc = stage_setup<Th, T, 3>(&n)) ||
        (rc = stage_setup<Th, T, 4>(&n)))
        return rc;
    if constexpr (sizeof(T) == 4 && Th<float>::C <= 5) {  // stage 1 with the low parts
        if ((rc = stage_setup_w<Th, T, 1, true, true>(&n)) || (rc = stage_setup_w<Th, T, 1, false, true>(&n)))
            return rc;
    }
    if constexpr (tma_allowed<Th, T>()) {
        if ((rc = stage_setup_w<Th, T, 1, true, false, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 2, true, false, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 3, true, false, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 4, true, false, true>(&n)))
            return rc;
        if constexpr (sizeof(T) == 4 && Th<float>::C <= 5) {
            if ((rc = stage_setup_w<Th, T, 1, true, true, true>(&n))) return rc;
        }
    }
    if constexpr (tma_allowed<Th, T>() && pair_allowed<Th, T>()) {
        if ((rc = stage_setup_w<Th, T, 1, true, false, true, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 2, true, false, true, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 3, true, false, true, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 4, true, false, true, true>(&n)) ||
            (rc = stage_setup_w<Th, T, 1, true, true, true, true>(&n)))
            return rc;
    }
    return SKY_OK;
}

template <template <typename> class Th>
static int setup_prec(int prec) {
    return prec ? setup_all<Th, double>() : setup_all<Th, float>();
}

static int setup_group(const Group& g) {
    switch (g.theory) {
        case SKY_THEORY_NUCLEAR: return setup_prec<Nuclear>(g.prec);
        case SKY_THEORY_OMEGA: return setup_prec<Omega>(g.prec);
        case SKY_THEORY_COULOMB: return setup_prec<Coulomb>(g.prec);
        case SKY_THEORY_RHO: return setup_prec<Rho>(g.prec);
        case SKY_THEORY_BERGER: return setup_prec<Berger>(g.prec);
        case SKY_THEORY_LIGHTLY_BOUND: return setup_prec<LightlyBound>(g.prec);
    }
    return invalid("unknown theory id");
}

// tail = 1: stage 4 also advances each instance and stage 1 also runs its control
// (the step's launch sequence); 0: the stage alone (admission, precision change).
static int launch_stage_group(int stage, const Group& g, int tb, int te, cudaStream_t st, int tail = 0) {
    switch (g.theory) {
        case SKY_THEORY_NUCLEAR: return stage_dispatch_prec<Nuclear>(g.prec, stage, g, tb, te, st, tail);
        case SKY_THEORY_OMEGA: return stage_dispatch_prec<Omega>(g.prec, stage, g, tb, te, st, tail);
        case SKY_THEORY_COULOMB: return stage_dispatch_prec<Coulomb>(g.prec, stage, g, tb, te, st, tail);
        case SKY_THEORY_RHO: return stage_dispatch_prec<Rho>(g.prec, stage, g, tb, te, st, tail);
        case SKY_THEORY_BERGER: return stage_dispatch_prec<Berger>(g.prec, stage, g, tb, te, st, tail);
        case SKY_THEORY_LIGHTLY_BOUND: return stage_dispatch_prec<LightlyBound>(g.prec, stage, g, tb, te, st, tail);
    }
    return invalid("unknown theory id");
}

// Tile geometry of a (theory, precision): (bz, by, tx) = (32, BY, 0) for the
// marching kernels, whose x-chunk is chosen per instance; per_sm = resident
// stage-4 blocks per SM.
template <template <typename> class Th>
static int shape_of(int prec, int& bz, int& by, int& tx, int& per_sm) {
    per_sm = 1;
    if (prec) {
        bz = 32, by = march_by<Th, double>(), tx = 0;
        return stage_setup<Th, double, 4>(&per_sm);
    }
    bz = 32, by = march_by<Th, float>(), tx = 0;
    return stage_setup<Th, float, 4>(&per_sm);
}

static int tile_shape(int theory, int prec, int& bz, int& by, int& tx, int& per_sm) {
    switch (theory) {
        case SKY_THEORY_NUCLEAR: return shape_of<Nuclear>(prec, bz, by, tx, per_sm);
        case SKY_THEORY_OMEGA: return shape_of<Omega>(prec, bz, by, tx, per_sm);
        case SKY_THEORY_COULOMB: return shape_of<Coulomb>(prec, bz, by, tx, per_sm);
        case SKY_THEORY_RHO: return shape_of<Rho>(prec, bz, by, tx, per_sm);
        case SKY_THEORY_BERGER: return shape_of<Berger>(prec, bz, by, tx, per_sm);
        default: return shape_of<LightlyBound>(prec, bz, by, tx, per_sm);
    }
}

static int launch_control(const Group& g, int ib, int ie, int mode, cudaStream_t st) {
    if (ie <= ib) return SKY_OK;
    if (g.prec)
        k_engine_control<double><<<ie - ib, 32, 0, st>>>(reinterpret_cast<InstDesc<double>*>(g.d_desc), ib, ie, mode);
    else
        k_engine_control<float><<<ie - ib, 32, 0, st>>>(reinterpret_cast<InstDesc<float>*>(g.d_desc), ib, ie, mode);
    return check_cuda(cudaGetLastError(), "launch engine control", __LINE__);
}


// Defect refresh of the group's defect-corrected FP32 instances (those whose
// refresh flag the stage-4 advance just set; the others' tiles are skipped).
template <template <typename> class Th, bool WIDE>
static int launch_defect_t(const Group& g, cudaStream_t st) {
    using M = MarchShape<Th<double>::C, march_by<Th, double>(), WIDE && march_wide_allowed<Th, double>()>;
    auto kern = k_march_defect<Th, M, march_by<Th, float>()>;
    const size_t smem = M::template smem_bytes<double, float>(2);
    static int per_sm = 0;
    if (per_sm == 0) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(defect)", __LINE__);
        if (rc) return rc;
        int n = 0;
        rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, M::NTHREADS, smem), "occupancy",
                        __LINE__);
        if (rc) return rc;
        per_sm = n < 1 ? 1 : n;
    }
    const int n = g.ntiles;
    if (n <= 0) return SKY_OK;
    const int blocks = n < num_sms() * per_sm ? n : num_sms() * per_sm;
    kern<<<blocks, dim3(M::BZ, M::BY), smem, st>>>(reinterpret_cast<InstDesc<float>*>(g.d_desc), g.d_tile_inst, 0,
                                                   n);
    return check_cuda(cudaGetLastError(), "launch defect refresh", __LINE__);
}

template <template <typename> class Th>
static int launch_defect_w(const Group& g, cudaStream_t st) {
    return g.all_wide ? launch_defect_t<Th, true>(g, st) : launch_defect_t<Th, false>(g, st);
}

static int launch_defect(const Group& g, cudaStream_t st) {
    if (g.prec || !g.any_defect) return SKY_OK;
    switch (g.theory) {
        case SKY_THEORY_NUCLEAR: return launch_defect_w<Nuclear>(g, st);
        case SKY_THEORY_OMEGA: return launch_defect_w<Omega>(g, st);
        case SKY_THEORY_COULOMB: return launch_defect_w<Coulomb>(g, st);
        case SKY_THEORY_BERGER: return launch_defect_w<Berger>(g, st);
        case SKY_THEORY_LIGHTLY_BOUND: return launch_defect_w<LightlyBound>(g, st);
        case SKY_THEORY_RHO: return launch_defect_w<Rho>(g, st);
        default: return SKY_OK;
    }
}

// ---------------------------------------------------------------------------
// conversion kernels (FP64 reference layout <-> engine storage)
// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_convert_in(int64_t n, const double* __restrict__ src, S* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src ? S(src[i]) : S(0);
}
template <typename S>
__global__ void k_convert_out(int64_t n, const S* __restrict__ src, double* __restrict__ dst, int zero) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = zero ? 0.0 : double(src[i]);
}
__global__ void k_f32_to_f64(int64_t n, const float* __restrict__ s, double* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = double(s[i]);
}
__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ s, float* __restrict__ d) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = float(s[i]);
}
// FP64 -> compensated FP32 pair (hi = nearest float, lo = nearest float of the remainder)
__global__ void k_f64_to_f32c(int64_t n, const double* __restrict__ s, float* __restrict__ hi,
                              float* __restrict__ lo) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = s[i];
        const float h = float(v);
        hi[i] = h;
        lo[i] = float(v - double(h));
    }
}
__global__ void k_f32c_to_f64(int64_t n, const float* __restrict__ hi, const float* __restrict__ lo,
                              double* __restrict__ d, int zero) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = zero ? 0.0 : double(hi[i]) + double(lo[i]);
}

// ---------------------------------------------------------------------------
// descriptors
// ---------------------------------------------------------------------------
// TMA plane maps of an instance's staged arrays (box: 40 z-values x (BY + 4) rows x 1
// plane x C components, the marching kernels' wide-row plane).
template <typename S>
static int encode_maps(const HostInst& h, InstDesc<S>& d, int by) {
    const void* arrs[kNumCentreMaps] = {h.F[0], h.F[1], h.Flo[0], h.Flo[1], h.V[0], h.V[1],
                                        h.L[0], h.L[1], h.L[2], h.Dlt};
    for (int k = 0; k < kNumCentreMaps; ++k) {
        if (!arrs[k]) continue;
        int rc = SKY_OK;
        if (k < kNumMaps)
            rc = encode_plane_map(&d.tm[k], arrs[k], (int)sizeof(S), h.p.X, h.p.Y, h.p.Z, h.C, 40, by + 4);
        // centre box: the tile's 32 z-values x BY rows, no halo
        if (!rc) rc = encode_plane_map(&d.tmc[k], arrs[k], (int)sizeof(S), h.p.X, h.p.Y, h.p.Z, h.C, 32, by);
        if (rc) return rc;
    }
    return SKY_OK;
}

template <typename S>
static InstDesc<S> make_desc(const HostInst& h, int tile_begin) {
    InstDesc<S> d;
    memset(&d, 0, sizeof(d));
    d.p = h.p;
    for (int i = 0; i < 2; ++i) {
        d.F[i] = reinterpret_cast<S*>(h.F[i]);
        d.Flo[i] = reinterpret_cast<S*>(h.Flo[i]);
        d.Dlt = reinterpret_cast<S*>(h.Dlt);
        d.V[i] = reinterpret_cast<S*>(h.V[i]);
    }
    for (int i = 0; i < 3; ++i) d.L[i] = reinterpret_cast<S*>(h.L[i]);
    d.epart = h.epart;
    d.bpart = h.bpart;
    d.gpart = h.gpart;
    d.stats = h.stats;
    d.stats_cap = kStatsCap;
    d.tile_begin = tile_begin;
    d.ntiles = h.ntiles;
    d.tiles_nz = h.tnz;
    d.tiles_ny = h.tny;
    d.tiles_nx = h.tnx;
    d.xc = h.xc;
    d.active = h.active ? 1 : 0;
    d.refresh_period = h.defect_period;
    return d;
}

// Rebuild a group's device descriptor array and tile list.  Device-updated
// control fields (e_prev, step, arrested, cur) of existing members are kept.
template <typename S>
static int rebuild_group_t(Engine& e, Group& g) {
    // gather current device state of the members (they may move slots)
    std::vector<InstDesc<S>> dev_old;
    if (g.d_desc && g.desc_cap > 0) {
        dev_old.resize(g.desc_cap);
        int rc = check_cuda(cudaMemcpyAsync(dev_old.data(), g.d_desc, sizeof(InstDesc<S>) * g.desc_cap,
                                            cudaMemcpyDeviceToHost, e.stream),
                            "read descriptors", __LINE__);
        if (rc) return rc;
        if ((rc = check_cuda(cudaStreamSynchronize(e.stream), "sync", __LINE__))) return rc;
    }
    std::vector<InstDesc<S>> descs;
    std::vector<int> tile_inst;
    int tb = 0;
    g.any_comp = false;
    g.all_wide = true;
    g.any_defect = false;
    g.all_tma = !g.members.empty();
    g.all_pair = !g.members.empty();
    for (size_t k = 0; k < g.members.size(); ++k) {
        HostInst& h = e.insts[g.members[k]];
        InstDesc<S> d = make_desc<S>(h, tb);
        d.status = e.d_status;
        if (h.tma) {
            int bz, by, tx, per_sm;
            int rc = tile_shape(h.theory, h.prec, bz, by, tx, per_sm);
            if (!rc) rc = encode_maps<S>(h, d, by);
            if (rc) return rc;
            d.tma = 1;
        } else {
            g.all_tma = false;
        }
        if (!h.pair) g.all_pair = false;
        if (h.group_slot >= 0 && h.group_slot < (int)dev_old.size()) {
            const InstDesc<S>& o = dev_old[h.group_slot];
            d.e_prev = o.e_prev;
            d.step = o.step;
            d.arrested = o.arrested;
            d.cur = o.cur;
            d.refresh = (o.refresh && d.Dlt != nullptr) ? 1 : 0;  // a pending defect refresh survives
        }
        h.group_slot = (int)k;
        if (h.comp) g.any_comp = true;
        if (h.defect) g.any_defect = true;
        if (!wide_ok(h.prec, h.p.Z)) g.all_wide = false;
        descs.push_back(d);
        for (int t = 0; t < h.ntiles; ++t) tile_inst.push_back((int)k);
        tb += h.ntiles;
    }
    g.ntiles = tb;
    if ((int)descs.size() > g.desc_cap) {
        if (g.d_desc) cudaFree(g.d_desc);
        g.desc_cap = (int)descs.size() * 2 + 4;
        int rc = check_cuda(cudaMalloc(&g.d_desc, sizeof(InstDesc<S>) * g.desc_cap), "cudaMalloc(desc)", __LINE__);
        if (rc) return rc;
        cudaMemsetAsync(g.d_desc, 0, sizeof(InstDesc<S>) * g.desc_cap, e.stream);
    }
    if (!g.d_done) {
        int rc = check_cuda(cudaMalloc(&g.d_done, sizeof(int)), "cudaMalloc(done)", __LINE__);
        if (rc) return rc;
        cudaMemsetAsync(g.d_done, 0, sizeof(int), e.stream);
    }
    if ((int)tile_inst.size() > g.tile_cap) {
        if (g.d_tile_inst) cudaFree(g.d_tile_inst);
        g.tile_cap = (int)tile_inst.size() * 2 + 64;
        int rc = check_cuda(cudaMalloc(&g.d_tile_inst, sizeof(int) * g.tile_cap), "cudaMalloc(tiles)", __LINE__);
        if (rc) return rc;
    }
    if (!descs.empty()) {
        int rc = check_cuda(cudaMemcpyAsync(g.d_desc, descs.data(), sizeof(InstDesc<S>) * descs.size(),
                                            cudaMemcpyHostToDevice, e.stream),
                            "write descriptors", __LINE__);
        if (rc) return rc;
        rc = check_cuda(cudaMemcpyAsync(g.d_tile_inst, tile_inst.data(), sizeof(int) * tile_inst.size(),
                                        cudaMemcpyHostToDevice, e.stream),
                        "write tile list", __LINE__);
        if (rc) return rc;
    }
    e.graph_valid = false;
    return check_cuda(cudaStreamSynchronize(e.stream), "sync", __LINE__);
}

static int rebuild_group(Engine& e, Group& g) {
    return g.prec ? rebuild_group_t<double>(e, g) : rebuild_group_t<float>(e, g);
}

static void free_inst(HostInst& h) {
    void* ptrs[] = {h.F[0], h.F[1], h.Flo[0], h.Flo[1], h.Dlt, h.V[0], h.V[1], h.L[0], h.L[1], h.L[2],
                    h.epart, h.bpart, h.gpart, h.stats};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    memset(h.F, 0, sizeof(h.F));
    memset(h.Flo, 0, sizeof(h.Flo));
    h.Dlt = nullptr;
    memset(h.V, 0, sizeof(h.V));
    memset(h.L, 0, sizeof(h.L));
    h.epart = h.bpart = nullptr;
    h.gpart = nullptr;
    h.stats = nullptr;
}

// Whether an instance's planes can be staged by TMA box copies: the option is on,
// the row pitch Z * sizeof(T) is a multiple of 16 bytes, and its (theory,
// precision) uses wide rows (every one but FP64 rho).
static bool tma_possible(const HostInst& h) {
    return wide_ok(h.prec, h.p.Z) && !(h.prec && theory_components(h.theory) > 5);
}
static bool tma_ok_for(const HostInst& h) { return option(2) == 1 && tma_possible(h); }
// Whether an instance can run as z-pair tiles (TMA staging, FP32, omega).
static bool pair_possible(const HostInst& h) { return h.prec == 0 && h.theory == SKY_THEORY_OMEGA; }

static int alloc_inst(Engine& e, HostInst& h) {
    const size_t es = h.prec ? sizeof(double) : sizeof(float);
    h.tma = tma_ok_for(h);
    h.pair = h.tma && option(3) == 1 && pair_possible(h);
    const size_t fb = es * (size_t)h.C * (size_t)h.N;
    int bz, by, tx, per_sm;
    int rc0 = tile_shape(h.theory, h.prec, bz, by, tx, per_sm);
    if (rc0) return rc0;
    h.tnz = (h.p.Z + bz - 1) / bz;
    h.tny = (h.p.Y + by - 1) / by;
    (void)tx;
    if ((int64_t)h.C * h.N >= ((int64_t)1 << 31)) return invalid("lattice too large for the marching kernels");
    h.xc = h.xc_request > 0 ? (h.xc_request < h.p.X ? h.xc_request : h.p.X)
                            : choose_xc(h.p.X, h.tnz * h.tny, num_sms() * per_sm);
    h.tnx = (h.p.X + h.xc - 1) / h.xc;
    h.ntiles = h.tnz * h.tny * h.tnx;
    void** bufs[] = {&h.F[0], &h.F[1], &h.V[0], &h.V[1], &h.L[0], &h.L[1], &h.L[2]};
    for (void** b : bufs) {
        if (cudaMalloc(b, fb) != cudaSuccess) {
            cudaGetLastError();
            free_inst(h);
            return SKY_ERR_NOMEM;
        }
    }
    if (cudaMalloc(&h.epart, sizeof(KSum) * h.ntiles) != cudaSuccess ||
        cudaMalloc(&h.bpart, sizeof(KSum) * h.ntiles) != cudaSuccess ||
        cudaMalloc(&h.gpart, sizeof(double) * 4 * h.ntiles) != cudaSuccess ||
        cudaMalloc(&h.stats, sizeof(StepStats) * kStatsCap) != cudaSuccess) {
        cudaGetLastError();
        free_inst(h);
        return SKY_ERR_NOMEM;
    }
    if (h.comp) {
        for (int i = 0; i < 2; ++i) {
            if (cudaMalloc(&h.Flo[i], fb) != cudaSuccess) {
                cudaGetLastError();
                free_inst(h);
                return SKY_ERR_NOMEM;
            }
            cudaMemsetAsync(h.Flo[i], 0, fb, e.stream);
        }
    }
    if (h.defect) {
        if (cudaMalloc(&h.Dlt, fb) != cudaSuccess) {
            cudaGetLastError();
            free_inst(h);
            return SKY_ERR_NOMEM;
        }
        cudaMemsetAsync(h.Dlt, 0, fb, e.stream);
    }
    cudaMemsetAsync(h.gpart, 0, sizeof(double) * 4 * h.ntiles, e.stream);
    cudaMemsetAsync(h.stats, 0, sizeof(StepStats) * kStatsCap, e.stream);
    h.bytes = (h.comp ? 9 : 7) * fb + (h.defect ? fb : 0) + (sizeof(KSum) * 2 + sizeof(double) * 4) * h.ntiles +
              sizeof(StepStats) * kStatsCap;
    return SKY_OK;
}

static int upload(Engine& e, HostInst& h, const double* field, const double* velocity, bool on_device) {
    const int64_t n = (int64_t)h.C * h.N;
    double* tmp = nullptr;
    int rc = SKY_OK;
    const double* srcs[2] = {field, velocity};
    void* dsts[2] = {h.F[0], h.V[0]};
    for (int k = 0; k < 2; ++k) {
        const double* src = srcs[k];
        if (src && !on_device) {
            if (!tmp && (rc = check_cuda(cudaMalloc(&tmp, sizeof(double) * n), "cudaMalloc(upload)", __LINE__)))
                return rc;
            if ((rc = check_cuda(cudaMemcpyAsync(tmp, src, sizeof(double) * n, cudaMemcpyHostToDevice, e.stream),
                                 "upload", __LINE__)))
                break;
            src = tmp;
        }
        if (h.prec)
            k_convert_in<double><<<ew_blocks(n), 256, 0, e.stream>>>(n, src, reinterpret_cast<double*>(dsts[k]));
        else if (k == 0 && h.comp)
            k_f64_to_f32c<<<ew_blocks(n), 256, 0, e.stream>>>(n, src, reinterpret_cast<float*>(h.F[0]),
                                                              reinterpret_cast<float*>(h.Flo[0]));
        else
            k_convert_in<float><<<ew_blocks(n), 256, 0, e.stream>>>(n, src, reinterpret_cast<float*>(dsts[k]));
        if ((rc = check_cuda(cudaGetLastError(), "convert", __LINE__))) break;
        if (tmp) cudaStreamSynchronize(e.stream);
    }
    if (tmp) {
        cudaStreamSynchronize(e.stream);
        cudaFree(tmp);
    }
    return rc;
}

// Stage 1 + control for one instance (admission or precision change).
static int init_instance(Engine& e, HostInst& h, int mode) {
    Group& g = e.groups[h.theory][h.prec];
    int tb = 0;
    for (int id : g.members) {
        if (id == h.id) break;
        tb += e.insts[id].ntiles;
    }
    int rc = launch_stage_group(1, g, tb, tb + h.ntiles, e.stream);
    if (rc) return rc;
    rc = launch_control(g, h.group_slot, h.group_slot + 1, mode, e.stream);
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(e.stream), "sync", __LINE__);
}

// Launch kinds of one step, in order: stage 2, 3, 4 (+ update), advance, the
// defect refresh (groups with defect-corrected instances only), stage 1 (on the
// updated field), control.  Groups are independent, so each kind is issued for
// every non-empty group before the next kind.
enum { kKindS2 = 0, kKindS3, kKindS4, kKindAdvance, kKindDefect, kKindS1, kKindControl, kNumKinds };

static int launch_kind(Engine& e, int kind) {
    for (int t = 0; t < 6; ++t)
        for (int pr = 0; pr < 2; ++pr) {
            Group& g = e.groups[t][pr];
            if (g.members.empty()) continue;
            int rc = SKY_OK;
            switch (kind) {
                case kKindS2: rc = launch_stage_group(2, g, 0, g.ntiles, e.stream); break;
                case kKindS3: rc = launch_stage_group(3, g, 0, g.ntiles, e.stream); break;
                case kKindS4: rc = launch_stage_group(4, g, 0, g.ntiles, e.stream, 1); break;
                case kKindAdvance: break;  // folded into stage 4
                case kKindDefect: rc = launch_defect(g, e.stream); break;
                case kKindS1: rc = launch_stage_group(1, g, 0, g.ntiles, e.stream, 1); break;
                default: break;  // the control is folded into stage 1
            }
            if (rc) return rc;
        }
    return SKY_OK;
}

static int record_step(Engine& e) {
    for (int k = 0; k < kNumKinds; ++k) {
        int rc = launch_kind(e, k);
        if (rc) return rc;
    }
    return SKY_OK;
}

static int count_launches(Engine& e) {
    int n = 0;
    for (int t = 0; t < 6; ++t)
        for (int pr = 0; pr < 2; ++pr)
            if (!e.groups[t][pr].members.empty())
                n += 4 + ((pr == 0 && e.groups[t][pr].any_defect) ? 1 : 0);  // stages 2, 3, 4, [defect,] 1
    return n;
}

// Capture `nsteps` steps of the current instance set into *exec.
static int capture_steps(Engine& e, int nsteps, cudaGraphExec_t* exec) {
    if (*exec) {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    cudaGraph_t graph;
    int rc = check_cuda(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal), "begin capture",
                        __LINE__);
    if (rc) return rc;
    for (int s = 0; s < nsteps && rc == SKY_OK; ++s) rc = record_step(e);
    cudaError_t ce = cudaStreamEndCapture(e.stream, &graph);
    if (rc) {
        if (ce == cudaSuccess) cudaGraphDestroy(graph);
        return rc;
    }
    if ((rc = check_cuda(ce, "end capture", __LINE__))) return rc;
    rc = check_cuda(cudaGraphInstantiate(exec, graph, 0), "graph instantiate", __LINE__);
    cudaGraphDestroy(graph);
    return rc;
}

// The step graphs: kGraphSteps steps, and one step for the remainder of a call.
// Each step depends only on device-side state, so replaying them is the same as
// launching the kernels one by one.
static int build_graph(Engine& e) {
    int rc = SKY_OK;
    for (int t = 0; t < 6; ++t)
        for (int pr = 0; pr < 2; ++pr)
            if (!e.groups[t][pr].members.empty() && (rc = setup_group(e.groups[t][pr]))) return rc;
    if ((rc = capture_steps(e, kGraphSteps, &e.graph)) || (rc = capture_steps(e, 1, &e.graph1))) return rc;
    e.graph_valid = true;
    e.graph_pdl = option(4);
    return SKY_OK;
}

// A statistics record written while the engine's error word was set: a stage
// kernel gave up waiting for a TMA copy, so the step's results are not valid.
static int status_error(const StepStats& st) {
    if (st.status == 0) return SKY_OK;
    char msg[160];
    snprintf(msg, sizeof(msg), "engine error word 0x%x: a stage kernel gave up waiting for a TMA plane copy",
             (unsigned)st.status);
    return fail(SKY_ERR_TIMEOUT, msg);
}

static HostInst* find(Engine* e, int id) {
    auto it = e->insts.find(id);
    return it == e->insts.end() ? nullptr : &it->second;
}

static int remove_from_group(Engine& e, HostInst& h) {
    Group& g = e.groups[h.theory][h.prec];
    // the remaining members still carry their old slots, from which the
    // rebuild gathers their device control state
    std::vector<int> keep;
    for (int id : g.members)
        if (id != h.id) keep.push_back(id);
    g.members = keep;
    const int rc = rebuild_group(e, g);
    h.group_slot = -1;
    return rc;
}

}  // namespace sky

using namespace sky;

// ---------------------------------------------------------------------------
// energy audit of the RK4 dynamics (k_engine_audit)
// ---------------------------------------------------------------------------
constexpr int kAuditBY = 4;  // 4-row tiles: a 13-component FP64 ring still fits

template <template <typename> class Th, typename S>
static int audit_t(Engine& e, const HostInst& h, double* out2) {
    using M = MarchShape<Th<double>::C, kAuditBY, false>;
    constexpr int NSRC = std::is_same<S, double>::value ? 1 : 2;
    auto kern = k_engine_audit<Th, M, S>;
    const size_t smem = M::template smem_bytes<double, S>(NSRC);
    static bool configured = false;
    if (!configured) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(audit)", __LINE__);
        if (rc) return rc;
        configured = true;
    }
    const MarchGrid mg = march_grid<M>(h.p, h.p.X < 16 ? h.p.X : 16);
    const int blocks = mg.count() < num_sms() ? mg.count() : num_sms();
    double* parts = nullptr;
    int rc = check_cuda(cudaMalloc(&parts, sizeof(double) * 4 * blocks), "cudaMalloc(audit)", __LINE__);
    if (rc) return rc;
    const Group& g = e.groups[h.theory][h.prec];
    const InstDesc<S>* d = reinterpret_cast<const InstDesc<S>*>(g.d_desc) + h.group_slot;
    kern<<<blocks, dim3(M::BZ, M::BY), smem, e.stream>>>(d, mg, parts);
    rc = check_cuda(cudaGetLastError(), "launch audit", __LINE__);
    std::vector<double> hp(4 * (size_t)blocks);
    if (!rc)
        rc = check_cuda(cudaMemcpyAsync(hp.data(), parts, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, e.stream),
                        "read audit", __LINE__);
    if (!rc) rc = check_cuda(cudaStreamSynchronize(e.stream), "sync audit", __LINE__);
    cudaFree(parts);
    if (rc) return rc;
    // fixed-order compensated sum of the block partials
    for (int q = 0; q < 2; ++q) {
        double sum = 0.0, comp = 0.0;
        for (int b = 0; b < blocks; ++b) {
            for (int k = 0; k < 2; ++k) {
                const double v = hp[4 * b + 2 * q + k];
                const double t = sum + v;
                comp += (std::fabs(sum) >= std::fabs(v)) ? ((sum - t) + v) : ((v - t) + sum);
                sum = t;
            }
        }
        out2[q] = sum + comp;
    }
    return SKY_OK;
}

template <template <typename> class Th>
static int audit_prec(Engine& e, const HostInst& h, double* out2) {
    return h.prec ? audit_t<Th, double>(e, h, out2) : audit_t<Th, float>(e, h, out2);
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int sky_engine_create(int device, void** out) {
    if (!out) return invalid("null output");
    Engine* e = new Engine();
    e->device = device;
    int rc = check_cuda(cudaSetDevice(device), "cudaSetDevice", __LINE__);
    if (!rc) rc = check_cuda(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream", __LINE__);
    if (!rc) rc = check_cuda(cudaMalloc(&e->d_status, sizeof(int)), "cudaMalloc(status)", __LINE__);
    if (!rc) rc = check_cuda(cudaMemset(e->d_status, 0, sizeof(int)), "memset(status)", __LINE__);
    if (rc) {
        if (e->d_status) cudaFree(e->d_status);
        if (e->stream) cudaStreamDestroy(e->stream);
        delete e;
        return rc;
    }
    for (int t = 0; t < 6; ++t)
        for (int p = 0; p < 2; ++p) {
            e->groups[t][p].theory = t;
            e->groups[t][p].prec = p;
        }
    *out = e;
    return SKY_OK;
}

int sky_engine_destroy(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return SKY_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->graph1) cudaGraphExecDestroy(e->graph1);
    for (auto& kv : e->insts) free_inst(kv.second);
    for (int t = 0; t < 6; ++t)
        for (int p = 0; p < 2; ++p) {
            if (e->groups[t][p].d_desc) cudaFree(e->groups[t][p].d_desc);
            if (e->groups[t][p].d_tile_inst) cudaFree(e->groups[t][p].d_tile_inst);
            if (e->groups[t][p].d_done) cudaFree(e->groups[t][p].d_done);
        }
    if (e->d_status) cudaFree(e->d_status);
    cudaStreamDestroy(e->stream);
    delete e;
    return SKY_OK;
}

int sky_engine_add(void* handle, int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                   int precision, const double* field, const double* velocity, int on_device, int* id_out) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !id_out || !field) return invalid("null argument");
    if (precision < 0 || precision > 3)
        return invalid("precision must be 0 (FP32), 1 (FP64), 2 (FP32 with a compensated field) or 3 "
                       "(compensated and defect-corrected FP32)");
    cudaSetDevice(e->device);
    HostInst h;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &h.p);
    if (rc) return rc;
    h.id = e->next_id++;
    h.theory = theory;
    h.prec = precision == 1 ? 1 : 0;
    h.comp = precision >= 2 ? 1 : 0;
    h.defect = precision == 3 ? 1 : 0;
    h.N = n_sites(h.p);
    h.C = h.p.C;
    if ((rc = alloc_inst(*e, h))) return rc;
    if ((rc = upload(*e, h, field, velocity, on_device != 0))) {
        free_inst(h);
        return rc;
    }
    e->insts[h.id] = h;
    Group& g = e->groups[theory][h.prec];
    g.members.push_back(h.id);
    if ((rc = rebuild_group(*e, g)) || (rc = init_instance(*e, e->insts[h.id], 1))) {
        g.members.pop_back();
        free_inst(e->insts[h.id]);
        e->insts.erase(h.id);
        rebuild_group(*e, g);
        return rc;
    }
    e->bytes += (int64_t)h.bytes;
    *id_out = h.id;
    return SKY_OK;
}

int sky_engine_remove(void* handle, int id) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* h = find(e, id);
    if (!h) return invalid("unknown instance id");
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    int rc = remove_from_group(*e, *h);
    e->bytes -= (int64_t)h->bytes;
    free_inst(*h);
    e->insts.erase(id);
    return rc;
}

int sky_engine_set_precision(void* handle, int id, int precision) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    if (precision < 0 || precision > 3) return invalid("precision must be 0, 1, 2 or 3");
    const int defect_new = precision == 3 ? 1 : 0;
    if ((hp->comp ? 2 + hp->defect : hp->prec) == precision) return SKY_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    HostInst& h = *hp;
    // read the control state of the instance
    int cur = 0, arrested = 0, step = 0;
    double e_prev = 0.0;
    {
        Group& g = e->groups[h.theory][h.prec];
        if (h.prec) {
            InstDesc<double> d;
            cudaMemcpy(&d, reinterpret_cast<InstDesc<double>*>(g.d_desc) + h.group_slot, sizeof(d),
                       cudaMemcpyDeviceToHost);
            cur = d.cur, arrested = d.arrested, step = d.step, e_prev = d.e_prev;
        } else {
            InstDesc<float> d;
            cudaMemcpy(&d, reinterpret_cast<InstDesc<float>*>(g.d_desc) + h.group_slot, sizeof(d),
                       cudaMemcpyDeviceToHost);
            cur = d.cur, arrested = d.arrested, step = d.step, e_prev = d.e_prev;
        }
    }
    HostInst nh = h;
    nh.prec = precision == 1 ? 1 : 0;
    nh.comp = precision >= 2 ? 1 : 0;
    nh.defect = defect_new;
    nh.Dlt = nullptr;
    nh.group_slot = -1;
    for (int i = 0; i < 2; ++i) nh.F[i] = nh.Flo[i] = nh.V[i] = nullptr;
    for (int i = 0; i < 3; ++i) nh.L[i] = nullptr;
    nh.epart = nh.bpart = nullptr;
    nh.gpart = nullptr;
    nh.stats = nullptr;
    int rc = alloc_inst(*e, nh);
    if (rc) return rc;
    const int64_t n = (int64_t)h.C * h.N;
    const void* srcs[2] = {h.F[cur], h.V[cur]};
    void* dsts[2] = {nh.F[0], nh.V[0]};
    const size_t fb = (h.prec ? sizeof(double) : sizeof(float)) * (size_t)n;
    for (int k = 0; k < 2; ++k) {
        const bool fieldk = k == 0;
        if (nh.prec == h.prec) {  // FP32 <-> compensated FP32: the high part carries over
            cudaMemcpyAsync(dsts[k], srcs[k], fb, cudaMemcpyDeviceToDevice, e->stream);
            if (fieldk && h.comp && nh.comp)
                cudaMemcpyAsync(nh.Flo[0], h.Flo[cur], fb, cudaMemcpyDeviceToDevice, e->stream);
        } else if (nh.prec) {     // FP32 (+ low part) -> FP64
            if (fieldk && h.comp)
                k_f32c_to_f64<<<ew_blocks(n), 256, 0, e->stream>>>(n, (const float*)srcs[k], (const float*)h.Flo[cur],
                                                                   (double*)dsts[k], 0);
            else
                k_f32_to_f64<<<ew_blocks(n), 256, 0, e->stream>>>(n, (const float*)srcs[k], (double*)dsts[k]);
        } else {                  // FP64 -> FP32 (+ low part)
            if (fieldk && nh.comp)
                k_f64_to_f32c<<<ew_blocks(n), 256, 0, e->stream>>>(n, (const double*)srcs[k], (float*)dsts[k],
                                                                   (float*)nh.Flo[0]);
            else
                k_f64_to_f32<<<ew_blocks(n), 256, 0, e->stream>>>(n, (const double*)srcs[k], (float*)dsts[k]);
        }
    }
    // carry the stats history
    cudaMemcpyAsync(nh.stats, h.stats, sizeof(StepStats) * kStatsCap, cudaMemcpyDeviceToDevice, e->stream);
    if ((rc = check_cuda(cudaStreamSynchronize(e->stream), "convert", __LINE__))) {
        free_inst(nh);
        return rc;
    }
    // leave the old group
    if ((rc = remove_from_group(*e, h))) {
        free_inst(nh);
        return rc;
    }
    free_inst(h);
    e->bytes += (int64_t)nh.bytes - (int64_t)h.bytes;
    h = nh;
    Group& g2 = e->groups[h.theory][h.prec];
    g2.members.push_back(h.id);
    if ((rc = rebuild_group(*e, g2))) return rc;
    // restore the control state, then recompute l1 / energy of the converted field
    if (h.prec) {
        InstDesc<double>* dd = reinterpret_cast<InstDesc<double>*>(g2.d_desc) + h.group_slot;
        cudaMemcpyAsync(&dd->step, &step, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&dd->arrested, &arrested, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&dd->e_prev, &e_prev, sizeof(double), cudaMemcpyHostToDevice, e->stream);
    } else {
        InstDesc<float>* dd = reinterpret_cast<InstDesc<float>*>(g2.d_desc) + h.group_slot;
        cudaMemcpyAsync(&dd->step, &step, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&dd->arrested, &arrested, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        cudaMemcpyAsync(&dd->e_prev, &e_prev, sizeof(double), cudaMemcpyHostToDevice, e->stream);
    }
    return init_instance(*e, h, 2);
}

int sky_engine_retile(void* handle, int id, int xc) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    if (xc < 0) return invalid("xc must be >= 0 (0: automatic)");
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    HostInst& h = *hp;
    int bz, by, tx, per_sm;
    int rc = tile_shape(h.theory, h.prec, bz, by, tx, per_sm);
    if (rc) return rc;
    const int tny = (h.p.Y + by - 1) / by, tnz = (h.p.Z + bz - 1) / bz;
    const int nxc = xc > 0 ? (xc < h.p.X ? xc : h.p.X) : choose_xc(h.p.X, tnz * tny, num_sms() * per_sm);
    const int ntiles = tnz * tny * ((h.p.X + nxc - 1) / nxc);
    KSum *ep = nullptr, *bp = nullptr;
    double* gp = nullptr;
    if (cudaMalloc(&ep, sizeof(KSum) * ntiles) != cudaSuccess || cudaMalloc(&bp, sizeof(KSum) * ntiles) != cudaSuccess ||
        cudaMalloc(&gp, sizeof(double) * 4 * ntiles) != cudaSuccess) {
        cudaGetLastError();
        if (ep) cudaFree(ep);
        if (bp) cudaFree(bp);
        if (gp) cudaFree(gp);
        return SKY_ERR_NOMEM;
    }
    // The per-tile partials of the latest stage 1 feed the next control launch:
    // re-run stage 1 and the control in resume mode under the new geometry (the
    // pending arrest decision and the step's gradient statistics are kept).
    cudaFree(h.epart);
    cudaFree(h.bpart);
    cudaFree(h.gpart);
    h.epart = ep;
    h.bpart = bp;
    h.gpart = gp;
    cudaMemsetAsync(h.gpart, 0, sizeof(double) * 4 * ntiles, e->stream);
    const int64_t dbytes = (int64_t)(sizeof(KSum) * 2 + sizeof(double) * 4) * ((int64_t)ntiles - h.ntiles);
    h.bytes += dbytes;
    e->bytes += dbytes;
    h.xc_request = xc;
    h.xc = nxc;
    h.tnx = (h.p.X + nxc - 1) / nxc;
    h.ntiles = ntiles;  // the staging (TMA, z-pairs) carries over
    Group& g = e->groups[h.theory][h.prec];
    if ((rc = rebuild_group(*e, g))) return rc;
    return init_instance(*e, h, 2);
}

int sky_engine_set_staging(void* handle, int id, int tma, int pair) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    if ((tma != 0 && tma != 1) || (pair != 0 && pair != 1)) return invalid("tma and pair must be 0 or 1");
    HostInst& h = *hp;
    if (tma && !tma_possible(h))
        return invalid("TMA staging needs Z * element size a multiple of 16 bytes (and no FP64 rho)");
    if (pair && !(tma && pair_possible(h))) return invalid("z-pair tiles need TMA staging and an FP32 omega instance");
    if (h.tma == tma && h.pair == pair) return SKY_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    h.tma = tma;
    h.pair = pair;
    return rebuild_group(*e, e->groups[h.theory][h.prec]);  // keeps the control state
}

int sky_engine_get_staging(void* handle, int id, int* tma, int* pair) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !tma || !pair) return invalid("null argument");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    *tma = hp->tma;
    *pair = hp->pair;
    return SKY_OK;
}

int sky_engine_audit(void* handle, int id, double* out2) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    if (!out2) return invalid("null output");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    cudaSetDevice(e->device);
    switch (hp->theory) {
        case SKY_THEORY_NUCLEAR: return audit_prec<Nuclear>(*e, *hp, out2);
        case SKY_THEORY_OMEGA: return audit_prec<Omega>(*e, *hp, out2);
        case SKY_THEORY_COULOMB: return audit_prec<Coulomb>(*e, *hp, out2);
        case SKY_THEORY_RHO: return audit_prec<Rho>(*e, *hp, out2);
        case SKY_THEORY_BERGER: return audit_prec<Berger>(*e, *hp, out2);
        case SKY_THEORY_LIGHTLY_BOUND: return audit_prec<LightlyBound>(*e, *hp, out2);
    }
    return invalid("unknown theory id");
}

int sky_engine_set_defect_period(void* handle, int id, int period) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* hp = find(e, id);
    if (!hp) return invalid("unknown instance id");
    if (period < 1) return invalid("defect refresh period must be >= 1");
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    hp->defect_period = period;
    Group& g = e->groups[hp->theory][hp->prec];
    const size_t sz = hp->prec ? sizeof(InstDesc<double>) : sizeof(InstDesc<float>);
    const size_t off = hp->prec ? offsetof(InstDesc<double>, refresh_period) : offsetof(InstDesc<float>, refresh_period);
    char* base = reinterpret_cast<char*>(g.d_desc) + sz * hp->group_slot;
    int rc = check_cuda(cudaMemcpyAsync(base + off, &period, sizeof(int), cudaMemcpyHostToDevice, e->stream),
                        "write refresh period", __LINE__);
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__);
}

int sky_engine_get_xc(void* handle, int id) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return -1;
    HostInst* h = find(e, id);
    return h ? h->xc : -1;
}

int sky_engine_set_active(void* handle, int id, int active) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* h = find(e, id);
    if (!h) return invalid("unknown instance id");
    h->active = active != 0;
    Group& g = e->groups[h->theory][h->prec];
    const int a = h->active ? 1 : 0;
    size_t off = h->prec ? offsetof(InstDesc<double>, active) : offsetof(InstDesc<float>, active);
    size_t sz = h->prec ? sizeof(InstDesc<double>) : sizeof(InstDesc<float>);
    char* base = reinterpret_cast<char*>(g.d_desc) + sz * h->group_slot + off;
    int rc = check_cuda(cudaMemcpyAsync(base, &a, sizeof(int), cudaMemcpyHostToDevice, e->stream), "set active",
                        __LINE__);
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__);
}

int sky_engine_step(void* handle, int nsteps) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    if (nsteps < 0) return invalid("nsteps must be >= 0");
    cudaSetDevice(e->device);
    int rc;
    int done = 0;
    if (e->graph_valid && e->graph_pdl != option(4)) e->graph_valid = false;
    if (nsteps > 0 && !e->graph_valid && (rc = build_graph(*e))) return rc;
    while (nsteps - done >= kGraphSteps) {
        if ((rc = check_cuda(cudaGraphLaunch(e->graph, e->stream), "graph launch", __LINE__))) return rc;
        done += kGraphSteps;
    }
    for (; done < nsteps; ++done)
        if ((rc = check_cuda(cudaGraphLaunch(e->graph1, e->stream), "graph launch", __LINE__))) return rc;
    for (auto& kv : e->insts)
        if (kv.second.active) kv.second.steps += nsteps;
    return SKY_OK;
}

int sky_engine_synchronize(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    return check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__);
}

void* sky_engine_stream(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    return e ? (void*)e->stream : nullptr;
}

int sky_engine_stats(void* handle, int id, int64_t step, double* out6) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !out6) return invalid("null argument");
    HostInst* h = find(e, id);
    if (!h) return invalid("unknown instance id");
    if (step < 0) step = h->steps;
    if (step > h->steps || h->steps - step >= kStatsCap) return invalid("step outside the retained history");
    StepStats st;
    int rc = check_cuda(cudaMemcpyAsync(&st, h->stats + (step % kStatsCap), sizeof(st), cudaMemcpyDeviceToHost,
                                        e->stream),
                        "read stats", __LINE__);
    if (rc) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__))) return rc;
    if ((rc = status_error(st))) return rc;
    out6[0] = st.energy;
    out6[1] = st.baryon;
    out6[2] = st.err;
    out6[3] = st.gabs;
    out6[4] = st.arrested;
    out6[5] = st.step;
    return SKY_OK;
}

int sky_engine_stats_ex(void* handle, int id, int64_t step, double* out8) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !out8) return invalid("null argument");
    HostInst* h = find(e, id);
    if (!h) return invalid("unknown instance id");
    if (step < 0) step = h->steps;
    if (step > h->steps || h->steps - step >= kStatsCap) return invalid("step outside the retained history");
    StepStats st;
    int rc = check_cuda(cudaMemcpyAsync(&st, h->stats + (step % kStatsCap), sizeof(st), cudaMemcpyDeviceToHost,
                                        e->stream),
                        "read stats", __LINE__);
    if (rc) return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__))) return rc;
    if ((rc = status_error(st))) return rc;
    out8[0] = st.energy;
    out8[1] = st.baryon;
    out8[2] = st.err;
    out8[3] = st.gabs;
    out8[4] = st.arrested;
    out8[5] = st.step;
    out8[6] = st.kinetic;
    out8[7] = h->comp ? 2 + h->defect : h->prec;
    return SKY_OK;
}

int sky_engine_stats_all(void* handle, int* ids_out, double* out7, int cap, int* count_out) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !count_out) return invalid("null argument");
    std::vector<StepStats> st(e->insts.size());
    std::vector<const HostInst*> hs;
    int k = 0;
    for (auto& kv : e->insts) {
        if (k >= cap) break;
        const HostInst& h = kv.second;
        int rc = check_cuda(cudaMemcpyAsync(&st[k], h.stats + (h.steps % kStatsCap), sizeof(StepStats),
                                            cudaMemcpyDeviceToHost, e->stream),
                            "read stats", __LINE__);
        if (rc) return rc;
        hs.push_back(&h);
        ++k;
    }
    int rc = check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__);
    if (rc) return rc;
    for (int i = 0; i < k; ++i)
        if ((rc = status_error(st[i]))) return rc;
    for (int i = 0; i < k; ++i) {
        if (ids_out) ids_out[i] = hs[i]->id;
        if (out7) {
            double* o = out7 + 7 * i;
            o[0] = st[i].energy;
            o[1] = st[i].baryon;
            o[2] = st[i].err;
            o[3] = st[i].gabs;
            o[4] = st[i].arrested;
            o[5] = st[i].step;
            o[6] = hs[i]->comp ? 2 + hs[i]->defect : hs[i]->prec;
        }
    }
    *count_out = k;
    return SKY_OK;
}

int sky_engine_read(void* handle, int id, double* field, double* velocity, int on_device) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e) return invalid("null engine");
    HostInst* h = find(e, id);
    if (!h) return invalid("unknown instance id");
    cudaSetDevice(e->device);
    Group& g = e->groups[h->theory][h->prec];
    int cur = 0, arrested = 0;
    int rc;
    size_t sz = h->prec ? sizeof(InstDesc<double>) : sizeof(InstDesc<float>);
    size_t ocur = h->prec ? offsetof(InstDesc<double>, cur) : offsetof(InstDesc<float>, cur);
    size_t oarr = h->prec ? offsetof(InstDesc<double>, arrested) : offsetof(InstDesc<float>, arrested);
    char* base = reinterpret_cast<char*>(g.d_desc) + sz * h->group_slot;
    cudaMemcpyAsync(&cur, base + ocur, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    cudaMemcpyAsync(&arrested, base + oarr, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
    if ((rc = check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__))) return rc;
    const int64_t n = (int64_t)h->C * h->N;
    double* tmp = nullptr;
    if (!on_device && (rc = check_cuda(cudaMalloc(&tmp, sizeof(double) * n), "cudaMalloc(read)", __LINE__)))
        return rc;
    double* outs[2] = {field, velocity};
    const void* srcs[2] = {h->F[cur], h->V[cur]};
    for (int k = 0; k < 2 && rc == SKY_OK; ++k) {
        if (!outs[k]) continue;
        double* dst = on_device ? outs[k] : tmp;
        const int zero = (k == 1 && arrested) ? 1 : 0;  // the reference zeroes V on arrest
        if (h->prec)
            k_convert_out<double><<<ew_blocks(n), 256, 0, e->stream>>>(n, (const double*)srcs[k], dst, zero);
        else if (k == 0 && h->comp)
            k_f32c_to_f64<<<ew_blocks(n), 256, 0, e->stream>>>(n, (const float*)srcs[k], (const float*)h->Flo[cur],
                                                               dst, 0);
        else
            k_convert_out<float><<<ew_blocks(n), 256, 0, e->stream>>>(n, (const float*)srcs[k], dst, zero);
        rc = check_cuda(cudaGetLastError(), "convert out", __LINE__);
        if (!rc && !on_device)
            rc = check_cuda(cudaMemcpyAsync(outs[k], tmp, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream),
                            "download", __LINE__);
        if (!rc) rc = check_cuda(cudaStreamSynchronize(e->stream), "sync", __LINE__);
    }
    if (tmp) cudaFree(tmp);
    return rc;
}

int sky_engine_time_stages(void* handle, int nsteps, double* ms_out) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    if (!e || !ms_out) return invalid("null argument");
    if (nsteps < 1) return invalid("nsteps must be >= 1");
    cudaSetDevice(e->device);
    int rc = SKY_OK;
    for (int t = 0; t < 6; ++t)
        for (int pr = 0; pr < 2; ++pr)
            if (!e->groups[t][pr].members.empty() && (rc = setup_group(e->groups[t][pr]))) return rc;
    cudaEvent_t ev[kNumKinds + 1];
    for (int k = 0; k <= kNumKinds; ++k)
        if ((rc = check_cuda(cudaEventCreate(&ev[k]), "cudaEventCreate", __LINE__))) return rc;
    double acc[kNumKinds] = {0.0};
    for (int s = 0; s < nsteps && rc == SKY_OK; ++s) {
        for (int k = 0; k < kNumKinds && rc == SKY_OK; ++k) {
            cudaEventRecord(ev[k], e->stream);
            rc = launch_kind(*e, k);
        }
        if (rc) break;
        cudaEventRecord(ev[kNumKinds], e->stream);
        if ((rc = check_cuda(cudaEventSynchronize(ev[kNumKinds]), "cudaEventSynchronize", __LINE__))) break;
        for (int k = 0; k < kNumKinds; ++k) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            acc[k] += ms;
        }
    }
    for (int k = 0; k <= kNumKinds; ++k) cudaEventDestroy(ev[k]);
    if (rc) return rc;
    for (auto& kv : e->insts)
        if (kv.second.active) kv.second.steps += nsteps;
    // report in the order stage 1, 2, 3, 4, control, advance
    ms_out[0] = (acc[kKindS1] + acc[kKindDefect]) / nsteps;  // stage 1 with the defect refresh
    ms_out[1] = acc[kKindS2] / nsteps;
    ms_out[2] = acc[kKindS3] / nsteps;
    ms_out[3] = acc[kKindS4] / nsteps;
    ms_out[4] = 0.0;  // the control and the advance run inside stages 1 and 4
    ms_out[5] = 0.0;
    return SKY_OK;
}

int sky_engine_launches_per_step(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    return e ? count_launches(*e) : 0;
}

int sky_engine_count(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    return e ? (int)e->insts.size() : 0;
}

int64_t sky_engine_bytes(void* handle) {
    Engine* e = reinterpret_cast<Engine*>(handle);
    return e ? e->bytes : 0;
}

}  // extern "C"
