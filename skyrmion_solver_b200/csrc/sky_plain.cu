// Reference-layout FP64 C ABI: drop-in replacements for the reference's
// per-theory Numba kernels and host reductions (declared in
// include/skyrmion_b200.h, which cites the reference interface of each).
#include <stdio.h>
#include <string.h>

#include "sky_host.h"
#include "sky_kernels.cuh"
#include "sky_march.cuh"

namespace sky {

// ---------------------------------------------------------------------------
// element-wise kernels (grid-stride over sites; z fastest => coalesced)
// ---------------------------------------------------------------------------

// do_rk4_step_kernel (core/integrator.py:50-92)
__global__ void k_rk4_stage(int64_t total, double dt, double factor, double* __restrict__ kout,
                            const double* __restrict__ v, const double* __restrict__ lin, double* __restrict__ temp,
                            const double* __restrict__ f, const double* __restrict__ kprev) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        kout[i] = dt * (v[i] + factor * lin[i]);
        temp[i] = f[i] + factor * kprev[i];
    }
}

// _do_rk4_kernel (core/integrator.py:163-175) with compute_norm_skyrme_field /
// project_orthogonal_skyrme_field (th/nuclear_skyrme/kernels.py:196-272) over
// the first nsky components; constrain = 0 gives do_rk4_kernel_no_constraint.
template <int C>
__global__ void k_rk4_finalize(int64_t N, int nsky, int constrain, double* __restrict__ v, double* __restrict__ f,
                               const double* __restrict__ k1, const double* __restrict__ k2,
                               const double* __restrict__ k3, const double* __restrict__ k4,
                               const double* __restrict__ l1, const double* __restrict__ l2,
                               const double* __restrict__ l3, const double* __restrict__ l4) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        double fv[C], vv[C];
#pragma unroll
        for (int a = 0; a < C; ++a) {
            const int64_t i = a * N + s;
            vv[a] = v[i] + (1.0 / 6.0) * (l1[i] + 2.0 * l2[i] + 2.0 * l3[i] + l4[i]);
            fv[a] = f[i] + (1.0 / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
        }
        if (constrain) {
            double ss = 0.0;
#pragma unroll
            for (int a = 0; a < C; ++a)
                if (a < nsky) ss += fv[a] * fv[a];
            ss = sqrt(ss);
            if (ss != 0.0) {
#pragma unroll
                for (int a = 0; a < C; ++a)
                    if (a < nsky) fv[a] /= ss;
            }
            double lm = 0.0;
#pragma unroll
            for (int a = 0; a < C; ++a)
                if (a < nsky) lm += vv[a] * fv[a];
#pragma unroll
            for (int a = 0; a < C; ++a)
                if (a < nsky) vv[a] -= lm * fv[a];
        }
#pragma unroll
        for (int a = 0; a < C; ++a) {
            v[a * N + s] = vv[a];
            f[a * N + s] = fv[a];
        }
    }
}

// Generic-C variant for the unconstrained fallback with arbitrary component count.
__global__ void k_rk4_finalize_any(int64_t total, double* __restrict__ v, double* __restrict__ f,
                                   const double* __restrict__ k1, const double* __restrict__ k2,
                                   const double* __restrict__ k3, const double* __restrict__ k4,
                                   const double* __restrict__ l1, const double* __restrict__ l2,
                                   const double* __restrict__ l3, const double* __restrict__ l4) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        v[i] += (1.0 / 6.0) * (l1[i] + 2.0 * l2[i] + 2.0 * l3[i] + l4[i]);
        f[i] += (1.0 / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
    }
}

__global__ void k_fill(int64_t total, double* __restrict__ a, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

__global__ void k_copy_comp(int64_t N, double* __restrict__ en, const double* __restrict__ src) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        en[i] = src[i];
}

// compute_rho_meson_kernel (th/rho_skyrme/kernels.py:385-412): accumulates onto en.
__global__ void k_rho_meson(int64_t N, int C, double* __restrict__ en, const double* __restrict__ f) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        double e = en[s];
        for (int a = 4; a < C; ++a) {
            const double v = f[a * N + s];
            e += v * v;
        }
        en[s] = e;
    }
}

// create_grid_kernel (th/nuclear_skyrme/kernels.py:27-56)
__global__ void k_create_grid(int X, int Y, int Z, double hx, double hy, double hz, double* __restrict__ grid) {
    const int64_t N = (int64_t)X * Y * Z;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(s % Z);
        const int64_t r = s / Z;
        const int y = (int)(r % Y);
        const int x = (int)(r / Y);
        grid[s] = hx * (double)x;
        grid[N + s] = hy * (double)y;
        grid[2 * N + s] = hz * (double)z;
    }
}

// compute_sum / compute_max (core/utils.py:201-279): compensated sum, signed max.
__global__ void __launch_bounds__(256) k_sum(const double* __restrict__ v, int64_t n, double* __restrict__ scratch,
                                             double* __restrict__ out_dev) {
    __shared__ KSum shk[32];
    KSum acc{0.0, 0.0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        ksum_add(acc, v[i]);
    finish_ksum(acc, scratch, out_dev, shk);
}

__global__ void __launch_bounds__(256) k_max(const double* __restrict__ v, int64_t n, double* __restrict__ scratch,
                                             double* __restrict__ out_dev) {
    __shared__ double shm[32];
    double acc = -1.0e300;  // padding value of reduce_max_kernel (core/utils.py:267)
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc = fmax(acc, v[i]);
    finish_max(acc, scratch, out_dev, shm);
}

// compute_min (core/utils.py:282-319, 375-400) as the negated maximum of the negated
// values: exact, and +1e300 padding becomes the maximum's -1e300.
__global__ void __launch_bounds__(256) k_min(const double* __restrict__ v, int64_t n, double* __restrict__ scratch,
                                             double* __restrict__ out_dev) {
    __shared__ double shm[32];
    double acc = -1.0e300;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc = fmax(acc, -v[i]);
    finish_max(acc, scratch, out_dev, shm, -1.0);
}

// arresting_criteria_kernel + arresting_criteria (core/integrator.py:178-282): per site
// the power V . EG over the C components (summed in component order), optionally stored
// in en, and its compensated sum over the lattice.
__global__ void __launch_bounds__(256) k_power(const double* __restrict__ vel, const double* __restrict__ eg,
                                               int64_t N, int C, double* __restrict__ en,
                                               double* __restrict__ scratch, double* __restrict__ out_dev) {
    __shared__ KSum shk[32];
    KSum acc{0.0, 0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        double f = 0.0;
        for (int a = 0; a < C; ++a) f += vel[a * N + s] * eg[a * N + s];
        if (en) en[s] = f;
        ksum_add(acc, f);
    }
    finish_ksum(acc, scratch, out_dev, shk);
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

void set_error(const char* fmt, const char* a, int line) {
    snprintf(g_err, sizeof(g_err), fmt, a, line);
}

int check_cuda(cudaError_t e, const char* what, int line) {
    if (e == cudaSuccess) return SKY_OK;
    snprintf(g_err, sizeof(g_err), "%s (line %d): %s", what, line, cudaGetErrorString(e));
    return SKY_ERR_CUDA;
}

int invalid(const char* msg) {
    snprintf(g_err, sizeof(g_err), "invalid argument: %s", msg);
    return SKY_ERR_INVALID;
}

int fail(int code, const char* msg) {
    snprintf(g_err, sizeof(g_err), "%s", msg);
    return code;
}

const char* last_error() { return g_err; }

int theory_components(int theory) {
    switch (theory) {
        case SKY_THEORY_NUCLEAR: return 4;
        case SKY_THEORY_OMEGA: return 5;
        case SKY_THEORY_COULOMB: return 5;
        case SKY_THEORY_RHO: return 13;
        case SKY_THEORY_BERGER: return 4;
        case SKY_THEORY_LIGHTLY_BOUND: return 4;
        default: return -1;
    }
}

// Core p_i / p_f checks shared by every entry point.
int pack_core(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, Params* out, bool need_f) {
    if (!p_i || n_pi < 11) return invalid("p_i must hold at least 11 entries");
    if (need_f && (!p_f || n_pf < 8)) return invalid("p_f must hold at least 8 entries");
    Params q;
    memset(&q, 0, sizeof(q));
    q.X = p_i[0];
    q.Y = p_i[1];
    q.Z = p_i[2];
    q.halo = p_i[3];
    q.C = p_i[5];
    q.nsky = p_i[5];
    q.killkinen = p_i[8];
    q.unit_length = p_i[10];
    if (q.X < 1 || q.Y < 1 || q.Z < 1) return invalid("grid dimensions must be positive");
    if (p_i[4] != 3) return invalid("number_coordinates (p_i[4]) must be 3");
    if (q.C < 1) return invalid("number_total_fields (p_i[5]) must be positive");
    if ((int64_t)p_i[6] != (int64_t)q.X * q.Y * q.Z) return invalid("dim_grid (p_i[6]) != xlen*ylen*zlen");
    if ((int64_t)p_i[7] != (int64_t)q.C * q.X * q.Y * q.Z) return invalid("dim_fields (p_i[7]) != nfields*dim_grid");
    if (need_f) {
        q.hx = p_f[3];
        q.hy = p_f[4];
        q.hz = p_f[5];
        q.vol = p_f[6];
        q.dt = p_f[7];
    }
    *out = q;
    return SKY_OK;
}

int pack_params(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, Params* out) {
    int st = pack_core(p_i, n_pi, p_f, n_pf, out, true);
    if (st) return st;
    Params& q = *out;
    const int C = theory_components(theory);
    if (C < 0) return invalid("unknown theory id");
    if (q.C != C) return invalid("number_total_fields does not match the theory's component count");
    if (q.halo < 2) return invalid("halo (p_i[3]) must be >= 2 for the 5-point stencils");
    if (!(q.hx > 0.0) || !(q.hy > 0.0) || !(q.hz > 0.0)) return invalid("lattice spacings must be positive");
    switch (theory) {
        case SKY_THEORY_NUCLEAR:  // th/nuclear_skyrme/params.py:203-245: mpi = p_f[8], kappa = p_f[9]
            if (n_pf < 10) return invalid("nuclear p_f needs mpi, kappa at [8], [9]");
            q.nsky = p_i[5];
            q.c0 = p_f[8];
            q.c1 = p_f[9];
            break;
        case SKY_THEORY_OMEGA:  // th/omega_skyrme/params.py: p_i[11] = nsky, mass = p_f[8], c_omega = p_f[9]
        case SKY_THEORY_COULOMB:  // th/coulomb_skyrme/params.py: p_i[11] = nsky, mass, kappa
            if (n_pi < 12 || n_pf < 10) return invalid("omega/coulomb need p_i[11] and p_f[8..9]");
            q.nsky = p_i[11];
            q.c0 = p_f[8];
            q.c1 = p_f[9];
            break;
        case SKY_THEORY_RHO:  // th/rho_skyrme/params.py: mpi, mrho, c_alpha = p_f[8..10]; nsky literal 4
            if (n_pf < 11) return invalid("rho p_f needs mpi, mrho, c_alpha at [8..10]");
            q.nsky = 4;
            q.c0 = p_f[8];
            q.c1 = p_f[9];
            q.c2 = p_f[10];
            break;
        case SKY_THEORY_BERGER:  // th/berger_skyrme/params.py: mpi, kappa = p_f[8], p_f[9]; alpha = p_f[12]
            if (n_pf < 13) return invalid("berger p_f needs alpha at [12]");
            q.nsky = p_i[5];
            q.c0 = p_f[8];
            q.c1 = p_f[9];
            q.c2 = p_f[12];
            break;
        case SKY_THEORY_LIGHTLY_BOUND:  // th/lightly_bound_skyrme/params.py: mpi, alpha = p_f[8], p_f[9]
            if (n_pf < 10) return invalid("lightly-bound p_f needs mpi, alpha at [8], [9]");
            q.nsky = p_i[5];
            q.c0 = p_f[8];
            q.c1 = p_f[9];
            break;
    }
    if (q.nsky < 0 || q.nsky > q.C) return invalid("number of Skyrme components out of range");
    return SKY_OK;
}

static int g_num_sms = 0;

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        g_num_sms = n;
    }
    return g_num_sms;
}

int ew_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    const int64_t cap = (int64_t)num_sms() * 16;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// x-chunk of a marching launch: minimise (waves of tiles over the resident
// blocks) x (planes a block walks: chunk + 4 halo planes).
int choose_xc(int X, int tiles_yz, int resident) {
    int best = X, best_cost = -1;
    for (int xc = 4; xc <= X; ++xc) {
        const int nt = tiles_yz * ((X + xc - 1) / xc);
        const int waves = (nt + resident - 1) / resident;
        const int cost = waves * (xc + 4);
        if (best_cost < 0 || cost < best_cost || (cost == best_cost && xc > best)) {
            best_cost = cost;
            best = xc;
        }
    }
    return best;
}

// Library options (sky_set_option): key 0 = kernel family of the
// reference-layout gradient and densities (1 = marching kernels, 0 = 3-D tile
// kernels); key 1 = x-chunk of those marching launches (0 = automatic); key 2 =
// staging of the engine's stage kernels (1 = TMA box copies, 0 = cp.async); key 3 =
// z-pair tiles for the FP32 stages of theories without mixed derivatives (1 = on; off
// by default: on the omega 128^3 stages they issue a third fewer instructions per site
// but run at half the resident warps, and measured no faster).
static int g_options[5] = {1, 0, 1, 0, 0};
int option(int key) { return (key >= 0 && key < 5) ? g_options[key] : 0; }

// ---------------------------------------------------------------------------
// templated launchers
// ---------------------------------------------------------------------------
// BY = 8-row tiles, or 4 for FP64 rho (13 components), whose 8-row ring would
// not fit in shared memory.
template <template <typename> class Th, typename T, bool WIDE, int BY = 8>
int launch_gradient_march(const Params& p, const T* field, T* eg, T* l, cudaStream_t st) {
    using M = MarchShape<Th<T>::C, BY, WIDE>;
    auto kern = k_march_plain<Th, M, T>;
    const size_t smem = M::template smem_bytes<T>(1);
    static int per_sm = 0;
    if (per_sm == 0) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(march gradient)", __LINE__);
        if (rc) return rc;
        int n = 0;
        rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, M::NTHREADS, smem), "occupancy",
                        __LINE__);
        if (rc) return rc;
        per_sm = n < 1 ? 1 : n;
    }
    const int resident = num_sms() * per_sm;
    const MarchGrid g0 = march_grid<M>(p, p.X);
    const int xc_opt = option(1);
    const int xc = xc_opt > 0 ? (xc_opt < p.X ? xc_opt : p.X) : choose_xc(p.X, g0.nz * g0.ny, resident);
    const MarchGrid mg = march_grid<M>(p, xc);
    const int blocks = mg.count() < resident ? mg.count() : resident;
    kern<<<blocks, dim3(M::BZ, M::BY), smem, st>>>(p, mg, field, eg, l);
    return check_cuda(cudaGetLastError(), "launch march gradient", __LINE__);
}
template <template <typename> class Th, typename T, typename S>
int launch_gradient(const Params& p, const S* field, S* eg, S* l, cudaStream_t st) {
    using Shape = typename GradTile<Th<T>::C, T>::type;
    auto kern = k_gradient<Th, Shape, T, S>;
    const size_t smem = Shape::template smem_bytes<T>();
    static bool attr_done = false;  // one per instantiation
    if (!attr_done) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(gradient)", __LINE__);
        if (rc) return rc;
        attr_done = true;
    }
    const TileGrid tg = tile_grid<Shape>(p);
    int blocks = tg.count();
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Shape::NTHREADS, smem);
    if (per_sm < 1) per_sm = 1;
    const int cap = num_sms() * per_sm;
    if (blocks > cap) blocks = cap;
    kern<<<blocks, dim3(Shape::BZ, Shape::BY), smem, st>>>(p, field, eg, l);
    return check_cuda(cudaGetLastError(), "launch gradient", __LINE__);
}

template <template <typename> class Th, int MODE, typename S>
int launch_density(const Params& p, const S* field, double* dens, double* scratch, double* out_dev, cudaStream_t st) {
    using Shape = typename DensTile<Th<double>::C>::type;
    constexpr int CL = (MODE == 0) ? Th<double>::C : 4;
    auto kern = k_density<Th, Shape, MODE, S>;
    const size_t smem = size_t(CL) * Shape::VOL * sizeof(double);
    static bool attr_done = false;
    if (!attr_done) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(density)", __LINE__);
        if (rc) return rc;
        attr_done = true;
    }
    const TileGrid tg = tile_grid<Shape>(p);
    int blocks = tg.count();
    if (blocks > kMaxRedBlocks) blocks = kMaxRedBlocks;
    if (scratch) {
        int rc = check_cuda(cudaMemsetAsync(scratch + 2 * kMaxRedBlocks + 1, 0, sizeof(double), st), "memset",
                            __LINE__);
        if (rc) return rc;
    }
    kern<<<blocks, dim3(Shape::BZ, Shape::BY), smem, st>>>(p, field, dens, scratch, out_dev);
    return check_cuda(cudaGetLastError(), "launch density", __LINE__);
}

#define SKY_DISPATCH(theory, FN, ...)                                         \
    switch (theory) {                                                         \
        case SKY_THEORY_NUCLEAR: return FN<Nuclear>(__VA_ARGS__);            \
        case SKY_THEORY_OMEGA: return FN<Omega>(__VA_ARGS__);                \
        case SKY_THEORY_COULOMB: return FN<Coulomb>(__VA_ARGS__);            \
        case SKY_THEORY_RHO: return FN<Rho>(__VA_ARGS__);                    \
        case SKY_THEORY_BERGER: return FN<Berger>(__VA_ARGS__);              \
        case SKY_THEORY_LIGHTLY_BOUND: return FN<LightlyBound>(__VA_ARGS__); \
        default: return invalid("unknown theory id");                        \
    }

template <template <typename> class Th>
int grad64(const Params& p, const double* f, double* eg, double* l, cudaStream_t st) {
    if constexpr (Th<double>::C <= 5) {
        if (option(0) == 1 && (int64_t)p.C * n_sites(p) < ((int64_t)1 << 31)) {
            // 16-byte staging needs a 16-byte aligned field and Z a multiple of two doubles
            if (p.Z % 2 == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0)
                return launch_gradient_march<Th, double, true>(p, f, eg, l, st);
            return launch_gradient_march<Th, double, false>(p, f, eg, l, st);
        }
    } else {
        if (option(0) == 1 && (int64_t)p.C * n_sites(p) < ((int64_t)1 << 31))
            return launch_gradient_march<Th, double, false, 4>(p, f, eg, l, st);
    }
    return launch_gradient<Th, double, double>(p, f, eg, l, st);
}
// Marching FP64 density with its fused compensated sum (energy: all components,
// in 4-row tiles for rho; baryon: phi_0..3 of any theory).
template <template <typename> class Th, int MODE, bool WIDE, int BY = 8>
int launch_density_march(const Params& p, const double* field, double* dens, double* scratch, double* out_dev,
                         cudaStream_t st) {
    using M = MarchShape<(MODE == 0 ? Th<double>::C : 4), BY, WIDE>;
    auto kern = k_march_density<Th, M, MODE>;
    const size_t smem = M::template smem_bytes<double>(1);
    static int per_sm = 0;
    if (per_sm == 0) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(march density)", __LINE__);
        if (rc) return rc;
        int n = 0;
        rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, M::NTHREADS, smem), "occupancy",
                        __LINE__);
        if (rc) return rc;
        per_sm = n < 1 ? 1 : n;
    }
    int resident = num_sms() * per_sm;
    if (resident > kMaxRedBlocks) resident = kMaxRedBlocks;
    const MarchGrid g0 = march_grid<M>(p, p.X);
    const MarchGrid mg = march_grid<M>(p, choose_xc(p.X, g0.nz * g0.ny, resident));
    const int blocks = mg.count() < resident ? mg.count() : resident;
    if (scratch) {
        int rc = check_cuda(cudaMemsetAsync(scratch + 2 * kMaxRedBlocks + 1, 0, sizeof(double), st), "memset",
                            __LINE__);
        if (rc) return rc;
    }
    kern<<<blocks, dim3(M::BZ, M::BY), smem, st>>>(p, mg, field, dens, scratch, out_dev);
    return check_cuda(cudaGetLastError(), "launch march density", __LINE__);
}

template <template <typename> class Th, int MODE>
int density_march(const Params& p, const double* f, double* dens, double* scratch, double* out_dev, cudaStream_t st) {
    if (p.Z % 2 == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0)
        return launch_density_march<Th, MODE, true>(p, f, dens, scratch, out_dev, st);
    return launch_density_march<Th, MODE, false>(p, f, dens, scratch, out_dev, st);
}

template <template <typename> class Th>
int dens64(const Params& p, int mode, const double* f, double* dens, double* scratch, double* out_dev,
           cudaStream_t st) {
    const bool march = option(0) == 1 && (int64_t)p.C * n_sites(p) < ((int64_t)1 << 31);
    if (march && mode == 1) return density_march<Th, 1>(p, f, dens, scratch, out_dev, st);
    if constexpr (Th<double>::C <= 5) {
        if (march) return density_march<Th, 0>(p, f, dens, scratch, out_dev, st);
    } else {
        if (march) return launch_density_march<Th, 0, false, 4>(p, f, dens, scratch, out_dev, st);
    }
    return mode == 0 ? launch_density<Th, 0, double>(p, f, dens, scratch, out_dev, st)
                     : launch_density<Th, 1, double>(p, f, dens, scratch, out_dev, st);
}

// Baryon moments (k_march_moments): at most kScratchDoubles / 18 blocks, so the
// per-block partials fit the standard reduction scratch.
template <template <typename> class Th>
int moments64(const Params& p, const double* f, double* scratch, double* out9, cudaStream_t st) {
    using M = MarchShape<4, 8, false>;
    auto kern = k_march_moments<Th, M>;
    const size_t smem = M::template smem_bytes<double>(1);
    static bool configured = false;
    if (!configured) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(moments)", __LINE__);
        if (rc) return rc;
        configured = true;
    }
    const int cap = kScratchDoubles / (2 * kMoments);
    const MarchGrid g0 = march_grid<M>(p, p.X);
    const MarchGrid mg = march_grid<M>(p, choose_xc(p.X, g0.nz * g0.ny, num_sms()));
    const int blocks = mg.count() < cap ? mg.count() : cap;
    kern<<<blocks, dim3(M::BZ, M::BY), smem, st>>>(p, mg, f, scratch);
    int rc = check_cuda(cudaGetLastError(), "launch moments", __LINE__);
    if (rc) return rc;
    double parts[2 * kMoments * (kScratchDoubles / (2 * kMoments))];
    rc = check_cuda(cudaMemcpyAsync(parts, scratch, sizeof(double) * 2 * kMoments * blocks, cudaMemcpyDeviceToHost, st),
                    "read moments", __LINE__);
    if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "sync", __LINE__);
    if (rc) return rc;
    for (int q = 0; q < kMoments; ++q) {   // fixed-order compensated sum over the blocks
        double sum = 0.0, comp = 0.0;
        for (int b = 0; b < blocks; ++b) {
            for (int k = 0; k < 2; ++k) {
                const double v = parts[2 * kMoments * b + 2 * q + k];
                const double t = sum + v;
                comp += (fabs(sum) >= fabs(v)) ? ((sum - t) + v) : ((v - t) + sum);
                sum = t;
            }
        }
        out9[q] = sum + comp;
    }
    return SKY_OK;
}

// Nuclear diagnostics (k_march_diag): at most kScratchDoubles / 56 blocks.
int diag64(const Params& p, const double* f, const double* com, double* scratch, double* out28, cudaStream_t st) {
    using M = MarchShape<4, 8, false>;
    auto kern = k_march_diag<M>;
    const size_t smem = M::template smem_bytes<double>(1);
    static bool configured = false;
    if (!configured) {
        int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "cudaFuncSetAttribute(diagnostics)", __LINE__);
        if (rc) return rc;
        configured = true;
    }
    const int cap = kScratchDoubles / (2 * kDiag);
    const MarchGrid g0 = march_grid<M>(p, p.X);
    const MarchGrid mg = march_grid<M>(p, choose_xc(p.X, g0.nz * g0.ny, num_sms()));
    const int blocks = mg.count() < cap ? mg.count() : cap;
    kern<<<blocks, dim3(M::BZ, M::BY), smem, st>>>(p, mg, f, com[0], com[1], com[2], scratch);
    int rc = check_cuda(cudaGetLastError(), "launch diagnostics", __LINE__);
    if (rc) return rc;
    double parts[2 * kDiag * (kScratchDoubles / (2 * kDiag))];
    rc = check_cuda(cudaMemcpyAsync(parts, scratch, sizeof(double) * 2 * kDiag * blocks, cudaMemcpyDeviceToHost, st),
                    "read diagnostics", __LINE__);
    if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "sync", __LINE__);
    if (rc) return rc;
    for (int q = 0; q < kDiag; ++q) {   // fixed-order compensated sum over the blocks
        double sum = 0.0, comp = 0.0;
        for (int b = 0; b < blocks; ++b) {
            for (int k = 0; k < 2; ++k) {
                const double v = parts[2 * kDiag * b + 2 * q + k];
                const double t = sum + v;
                comp += (fabs(sum) >= fabs(v)) ? ((sum - t) + v) : ((v - t) + sum);
                sum = t;
            }
        }
        out28[q] = sum + comp;
    }
    return SKY_OK;
}

int gradient_fp64(int theory, const Params& p, const double* f, double* eg, double* l, cudaStream_t st) {
    SKY_DISPATCH(theory, grad64, p, f, eg, l, st)
}

int density_fp64(int theory, const Params& p, int mode, const double* f, double* dens, double* scratch,
                 double* out_dev, cudaStream_t st) {
    SKY_DISPATCH(theory, dens64, p, mode, f, dens, scratch, out_dev, st)
}

int rk4_stage(const Params& p, double* kout, const double* v, const double* lin, double* temp, const double* f,
              const double* kprev, double factor, cudaStream_t st) {
    const int64_t total = (int64_t)p.C * n_sites(p);
    k_rk4_stage<<<ew_blocks(total), 256, 0, st>>>(total, p.dt, factor, kout, v, lin, temp, f, kprev);
    return check_cuda(cudaGetLastError(), "launch rk4_stage", __LINE__);
}

int rk4_finalize(int theory, const Params& p, double* v, double* f, const double* k1, const double* k2,
                 const double* k3, const double* k4, const double* l1, const double* l2, const double* l3,
                 const double* l4, cudaStream_t st) {
    const int64_t N = n_sites(p);
    const int constrain = p.unit_length ? 1 : 0;
    if (theory < 0) {
        const int64_t total = (int64_t)p.C * N;
        k_rk4_finalize_any<<<ew_blocks(total), 256, 0, st>>>(total, v, f, k1, k2, k3, k4, l1, l2, l3, l4);
    } else {
        switch (theory_components(theory)) {
            case 4:
                k_rk4_finalize<4><<<ew_blocks(N), 256, 0, st>>>(N, p.nsky, constrain, v, f, k1, k2, k3, k4, l1, l2,
                                                                l3, l4);
                break;
            case 5:
                k_rk4_finalize<5><<<ew_blocks(N), 256, 0, st>>>(N, p.nsky, constrain, v, f, k1, k2, k3, k4, l1, l2,
                                                                l3, l4);
                break;
            case 13:
                k_rk4_finalize<13><<<ew_blocks(N), 256, 0, st>>>(N, p.nsky, constrain, v, f, k1, k2, k3, k4, l1, l2,
                                                                 l3, l4);
                break;
            default: return invalid("unknown theory id");
        }
    }
    return check_cuda(cudaGetLastError(), "launch rk4_finalize", __LINE__);
}

int fill(double* a, int64_t n, double v, cudaStream_t st) {
    k_fill<<<ew_blocks(n), 256, 0, st>>>(n, a, v);
    return check_cuda(cudaGetLastError(), "launch fill", __LINE__);
}

int reduce(int kind, const double* v, int64_t n, double* scratch, double* out_dev, cudaStream_t st) {
    int64_t b = (n + 1023) / 1024;
    if (b > kMaxRedBlocks) b = kMaxRedBlocks;
    if (b < 1) b = 1;
    int rc = check_cuda(cudaMemsetAsync(scratch + 2 * kMaxRedBlocks + 1, 0, sizeof(double), st), "memset", __LINE__);
    if (rc) return rc;
    if (kind == 0)
        k_sum<<<(int)b, 256, 0, st>>>(v, n, scratch, out_dev);
    else if (kind == 1)
        k_max<<<(int)b, 256, 0, st>>>(v, n, scratch, out_dev);
    else
        k_min<<<(int)b, 256, 0, st>>>(v, n, scratch, out_dev);
    return check_cuda(cudaGetLastError(), "launch reduce", __LINE__);
}

int read_result(double* scratch, double* out_host, cudaStream_t st) {
    int rc = check_cuda(cudaMemcpyAsync(out_host, scratch + 2 * kMaxRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, st),
                        "cudaMemcpyAsync(result)", __LINE__);
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize", __LINE__);
}

}  // namespace sky

using namespace sky;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* sky_version(void) { return "skyrmion_b200 0.2 (sm_100a)"; }

int sky_set_option(int key, int value) {
    if (key == 0 && value != 0 && value != 1) return invalid("option 0 takes 0 (tile kernels) or 1 (marching kernels)");
    if (key == 1 && value < 0) return invalid("option 1 (x-chunk) must be >= 0");
    if (key == 2 && value != 0 && value != 1) return invalid("option 2 takes 0 (cp.async staging) or 1 (TMA staging)");
    if (key == 3 && value != 0 && value != 1) return invalid("option 3 takes 0 (one site per thread) or 1 (z-pairs)");
    if (key == 4 && value != 0 && value != 1)
        return invalid("option 4 takes 0 (stream order) or 1 (programmatic dependent launch)");
    if (key < 0 || key > 4) return invalid("unknown option key");
    g_options[key] = value;
    return SKY_OK;
}

int sky_get_option(int key) { return option(key); }
const char* sky_last_error(void) { return last_error(); }
int sky_theory_components(int theory) { return theory_components(theory); }
int64_t sky_reduce_scratch_size(int64_t n) {
    (void)n;
    return kScratchDoubles;
}

#define SKY_STREAM(s) reinterpret_cast<cudaStream_t>(s)

int sky_gradient_step(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* l_out,
                      const double* field, double* energy_gradient, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!l_out || !field || !energy_gradient) return invalid("null buffer");
    return gradient_fp64(theory, p, field, energy_gradient, l_out, SKY_STREAM(stream));
}

int sky_rk4_stage(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* k_out,
                  const double* velocity, const double* l_in, double* temp, const double* field, const double* k_prev,
                  double factor, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, p_f, n_pf, &p, true);
    if (rc) return rc;
    if (!k_out || !velocity || !l_in || !temp || !field || !k_prev) return invalid("null buffer");
    return rk4_stage(p, k_out, velocity, l_in, temp, field, k_prev, factor, SKY_STREAM(stream));
}

int sky_rk4_finalize(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* velocity,
                     double* field, const double* k1, const double* k2, const double* k3, const double* k4,
                     const double* l1, const double* l2, const double* l3, const double* l4, void* stream) {
    Params p;
    int rc = theory < 0 ? pack_core(p_i, n_pi, p_f, n_pf, &p, false) : pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!velocity || !field || !k1 || !k2 || !k3 || !k4 || !l1 || !l2 || !l3 || !l4) return invalid("null buffer");
    return rk4_finalize(theory, p, velocity, field, k1, k2, k3, k4, l1, l2, l3, l4, SKY_STREAM(stream));
}

int sky_energy_density(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* en,
                       const double* field, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!en || !field) return invalid("null buffer");
    return density_fp64(theory, p, 0, field, en, nullptr, nullptr, SKY_STREAM(stream));
}

int sky_baryon_density(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* en,
                       const double* field, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!en || !field) return invalid("null buffer");
    return density_fp64(theory, p, 1, field, en, nullptr, nullptr, SKY_STREAM(stream));
}

int sky_potential_density(const int32_t* p_i, int32_t n_pi, double* en, const double* field, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, nullptr, 0, &p, false);
    if (rc) return rc;
    if (n_pi < 12) return invalid("potential density needs p_i[11]");
    const int comp = p_i[11];
    if (comp < 0 || comp >= p.C) return invalid("p_i[11] out of range");
    if (!en || !field) return invalid("null buffer");
    const int64_t N = n_sites(p);
    k_copy_comp<<<ew_blocks(N), 256, 0, SKY_STREAM(stream)>>>(N, en, field + comp * N);
    return check_cuda(cudaGetLastError(), "launch potential", __LINE__);
}

int sky_rho_meson_density(const int32_t* p_i, int32_t n_pi, double* en, const double* field, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, nullptr, 0, &p, false);
    if (rc) return rc;
    if (!en || !field) return invalid("null buffer");
    const int64_t N = n_sites(p);
    k_rho_meson<<<ew_blocks(N), 256, 0, SKY_STREAM(stream)>>>(N, p.C, en, field);
    return check_cuda(cudaGetLastError(), "launch rho_meson", __LINE__);
}

int sky_set_field_zero(const int32_t* p_i, int32_t n_pi, double* field, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, nullptr, 0, &p, false);
    if (rc) return rc;
    if (!field) return invalid("null buffer");
    return fill(field, (int64_t)p.C * n_sites(p), 0.0, SKY_STREAM(stream));
}

int sky_create_grid(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, double* grid, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, p_f, n_pf, &p, true);
    if (rc) return rc;
    if (!grid) return invalid("null buffer");
    const int64_t N = n_sites(p);
    k_create_grid<<<ew_blocks(N), 256, 0, SKY_STREAM(stream)>>>(p.X, p.Y, p.Z, p.hx, p.hy, p.hz, grid);
    return check_cuda(cudaGetLastError(), "launch create_grid", __LINE__);
}

static int reduce_entry(int kind, const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host,
                        double* out_dev, void* stream) {
    if (!values || n < 1) return invalid("empty reduction input");
    if (!scratch || n_scratch < kScratchDoubles) return SKY_ERR_NOMEM;
    cudaStream_t st = SKY_STREAM(stream);
    int rc = reduce(kind, values, n, scratch, out_dev, st);
    if (rc) return rc;
    if (out_host) return read_result(scratch, out_host, st);
    return SKY_OK;
}

int sky_sum(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host, double* out_dev,
            void* stream) {
    return reduce_entry(0, values, n, scratch, n_scratch, out_host, out_dev, stream);
}

int sky_max(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host, double* out_dev,
            void* stream) {
    return reduce_entry(1, values, n, scratch, n_scratch, out_host, out_dev, stream);
}

int sky_min(const double* values, int64_t n, double* scratch, int64_t n_scratch, double* out_host, double* out_dev,
            void* stream) {
    return reduce_entry(2, values, n, scratch, n_scratch, out_host, out_dev, stream);
}

int sky_arresting_criteria(const int32_t* p_i, int32_t n_pi, const double* velocity, const double* energy_gradient,
                           double* en, double* scratch, int64_t n_scratch, double* out_host, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, nullptr, 0, &p, false);
    if (rc) return rc;
    if (!velocity || !energy_gradient) return invalid("null buffer");
    if (!scratch || n_scratch < kScratchDoubles) return SKY_ERR_NOMEM;
    cudaStream_t st = SKY_STREAM(stream);
    const int64_t N = n_sites(p);
    int64_t b = (N + 1023) / 1024;
    if (b > kMaxRedBlocks) b = kMaxRedBlocks;
    rc = check_cuda(cudaMemsetAsync(scratch + 2 * kMaxRedBlocks + 1, 0, sizeof(double), st), "memset", __LINE__);
    if (rc) return rc;
    k_power<<<(int)b, 256, 0, st>>>(velocity, energy_gradient, N, p.C, en, scratch, nullptr);
    rc = check_cuda(cudaGetLastError(), "launch arresting criteria", __LINE__);
    if (rc || !out_host) return rc;
    return read_result(scratch, out_host, st);
}

static int total_entry(int mode, int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                       const double* field, double* scratch, int64_t n_scratch, double* out_host, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!field) return invalid("null buffer");
    if (!scratch || n_scratch < kScratchDoubles) return SKY_ERR_NOMEM;
    cudaStream_t st = SKY_STREAM(stream);
    rc = density_fp64(theory, p, mode, field, nullptr, scratch, nullptr, st);
    if (rc) return rc;
    if (out_host) return read_result(scratch, out_host, st);
    return SKY_OK;
}

int sky_total_energy(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                     const double* field, double* scratch, int64_t n_scratch, double* out_host, void* stream) {
    return total_entry(0, theory, p_i, n_pi, p_f, n_pf, field, scratch, n_scratch, out_host, stream);
}

int sky_total_baryon(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                     const double* field, double* scratch, int64_t n_scratch, double* out_host, void* stream) {
    return total_entry(1, theory, p_i, n_pi, p_f, n_pf, field, scratch, n_scratch, out_host, stream);
}

int sky_baryon_moments(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                       const double* field, double* scratch, int64_t n_scratch, double* out9_host, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!field || !out9_host) return invalid("null buffer");
    if (!scratch || n_scratch < kScratchDoubles) return SKY_ERR_NOMEM;
    if ((int64_t)4 * n_sites(p) >= ((int64_t)1 << 31)) return invalid("lattice too large for the moments kernel");
    SKY_DISPATCH(theory, moments64, p, field, scratch, out9_host, SKY_STREAM(stream))
}

int sky_nuclear_diagnostics(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                            const double* field, const double* com_host, double* scratch, int64_t n_scratch,
                            double* out28_host, void* stream) {
    Params p;
    int rc = pack_params(SKY_THEORY_NUCLEAR, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!field || !com_host || !out28_host) return invalid("null buffer");
    if (!scratch || n_scratch < kScratchDoubles) return SKY_ERR_NOMEM;
    if ((int64_t)4 * n_sites(p) >= ((int64_t)1 << 31)) return invalid("lattice too large for the diagnostics kernel");
    return diag64(p, field, com_host, scratch, out28_host, SKY_STREAM(stream));
}

int sky_arrested_newton_step(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf,
                             double* velocity, double* field, double* energy_gradient, double* k1, double* k2,
                             double* k3, double* k4, double* l1, double* l2, double* l3, double* l4, double* temp,
                             double* scratch, int64_t n_scratch, double prev_energy, double* new_energy_host,
                             double* err_host, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!velocity || !field || !energy_gradient || !k1 || !k2 || !k3 || !k4 || !l1 || !l2 || !l3 || !l4 || !temp)
        return invalid("null buffer");
    if (!new_energy_host || !err_host) return invalid("null host output");
    if (!scratch || n_scratch < 2 * kScratchDoubles) return SKY_ERR_NOMEM;
    cudaStream_t st = SKY_STREAM(stream);
    // core/integrator.py:382-398
    double* ks[4] = {k1, k2, k3, k4};
    double* ls[4] = {l1, l2, l3, l4};
    const double fac[4] = {0.0, 0.5, 0.5, 1.0};
    for (int s = 0; s < 4; ++s) {
        const double* lin = s == 0 ? velocity : ls[s - 1];
        const double* kprev = s == 0 ? field : ks[s - 1];
        if ((rc = rk4_stage(p, ks[s], velocity, lin, temp, field, kprev, fac[s], st))) return rc;
        if ((rc = gradient_fp64(theory, p, temp, energy_gradient, ls[s], st))) return rc;
    }
    if ((rc = rk4_finalize(theory, p, velocity, field, k1, k2, k3, k4, l1, l2, l3, l4, st))) return rc;
    // new energy (core/integrator.py:402) and err = signed max of the stage-4 EG (:409)
    double* s_e = scratch;
    double* s_m = scratch + kScratchDoubles;
    if ((rc = density_fp64(theory, p, 0, field, nullptr, s_e, nullptr, st))) return rc;
    if ((rc = reduce(1, energy_gradient, (int64_t)p.C * n_sites(p), s_m, nullptr, st))) return rc;
    double res[2];
    if ((rc = check_cuda(cudaMemcpyAsync(&res[0], s_e + 2 * kMaxRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, st),
                         "memcpy", __LINE__)))
        return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(&res[1], s_m + 2 * kMaxRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, st),
                         "memcpy", __LINE__)))
        return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(st), "sync", __LINE__))) return rc;
    *new_energy_host = res[0];
    *err_host = res[1];
    // arrest (core/integrator.py:403-407)
    if (p.killkinen && res[0] > prev_energy) {
        if ((rc = fill(velocity, (int64_t)p.C * n_sites(p), 0.0, st))) return rc;
    }
    return SKY_OK;
}

}  // extern "C"
