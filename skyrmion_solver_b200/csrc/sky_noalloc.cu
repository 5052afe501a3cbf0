// One arrested-Newton step that allocates no device memory.
//
// sky_arrested_newton_step needs, besides the caller's field, velocity and
// gradient buffers, eight RK4 slope buffers, a stage-field buffer and a
// reduction scratch buffer.  Some callers cannot provide those: a plugin that
// only receives the field and velocity arrays of a host application whose
// allocator owns the device memory budget (a pooling framework that forbids
// raw cudaMalloc), or an interactive loop that must not call cudaMalloc /
// cudaFree between frames because they synchronise the whole device.  This
// variant keeps that working memory in one file-scope device array of fixed
// size that every GPU loading the library holds until the process exits.
#include <stdio.h>

#include <mutex>

#include "sky_host.h"
#include "sky_kernels.cuh"

namespace sky {

// 16 MiB of FP64 working memory: 9 * C * N doubles (k1..k4, l1..l4, stage
// field) plus two reduction scratch areas.
constexpr int64_t kNoAllocDoubles = (int64_t)2 * 1024 * 1024;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Device address of g_noalloc_scratch per device, looked up with that device
// current (host code must not use the symbol's name as an address).  The
// address belongs to the module loaded into the device's current context; after
// cudaDeviceReset (or any re-creation of the primary context) the module is
// loaded again, possibly elsewhere.  Each entry therefore records the unique id
// of the context it was looked up in (cuCtxGetId, reached through the runtime's
// driver entry points so that the library does not link libcuda), and a call
// in a different context looks the address up again.
typedef int (*PfnCtxGetCurrent)(void** ctx);
typedef int (*PfnCtxGetId)(void* ctx, unsigned long long* id);

struct NoAllocSlot {
    double* ptr;
    unsigned long long ctx_id;
};
static std::mutex g_noalloc_mutex;
static NoAllocSlot g_noalloc_slot[128] = {};

// Unique id of the calling thread's current context (0 when it cannot be read).
static unsigned long long current_context_id() {
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnCtxGetId>(f);
        cudaGetLastError();  // a missing entry point is not an error of the step
        resolved = true;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&ctx) == 0 && ctx != nullptr && get_id(ctx, &id) == 0) return id;
    return 0;
}

static int noalloc_scratch(double** out) {
    int dev = 0;
    int rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice", __LINE__);
    if (rc) return rc;
    if (dev < 0 || dev >= 128) return invalid("device ordinal out of range for the static scratch table");
    // make the device's primary context current (cudaSetDevice initialises it) before reading its id
    if ((rc = check_cuda(cudaSetDevice(dev), "cudaSetDevice", __LINE__))) return rc;
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocSlot& slot = g_noalloc_slot[dev];
    // without a readable context id (ctx == 0) the address is looked up on every call
    if (!slot.ptr || ctx == 0 || slot.ctx_id != ctx) {
        void* p = nullptr;
        rc = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(static scratch)", __LINE__);
        if (rc) return rc;
        slot.ptr = static_cast<double*>(p);
        slot.ctx_id = ctx;
    }
    *out = slot.ptr;
    return SKY_OK;
}

}  // namespace sky

using namespace sky;

extern "C" int sky_arrested_newton_step_noalloc(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f,
                                                int32_t n_pf, double* velocity, double* field,
                                                double* energy_gradient, double prev_energy, double* new_energy_host,
                                                double* err_host, void* stream) {
    Params p;
    int rc = pack_params(theory, p_i, n_pi, p_f, n_pf, &p);
    if (rc) return rc;
    if (!velocity || !field || !energy_gradient) return invalid("null buffer");
    if (!new_energy_host || !err_host) return invalid("null host output");
    const int64_t cn = (int64_t)p.C * n_sites(p);
    const int64_t need = 9 * cn + 2 * kScratchDoubles;
    if (need > kNoAllocDoubles) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "lattice too large for the allocation-free step: C*N = %lld needs %lld doubles of working memory, "
                 "the static scratch holds %lld (C*N <= %lld)",
                 (long long)cn, (long long)need, (long long)kNoAllocDoubles,
                 (long long)((kNoAllocDoubles - 2 * kScratchDoubles) / 9));
        return invalid(msg);
    }
    double* base = nullptr;
    if ((rc = noalloc_scratch(&base))) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    double* ks[4] = {base, base + cn, base + 2 * cn, base + 3 * cn};
    double* ls[4] = {base + 4 * cn, base + 5 * cn, base + 6 * cn, base + 7 * cn};
    double* temp = base + 8 * cn;
    double* s_e = base + 9 * cn;
    double* s_m = s_e + kScratchDoubles;
    // core/integrator.py:382-398; every slope and the stage field are written before they are read
    const double fac[4] = {0.0, 0.5, 0.5, 1.0};
    for (int s = 0; s < 4; ++s) {
        const double* lin = s == 0 ? velocity : ls[s - 1];
        const double* kprev = s == 0 ? field : ks[s - 1];
        if ((rc = rk4_stage(p, ks[s], velocity, lin, temp, field, kprev, fac[s], st))) return rc;
        if ((rc = gradient_fp64(theory, p, temp, energy_gradient, ls[s], st))) return rc;
    }
    if ((rc = rk4_finalize(theory, p, velocity, field, ks[0], ks[1], ks[2], ks[3], ls[0], ls[1], ls[2], ls[3], st)))
        return rc;
    // energy (core/integrator.py:402) and err = signed max of the stage-4 gradient (:409); the
    // reduction launchers clear their completion counters before each use
    if ((rc = density_fp64(theory, p, 0, field, nullptr, s_e, nullptr, st))) return rc;
    if ((rc = reduce(1, energy_gradient, cn, s_m, nullptr, st))) return rc;
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
        if ((rc = fill(velocity, cn, 0.0, st))) return rc;
    }
    return SKY_OK;
}
