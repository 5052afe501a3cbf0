// Host side of the TMA plane staging: encoding the rank-4 plane-box tensor
// maps (sky_tma.cuh).  cuTensorMapEncodeTiled is a driver entry point; it is
// reached through the runtime's driver-entry-point query so that the library
// does not link libcuda directly.
#include <stdio.h>

#include <mutex>

#include "sky_host.h"
#include "sky_tma.cuh"

namespace sky {

typedef CUresult (*PfnEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PfnEncodeTiled encode_fn() {
    static std::once_flag once;
    static PfnEncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PfnEncodeTiled>(f);
        cudaGetLastError();
    });
    return fn;
}

int encode_plane_map(TmaMap* out, const void* base, int esize, int X, int Y, int Z, int C, int hz, int hy) {
    if (!out || !base) return invalid("null tensor-map argument");
    if (esize != 4 && esize != 8) return invalid("TMA plane maps hold FP32 or FP64 values");
    const uint64_t es = (uint64_t)esize;
    const uint64_t N = (uint64_t)X * Y * Z;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return invalid("TMA plane map: base not 16-byte aligned");
    if ((Z * es) % 16 != 0 || (N * es) % 16 != 0) return invalid("TMA plane map: row pitch not a multiple of 16 B");
    if ((hz * es) % 16 != 0 || hz > 256 || hy > 256 || C > 256) return invalid("TMA plane map: box out of range");
    PfnEncodeTiled fn = encode_fn();
    if (!fn) return invalid("cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[4] = {(cuuint64_t)Z, (cuuint64_t)Y, (cuuint64_t)X, (cuuint64_t)C};
    const cuuint64_t strides[3] = {(cuuint64_t)(Z * es), (cuuint64_t)((uint64_t)Y * Z * es), (cuuint64_t)(N * es)};
    const cuuint32_t box[4] = {(cuuint32_t)hz, (cuuint32_t)hy, 1u, (cuuint32_t)C};
    const cuuint32_t estride[4] = {1u, 1u, 1u, 1u};
    const CUresult r = fn(&out->m, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                          const_cast<void*>(base), dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        char msg[128];
        snprintf(msg, sizeof(msg), "cuTensorMapEncodeTiled failed (CUresult %d)", (int)r);
        return invalid(msg);
    }
    return SKY_OK;
}

}  // namespace sky
