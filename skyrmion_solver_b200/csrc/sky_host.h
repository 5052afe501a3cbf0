// Host-side helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sky_common.cuh"

namespace sky {

int check_cuda(cudaError_t e, const char* what, int line);
int invalid(const char* msg);
int fail(int code, const char* msg);  // records msg as the last error and returns code
const char* last_error();
int theory_components(int theory);
int pack_core(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, Params* out, bool need_f);
int pack_params(int theory, const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, Params* out);
int num_sms();
int ew_blocks(int64_t n);
int choose_xc(int X, int tiles_yz, int resident);
int option(int key);

int gradient_fp64(int theory, const Params& p, const double* f, double* eg, double* l, cudaStream_t st);
int density_fp64(int theory, const Params& p, int mode, const double* f, double* dens, double* scratch,
                 double* out_dev, cudaStream_t st);
int rk4_stage(const Params& p, double* kout, const double* v, const double* lin, double* temp, const double* f,
              const double* kprev, double factor, cudaStream_t st);
int rk4_finalize(int theory, const Params& p, double* v, double* f, const double* k1, const double* k2,
                 const double* k3, const double* k4, const double* l1, const double* l2, const double* l3,
                 const double* l4, cudaStream_t st);
int fill(double* a, int64_t n, double v, cudaStream_t st);
int reduce(int kind, const double* v, int64_t n, double* scratch, double* out_dev, cudaStream_t st);
int read_result(double* scratch, double* out_host, cudaStream_t st);

}  // namespace sky
