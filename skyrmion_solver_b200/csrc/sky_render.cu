// Headless volume path: the reference viewer's RGBA volume and its ray-marched
// image, computed on the device into plain buffers (no graphics API).
//
//  * Volume (build_rgba_volume_kernel, th/nuclear_skyrme/render_gl.py:157-222,
//    with the density extrema of its _reduce_density_extrema, :455-500):
//    channel 0 = (e - min e) / (max e - min e + 1e-30), channels 1..3 = the unit
//    pion vector ((0, 0, 1) where |pi|^2 <= 1e-20), FP64 arithmetic stored as
//    FP32, layout (z, y, x, channel).
//  * Image (the fragment shader of visualization/gl_backend.py:519-710):
//    per pixel a ray from the inverse view rows, clipped to the box, marched
//    front to back with early exit at alpha > 0.95; samples are trilinear with
//    clamp-to-edge (GL_LINEAR / GL_CLAMP_TO_EDGE of the volume texture), colour
//    from the 1-D transfer table (color_mode 0) or from the pion vector's HSL
//    colour (otherwise); pixels whose ray misses the box keep the white clear
//    colour.  Rows are stored top first.
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include "sky_host.h"

namespace sky {

// ---------------------------------------------------------------------------
// volume
// ---------------------------------------------------------------------------
constexpr int kMMBlocks = 592;  // partial extrema per launch (4 x 148 SMs)

__global__ void k_minmax_partial(const double* __restrict__ d, int64_t n, double* __restrict__ part) {
    __shared__ double smin[256], smax[256];
    double lo = 1.0e300, hi = -1.0e300;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = d[i];
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = smin[0];
        part[2 * blockIdx.x + 1] = smax[0];
    }
}

// One block: the global extrema of nb partials into out[0], out[1].
__global__ void k_minmax_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    __shared__ double smin[256], smax[256];
    double lo = 1.0e300, hi = -1.0e300;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        lo = fmin(lo, part[2 * b]);
        hi = fmax(hi, part[2 * b + 1]);
    }
    smin[threadIdx.x] = lo;
    smax[threadIdx.x] = hi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
            smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = smin[0];
        out[1] = smax[0];
    }
}

// One block per (32 x) x (32 z) tile of one y plane.  The field and density are
// read along z, their fastest axis, and the volume is written along x, its
// fastest axis; the tile is transposed through shared memory so both sides
// stay coalesced.
__global__ void __launch_bounds__(256) k_build_volume(int X, int Y, int Z, const double* __restrict__ dens,
                                                      const double* __restrict__ field,
                                                      const double* __restrict__ mm, float4* __restrict__ vol) {
    __shared__ float4 tile[32][33];
    const int64_t N = (int64_t)X * Y * Z;
    const int z0 = blockIdx.x * 32, y = blockIdx.y, x0 = blockIdx.z * 32;
    const double vmin = mm[0], vmax = mm[1];
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int x = x0 + i, z = z0 + threadIdx.x;
        if (x < X && z < Z) {
            const int64_t s = ((int64_t)x * Y + y) * Z + z;
            const double dn = (dens[s] - vmin) / (vmax - vmin + 1.0e-30);
            const double p1 = field[N + s], p2 = field[2 * N + s], p3 = field[3 * N + s];
            const double n2 = p1 * p1 + p2 * p2 + p3 * p3;
            double nx = 0.0, ny = 0.0, nz = 1.0;
            if (!(n2 <= 1.0e-20)) {
                const double inv = 1.0 / sqrt(n2);
                nx = p1 * inv;
                ny = p2 * inv;
                nz = p3 * inv;
            }
            tile[i][threadIdx.x] = make_float4((float)dn, (float)nx, (float)ny, (float)nz);
        }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int z = z0 + j, x = x0 + threadIdx.x;
        if (z < Z && x < X) vol[((int64_t)z * Y + y) * X + x] = tile[threadIdx.x][j];
    }
}

// ---------------------------------------------------------------------------
// ray march
// ---------------------------------------------------------------------------
struct RenderParams {
    float inv0[4], inv1[4], inv2[4];
    float box[3];
    float zoom, brightness, levelset, dmin, dmax, tscale, oscale, tstep;
    int max_steps, color_mode, width, height;
};

// The viewer's 1-D transfer texture (gl_backend.py:839), nine RGBA entries.
__constant__ float c_transfer[9][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {1.0f, 0.0f, 0.0f, 1.0f}, {1.0f, 0.5f, 0.0f, 1.0f},
                                       {1.0f, 1.0f, 0.0f, 1.0f}, {0.0f, 1.0f, 0.0f, 1.0f}, {0.0f, 1.0f, 1.0f, 1.0f},
                                       {0.0f, 0.0f, 1.0f, 1.0f}, {1.0f, 0.0f, 1.0f, 1.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};

// Linear filtering with clamp-to-edge along one axis: texel indices and weight.
__device__ __forceinline__ void lin_axis(float s, int n, int& i0, int& i1, float& w) {
    const float u = s * (float)n - 0.5f;
    const float f = floorf(u);
    w = u - f;
    const int i = (int)f;
    i0 = min(max(i, 0), n - 1);
    i1 = min(max(i + 1, 0), n - 1);
}

// Texel indices and weight along one axis from the texel-space coordinate u = s n - 1/2.
__device__ __forceinline__ void lin_texel(float u, int n, int& i0, int& i1, float& w) {
    const float f = floorf(u);
    w = u - f;
    const int i = (int)f;
    i0 = min(max(i, 0), n - 1);
    i1 = min(max(i + 1, 0), n - 1);
}

// Trilinear lookup at texel-space coordinates (ux, uy, uz).
__device__ __forceinline__ float4 sample3(const float4* __restrict__ v, int X, int Y, int Z, float ux, float uy,
                                          float uz) {
    int x0, x1, y0, y1, z0, z1;
    float wx, wy, wz;
    lin_texel(ux, X, x0, x1, wx);
    lin_texel(uy, Y, y0, y1, wy);
    lin_texel(uz, Z, z0, z1, wz);
    auto at = [&](int x, int y, int z) { return v[((int64_t)z * Y + y) * X + x]; };
    float4 c[8] = {at(x0, y0, z0), at(x1, y0, z0), at(x0, y1, z0), at(x1, y1, z0),
                   at(x0, y0, z1), at(x1, y0, z1), at(x0, y1, z1), at(x1, y1, z1)};
    auto lerp4 = [](float4 a, float4 b, float t) {
        return make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t);
    };
    const float4 c00 = lerp4(c[0], c[1], wx), c10 = lerp4(c[2], c[3], wx);
    const float4 c01 = lerp4(c[4], c[5], wx), c11 = lerp4(c[6], c[7], wx);
    return lerp4(lerp4(c00, c10, wy), lerp4(c01, c11, wy), wz);
}

// The transfer table is read from a shared-memory copy: lanes index different entries,
// which the constant cache would serialise.
__device__ __forceinline__ float4 transfer(const float4* tf, float s) {
    int i0, i1;
    float w;
    lin_axis(s, 9, i0, i1, w);
    const float4 a = tf[i0], b = tf[i1];
    return make_float4(a.x + (b.x - a.x) * w, a.y + (b.y - a.y) * w, a.z + (b.z - a.z) * w, a.w + (b.w - a.w) * w);
}

// pionVectorToRGB (gl_backend.py:573-592): HSL with saturation 1, lightness from n_z
// and hue from the azimuth of (n_x, n_y).
__device__ __forceinline__ float3 pion_rgb(float nx, float ny, float nz) {
    const float PI = 3.14159265359f;
    const float l = 0.5f * (nz + 1.0f);
    const float c = 1.0f - fabsf(2.0f * l - 1.0f);
    float h = atan2f(ny, nx);
    if (h < 0.0f) h += 2.0f * PI;
    const float q = 3.0f * h / PI;
    const float md = q - 2.0f * floorf(q / 2.0f);  // GLSL mod(q, 2)
    const float x = c * (1.0f - fabsf(md - 1.0f));
    const float m = l - 0.5f * c;
    if (q >= 0.0f && q < 1.0f) return make_float3(c + m, x + m, m);
    if (q >= 1.0f && q < 2.0f) return make_float3(x + m, c + m, m);
    if (q >= 2.0f && q < 3.0f) return make_float3(m, c + m, x + m);
    if (q >= 3.0f && q < 4.0f) return make_float3(m, x + m, c + m);
    if (q >= 4.0f && q < 5.0f) return make_float3(x + m, m, c + m);
    if (q >= 5.0f && q < 6.0f) return make_float3(c + m, m, x + m);
    return make_float3(0.0f, 0.0f, 0.0f);
}

__global__ void k_render(const float4* __restrict__ vol, int X, int Y, int Z, RenderParams rp,
                         float4* __restrict__ img) {
    __shared__ float4 tf[9];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < 9) tf[tid] = make_float4(c_transfer[tid][0], c_transfer[tid][1], c_transfer[tid][2], c_transfer[tid][3]);
    __syncthreads();
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= rp.width || row >= rp.height) return;
    float4* out = img + (int64_t)row * rp.width + px;
    const float u = ((px + 0.5f) / (float)rp.width) * 2.0f - 1.0f;
    const float v = (1.0f - (row + 0.5f) / (float)rp.height) * 2.0f - 1.0f;
    // eye ray: origin = translation column of the inverse view, direction = R^-1 (u, v, -zoom)
    const float ox = rp.inv0[3], oy = rp.inv1[3], oz = rp.inv2[3];
    float dx = rp.inv0[0] * u + rp.inv0[1] * v + rp.inv0[2] * -rp.zoom;
    float dy = rp.inv1[0] * u + rp.inv1[1] * v + rp.inv1[2] * -rp.zoom;
    float dz = rp.inv2[0] * u + rp.inv2[1] * v + rp.inv2[2] * -rp.zoom;
    const float dl = sqrtf(dx * dx + dy * dy + dz * dz);
    dx /= dl;
    dy /= dl;
    dz /= dl;
    // box intersection (slab test)
    const float bx = rp.box[0], by = rp.box[1], bz = rp.box[2];
    const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
    const float tbx = ix * (-bx - ox), tby = iy * (-by - oy), tbz = iz * (-bz - oz);
    const float ttx = ix * (bx - ox), tty = iy * (by - oy), ttz = iz * (bz - oz);
    const float tnear0 = fmaxf(fmaxf(fminf(ttx, tbx), fminf(tty, tby)), fminf(ttz, tbz));
    const float tfar = fminf(fminf(fmaxf(ttx, tbx), fmaxf(tty, tby)), fmaxf(ttz, tbz));
    if (!(tfar > tnear0)) {
        *out = make_float4(1.0f, 1.0f, 1.0f, 1.0f);  // discarded: the clear colour
        return;
    }
    const float tnear = tnear0 < 0.0f ? 0.0f : tnear0;
    float sr = 0.0f, sg = 0.0f, sb = 0.0f, sa = 0.0f;
    float t = tnear;
    float p0 = ox + dx * tnear, p1 = oy + dy * tnear, p2 = oz + dz * tnear;
    const float st0 = dx * rp.tstep, st1 = dy * rp.tstep, st2 = dz * rp.tstep;
    const float inv_denom = 1.0f / fmaxf(rp.dmax - rp.dmin, 1.0e-30f);
    // texel-space coordinate per axis: ((p / b) / 2 + 1/2) n - 1/2 = p (n / 2b) + (n - 1) / 2
    const float kx = 0.5f * (float)X / bx, ky = 0.5f * (float)Y / by, kz = 0.5f * (float)Z / bz;
    const float cx = 0.5f * (float)(X - 1), cy = 0.5f * (float)(Y - 1), cz = 0.5f * (float)(Z - 1);
    for (int i = 0; i < rp.max_steps; ++i) {
        // box edges are drawn black
        const float e0 = fminf(fabsf(p0 + bx), fabsf(p0 - bx));
        const float e1 = fminf(fabsf(p1 + by), fabsf(p1 - by));
        const float e2 = fminf(fabsf(p2 + bz), fabsf(p2 - bz));
        const int near_faces = (e0 < 0.005f) + (e1 < 0.005f) + (e2 < 0.005f);
        if (near_faces >= 2) {
            *out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            return;
        }
        const float4 sv = sample3(vol, X, Y, Z, p0 * kx + cx, p1 * ky + cy, p2 * kz + cz);
        const float norm = (sv.x - rp.dmin) * inv_denom;
        float inp = (norm - rp.levelset) * rp.tscale;
        if (inp < 0.0f) inp = 0.0f;
        float cr, cg, cb, ca;
        if (rp.color_mode == 0) {
            const float4 c = transfer(tf, fminf(fmaxf(norm, 0.0f), 1.0f));
            cr = c.x, cg = c.y, cb = c.z, ca = c.w * rp.oscale;
        } else {
            const float3 rgb = pion_rgb(sv.y, sv.z, sv.w);
            cr = inp * rgb.x, cg = inp * rgb.y, cb = inp * rgb.z, ca = inp * rp.oscale;
        }
        cr *= ca;
        cg *= ca;
        cb *= ca;
        const float k = 1.0f - sa;
        sr += cr * k;
        sg += cg * k;
        sb += cb * k;
        sa += ca * k;
        if (sa > 0.95f) break;
        t += rp.tstep;
        if (t > tfar) break;
        p0 += st0;
        p1 += st1;
        p2 += st2;
    }
    auto cl = [](float a) { return fminf(fmaxf(a, 0.0f), 1.0f); };
    *out = make_float4(cl(sr * rp.brightness), cl(sg * rp.brightness), cl(sb * rp.brightness),
                       cl(sa * rp.brightness));
}

}  // namespace sky

using namespace sky;

extern "C" {

int64_t sky_volume_scratch_size(void) { return 2 * kMMBlocks + 2; }

int sky_build_rgba_volume(const int32_t* p_i, int32_t n_pi, const double* density, const double* field,
                          double* scratch, int64_t n_scratch, float* volume, double* minmax_host, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, nullptr, 0, &p, false);
    if (rc) return rc;
    if (p.C < 4) return invalid("the volume needs the four pion components");
    if (!density || !field || !volume) return invalid("null buffer");
    if (reinterpret_cast<uintptr_t>(volume) % 16) return invalid("the volume must be 16-byte aligned");
    if (p.Y > 65535 || (p.X + 31) / 32 > 65535) return invalid("lattice too large for the volume builder");
    if (!scratch || n_scratch < 2 * kMMBlocks + 2) return SKY_ERR_NOMEM;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int64_t N = n_sites(p);
    int nb = ew_blocks(N);
    if (nb > kMMBlocks) nb = kMMBlocks;
    // partial extrema at scratch[2 ..], the global pair at scratch[0], scratch[1]
    k_minmax_partial<<<nb, 256, 0, st>>>(density, N, scratch + 2);
    k_minmax_final<<<1, 256, 0, st>>>(scratch + 2, nb, scratch);
    const dim3 vgrid((p.Z + 31) / 32, p.Y, (p.X + 31) / 32);
    k_build_volume<<<vgrid, dim3(32, 8), 0, st>>>(p.X, p.Y, p.Z, density, field, scratch,
                                                  reinterpret_cast<float4*>(volume));
    rc = check_cuda(cudaGetLastError(), "launch volume", __LINE__);
    if (rc || !minmax_host) return rc;
    rc = check_cuda(cudaMemcpyAsync(minmax_host, scratch, 2 * sizeof(double), cudaMemcpyDeviceToHost, st),
                    "read extrema", __LINE__);
    if (rc) return rc;
    return check_cuda(cudaStreamSynchronize(st), "sync", __LINE__);
}

int sky_render_volume(const float* volume, int32_t xlen, int32_t ylen, int32_t zlen, const float* params,
                      int32_t n_params, int32_t max_steps, int32_t color_mode, int32_t width, int32_t height,
                      float* image, void* stream) {
    if (!volume || !params || !image) return invalid("null buffer");
    if (n_params < 23) return invalid("the shader parameters are 23 floats");
    if (reinterpret_cast<uintptr_t>(volume) % 16 || reinterpret_cast<uintptr_t>(image) % 16)
        return invalid("the volume and the image must be 16-byte aligned");
    if (xlen < 1 || ylen < 1 || zlen < 1 || width < 1 || height < 1) return invalid("empty volume or image");
    if ((height + 15) / 16 > 65535) return invalid("image too tall");
    if (max_steps < 0) return invalid("max_steps must be >= 0");
    RenderParams rp;
    for (int k = 0; k < 4; ++k) rp.inv0[k] = params[k], rp.inv1[k] = params[4 + k], rp.inv2[k] = params[8 + k];
    for (int k = 0; k < 3; ++k) rp.box[k] = params[12 + k];
    rp.zoom = params[15];
    rp.brightness = params[16];
    rp.levelset = params[17];
    rp.dmin = params[18];
    rp.dmax = params[19];
    rp.tscale = params[20];
    rp.oscale = params[21];
    rp.tstep = params[22];
    rp.max_steps = max_steps;
    rp.color_mode = color_mode;
    rp.width = width;
    rp.height = height;
    if (!(rp.box[0] > 0.0f && rp.box[1] > 0.0f && rp.box[2] > 0.0f)) return invalid("box scale must be > 0");
    if (!(rp.tstep > 0.0f)) return invalid("tstep must be > 0");
    const dim3 block(16, 16);
    const dim3 grid((width + 15) / 16, (height + 15) / 16);
    k_render<<<grid, block, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(volume), xlen, ylen, zlen, rp, reinterpret_cast<float4*>(image));
    return check_cuda(cudaGetLastError(), "launch render", __LINE__);
}

}  // extern "C"
