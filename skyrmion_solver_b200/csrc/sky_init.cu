// Initial Skyrme fields built on the device, in the reference layout (FP64,
// field[c * N + x * Y * Z + y * Z + z]).  The construction follows the
// reference's initial configurations (th/nuclear_skyrme/initial_config.py):
//   * centred coordinates x_i = h i - (L - 1) h / 2 - centre (:664-698);
//   * profile f(r) = pi exp(-r / scale); phi = (cos f, sin f n) (:583-587);
//   * n = x / r for a B = 1 hedgehog, else the rational map R(z) of the
//     stereographic angle z = tan(theta / 2) e^{i phi} (:941-953), through
//     n = (2 Re R, 2 Im R, 1 - |R|^2) / (1 + |R|^2) (zton, :284-306), with
//     R = z^2 (B = 2) or the cubic map (z^4 + 2 sqrt3 i z^2 + 1) /
//     (z^4 - 2 sqrt3 i z^2 + 1) (B = 4) (:481-504);
//   * solitons isorotated by unit quaternions (phi -> q phi q^-1) and combined
//     by quaternion products in order (:591-627, 1082-1126), then normalised.
// One thread per site; nothing is read but the soliton list.
#include <stdio.h>
#include <string.h>

#include "sky_host.h"

namespace sky {

constexpr int kMaxSolitons = 48;  // keeps the soliton list (by value) at 3 KB of kernel parameters

struct Soliton {
    double c[3];  // centre
    double q[4];  // isorotation (unit quaternion); (1, 0, 0, 0) for none
    int B;        // 1: hedgehog, 2 or 4: rational map
};

struct SolitonList {
    Soliton s[kMaxSolitons];
    int n;
};

__device__ __forceinline__ void qmul(const double (&a)[4], const double (&b)[4], double (&o)[4]) {
    o[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    o[1] = a[0] * b[1] + b[0] * a[1] + a[2] * b[3] - a[3] * b[2];
    o[2] = a[0] * b[2] + b[0] * a[2] + a[3] * b[1] - a[1] * b[3];
    o[3] = a[0] * b[3] + b[0] * a[3] + a[1] * b[2] - a[2] * b[1];
}

// One soliton's Skyrme field at (x, y, z) relative to its centre.
__device__ void soliton_field(const Soliton& so, double x, double y, double z, double scale, double (&out)[4]) {
    const double r = sqrt(x * x + y * y + z * z);
    const double f = M_PI * exp(-r / scale);
    const double sf = sin(f);
    out[0] = cos(f);
    if (so.B == 1) {
        if (r > 0.0) {
            out[1] = sf * x / r;
            out[2] = sf * y / r;
            out[3] = sf * z / r;
        } else {
            out[1] = out[2] = out[3] = 0.0;
        }
    } else {
        double theta = 0.0, ph = 0.0;
        if (r >= 1.0e-6) {
            theta = acos(fmin(1.0, fmax(-1.0, z / r)));
            ph = atan2(y, x);
        }
        const double t = tan(0.5 * theta);
        const double zr = t * cos(ph), zi = t * sin(ph);
        double Rr, Ri;
        const double z2r = zr * zr - zi * zi, z2i = 2.0 * zr * zi;
        if (so.B == 2) {
            Rr = z2r;
            Ri = z2i;
        } else {  // B = 4
            const double z4r = z2r * z2r - z2i * z2i, z4i = 2.0 * z2r * z2i;
            const double k = 2.0 * sqrt(3.0);      // t2 = 2 sqrt3 i z^2
            const double tr = -k * z2i, ti = k * z2r;
            const double nr = z4r + tr + 1.0, ni = z4i + ti;
            const double dr = z4r - tr + 1.0, di = z4i - ti;
            const double dd = dr * dr + di * di;
            Rr = (nr * dr + ni * di) / dd;
            Ri = (ni * dr - nr * di) / dd;
        }
        const double a = Rr * Rr + Ri * Ri;
        const double den = 1.0 + a;
        out[1] = sf * (2.0 * Rr / den);
        out[2] = sf * (2.0 * Ri / den);
        out[3] = sf * ((1.0 - a) / den);
    }
    const double* q = so.q;
    if (!(q[0] == 1.0 && q[1] == 0.0 && q[2] == 0.0 && q[3] == 0.0)) {
        const double qa[4] = {q[0], q[1], q[2], q[3]};
        const double qc[4] = {q[0], -q[1], -q[2], -q[3]};
        double t1[4];
        qmul(qa, out, t1);
        qmul(t1, qc, out);
    }
}

__global__ void k_init_field(Params p, SolitonList list, double scale, int shell, double* __restrict__ field) {
    const int64_t N = n_sites(p);
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        const int iz = (int)(s % p.Z);
        const int64_t rr = s / p.Z;
        const int iy = (int)(rr % p.Y);
        const int ix = (int)(rr / p.Y);
        const double x = (ix - (p.X - 1) / 2.0) * p.hx;
        const double y = (iy - (p.Y - 1) / 2.0) * p.hy;
        const double z = (iz - (p.Z - 1) / 2.0) * p.hz;
        double acc[4] = {1.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < list.n; ++k) {
            const Soliton& so = list.s[k];
            double v[4];
            soliton_field(so, x - so.c[0], y - so.c[1], z - so.c[2], scale, v);
            if (k == 0) {
                for (int c = 0; c < 4; ++c) acc[c] = v[c];
            } else {
                double o[4];
                qmul(acc, v, o);
                for (int c = 0; c < 4; ++c) acc[c] = o[c];
            }
        }
        const double nn = sqrt(acc[0] * acc[0] + acc[1] * acc[1] + acc[2] * acc[2] + acc[3] * acc[3]);
        if (nn > 0.0)
            for (int c = 0; c < 4; ++c) acc[c] /= nn;
        const bool edge = ix < shell || iy < shell || iz < shell || ix >= p.X - shell || iy >= p.Y - shell ||
                          iz >= p.Z - shell;
        if (edge) acc[0] = 1.0, acc[1] = acc[2] = acc[3] = 0.0;
        for (int c = 0; c < 4; ++c) field[c * N + s] = acc[c];
        for (int c = 4; c < p.C; ++c) field[c * N + s] = 0.0;
    }
}

}  // namespace sky

using namespace sky;

extern "C" {

int sky_init_field(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, int32_t nsol,
                   const int32_t* baryon, const double* centers, const double* quats, double scale,
                   int32_t vacuum_shell, double* field, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, p_f, n_pf, &p, true);
    if (rc) return rc;
    if (!field) return invalid("null field buffer");
    if (nsol < 0 || nsol > kMaxSolitons) return invalid("number of solitons must be 0..48");
    if (nsol > 0 && (!baryon || !centers)) return invalid("null soliton list");
    if (!(scale > 0.0)) return invalid("profile scale must be > 0");
    if (vacuum_shell < 0) return invalid("vacuum shell width must be >= 0");
    SolitonList list;
    memset(&list, 0, sizeof(list));
    list.n = nsol;
    for (int k = 0; k < nsol; ++k) {
        if (baryon[k] != 1 && baryon[k] != 2 && baryon[k] != 4) return invalid("soliton baryon number must be 1, 2 or 4");
        list.s[k].B = baryon[k];
        for (int d = 0; d < 3; ++d) list.s[k].c[d] = centers[3 * k + d];
        if (quats) {
            for (int d = 0; d < 4; ++d) list.s[k].q[d] = quats[4 * k + d];
        } else {
            list.s[k].q[0] = 1.0;
        }
    }
    const int64_t N = n_sites(p);
    k_init_field<<<ew_blocks(N), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p, list, scale, vacuum_shell,
                                                                                   field);
    return check_cuda(cudaGetLastError(), "launch init field", __LINE__);
}

}  // extern "C"
