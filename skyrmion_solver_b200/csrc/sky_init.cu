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
#include <math.h>
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

// ---------------------------------------------------------------------------
// The reference's own initial configurations (th/*/initial_config.py):
// a product, in order, of lumps, each a Gaussian hedgehog (hedgehog_field,
// :701-758) or a rational-map Skyrmion with the fitted profile
// (create_rational_map_skyrmion_kernel :979-1078, profilefun :342-442,
// rational_map_value :445-550, calc_rational_map_skyrmion :552-588), each
// normalised, composed by quaternion products that are normalised in turn
// (product_ansatz_kernel :1081-1126).
// ---------------------------------------------------------------------------
constexpr int kLumpStride = 16;    // doubles per lump in the host list
constexpr int kLumpsPerLaunch = 24;  // 24 x 112 B of kernel parameters per launch

struct Lump {
    double c[3];      // centre (grid coordinates)
    double alpha[3];  // Euler angles (z, y, z) applied to the position
    double beta[3];   // Euler angles applied to the target direction (hedgehog: beta[2] about z)
    double B;         // baryon number (rational map: rounded, >= 1)
    double r0;        // profile length: hedgehog f = pi exp(-(r / r0)^2); map f = profile(r / r0)
    double m0;        // profile mass mixing (the map's fitted profile)
    int kind;         // 0 hedgehog, 1 rational map
};

struct LumpList {
    Lump l[kLumpsPerLaunch];
    int n;
};

// profilefun's fits pi (1 - tanh|r (a + r (b + r (c + r (d + r e))))|): row 0 for the
// massless profile, row 1 for the massive one, per baryon number 1..9.
__constant__ double c_profile[9][2][5] = {
    {{0.630647, 0.0218873, -0.0245431, 0.00300978, -0.00010542},
     {0.839091, -0.148868, 0.222428, -0.0900171, 0.0107864}},
    {{0.162388, 0.297889, -0.0878554, 0.00931881, -0.000317398},
     {0.219378, 0.485652, -0.154501, 0.0197873, -0.000774393}},
    {{-0.000352877, 0.324957, -0.0792377, 0.00740042, -0.000232486},
     {0.0354001, 0.502948, -0.13181, 0.0142808, -0.000509656}},
    {{-0.0469393, 0.294323, -0.0599714, 0.00457823, -0.000110399},
     {-0.0127361, 0.4427, -0.0941955, 0.00808476, -0.00024485}},
    {{-0.0575367, 0.187057, -0.00254209, -0.00580857, 0.000517839},
     {-0.0568381, 0.337281, -0.0167685, -0.010309, 0.00119672}},
    {{-0.0450119, 0.104984, 0.0347624, -0.0119037, 0.000864464},
     {-0.05592, 0.229393, 0.0498254, -0.0257167, 0.00248365}},
    {{-0.0383968, 0.0703267, 0.0464174, -0.0130402, 0.000887014},
     {-0.0575166, 0.196602, 0.056918, -0.0244016, 0.00219296}},
    {{-0.013271, -0.00611001, 0.0751757, -0.0170388, 0.0010835},
     {-0.0335398, 0.0655383, 0.135378, -0.0430527, 0.00381564}},
    {{0.00853506, -0.0576792, 0.0896121, -0.0181863, 0.00109042},
     {-0.0101412, -0.0285699, 0.181351, -0.0517179, 0.00441035}}};

__device__ __forceinline__ double fitted(double r, int B, int row) {
    double k[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (B >= 1 && B <= 9)
        for (int i = 0; i < 5; ++i) k[i] = c_profile[B - 1][row][i];
    const double poly = r * (k[0] + r * (k[1] + r * (k[2] + r * (k[3] + r * k[4]))));
    return M_PI * (1.0 - tanh(fabs(poly)));
}

// The map's radial profile: pi at the centre, 0 beyond r = 15; below m0 = 1 a blend of the
// massless and massive fits.
__device__ double map_profile(double r, int B, double m0) {
    if (r < 1.0e-6) return M_PI;
    if (r > 15.0) return 0.0;
    if (m0 < 1.0) return (1.0 - m0) * fitted(r, B, 0) + m0 * fitted(r, B, 1);
    return fitted(r, B, 1);
}

struct Cx {
    double re, im;
};
__device__ __forceinline__ Cx cx_mul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cx cx_add(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx cx_sub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx cx_scale(double s, Cx a) { return {s * a.re, s * a.im}; }
// Quotient with the 1e-18 guard on |b|^2 that the reference's maps divide by.
__device__ __forceinline__ Cx cx_div(Cx a, Cx b) {
    const double den = b.re * b.re + b.im * b.im + 1.0e-18;
    return {(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
}
__device__ __forceinline__ Cx cx_pow(Cx z, int n) {
    Cx r = {1.0, 0.0};
    for (int i = 0; i < n; ++i) r = cx_mul(r, z);
    return r;
}

// The symmetric rational maps R_B(z) of the reference (B = 1..8; z^B beyond), with its
// 1e-9 offsets on the denominators that vanish at z = 0.
__device__ Cx rational_map(Cx z, int B) {
    const Cx one = {1.0, 0.0}, eps = {1.0e-9, 0.0};
    const double s3 = sqrt(3.0);
    switch (B) {
        case 1:
            return z;
        case 2:
            return cx_mul(z, z);
        case 3: {  // (i sqrt3 z^2 - 1) / (z (z^2 - i sqrt3))
            const Cx z2 = cx_mul(z, z);
            const Cx num = cx_sub(cx_mul(Cx{0.0 * s3, 1.0 * s3}, z2), one);
            const Cx den = cx_add(cx_mul(z, cx_sub(z2, Cx{s3 * 0.0, s3 * 1.0})), eps);
            return cx_div(num, den);
        }
        case 4: {  // (z^4 + 2 sqrt3 i z^2 + 1) / (z^4 - 2 sqrt3 i z^2 + 1)
            const Cx z4 = cx_pow(z, 4);
            const Cx t = cx_mul(cx_mul(cx_scale(2.0 * s3, Cx{0.0, 1.0}), z), z);
            const Cx num = cx_add(cx_add(z4, t), one);
            const Cx den = cx_add(cx_sub(z4, t), one);
            return cx_div(cx_scale(1.0, num), den);
        }
        case 5: {  // z (z^4 + b z^2 + a) / (a z^4 - b z^2 + 1)
            const double a = 3.0660, b = 3.9334;
            const Cx z4 = cx_pow(z, 4), z2 = cx_mul(z, z);
            const Cx num = cx_mul(z, cx_add(cx_add(z4, Cx{b * z2.re, b * z2.im}), Cx{a, 0.0}));
            const Cx den = cx_add(cx_sub(cx_scale(a, z4), Cx{b * z2.re, b * z2.im}), one);
            return cx_div(num, den);
        }
        case 6: {  // (z^4 + i a) / (z^2 (i a z^4 + 1))
            const double a = 0.1585;
            const Cx z4 = cx_pow(z, 4);
            const Cx num = cx_add(z4, Cx{a * 0.0, a * 1.0});
            Cx den = cx_add(cx_mul(Cx{a * 0.0, a * 1.0}, z4), one);
            den = cx_add(cx_mul(cx_mul(z, z), den), eps);
            return cx_div(num, den);
        }
        case 7: {  // (z^7 - 7 z^5 - 7 z^2 - 1) / (z^7 + 7 z^5 - 7 z^2 + 1)
            const Cx z7 = cx_pow(z, 7), z5 = cx_pow(z, 5), z2 = cx_mul(z, z);
            const Cx s5 = {7.0 * z5.re, 7.0 * z5.im}, s2 = {7.0 * z2.re, 7.0 * z2.im};
            const Cx num = cx_sub(cx_sub(cx_sub(z7, s5), s2), one);
            const Cx den = cx_add(cx_sub(cx_add(z7, s5), s2), one);
            return cx_div(num, den);
        }
        case 8: {  // (z^6 - a) / (z^2 (a z^6 + 1))
            const double a = 0.1352;
            const Cx z6 = cx_pow(z, 6);
            const Cx num = cx_sub(z6, Cx{a, 0.0});
            Cx den = cx_add(cx_scale(a, z6), one);
            den = cx_add(cx_mul(cx_mul(z, z), den), eps);
            return cx_div(num, den);
        }
        default:
            return cx_pow(z, B);
    }
}

// Rotations of the reference's rational-map code: about z by a (x, y) -> (c x + s y, -s x + c y),
// about y by a (x, z) -> (c x - s z, s x + c z), and the Euler product z(a0), y(a1), z(a2).
__device__ __forceinline__ void rot_z(double (&v)[3], double a) {
    const double c = cos(a), s = sin(a);
    const double x = c * v[0] + s * v[1], y = -s * v[0] + c * v[1];
    v[0] = x, v[1] = y;
}
__device__ __forceinline__ void rot_y(double (&v)[3], double a) {
    const double c = cos(a), s = sin(a);
    const double x = c * v[0] - s * v[2], z = s * v[0] + c * v[2];
    v[0] = x, v[2] = z;
}
__device__ __forceinline__ void rot_euler(double (&v)[3], const double (&a)[3]) {
    rot_z(v, a[0]);
    rot_y(v, a[1]);
    rot_z(v, a[2]);
}

__device__ void lump_field(const Lump& L, double gx, double gy, double gz, double (&out)[4]) {
    double r3[3] = {gx - L.c[0], gy - L.c[1], gz - L.c[2]};
    if (L.kind == 0) {  // Gaussian hedgehog, isorotated about z by beta[2]
        const double r = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
        if (r < 1.0e-12) {
            out[0] = -1.0, out[1] = out[2] = out[3] = 0.0;
            return;
        }
        const double q = r / L.r0;
        const double f = M_PI * exp(-(q * q));
        const double sf = sin(f), inv = 1.0 / r;
        double n[3] = {r3[0] * inv, r3[1] * inv, r3[2] * inv};
        rot_z(n, L.beta[2]);
        out[0] = cos(f), out[1] = sf * n[0], out[2] = sf * n[1], out[3] = sf * n[2];
        return;
    }
    rot_euler(r3, L.alpha);
    const double r = sqrt(r3[0] * r3[0] + r3[1] * r3[1] + r3[2] * r3[2]);
    int B = (int)(fabs(L.B) + 0.5);
    if (B < 1) B = 1;
    double theta = 0.0, ph = 0.0;
    if (!(r < 1.0e-6)) {
        theta = acos(r3[2] / r);
        ph = atan2(r3[1], r3[0]);
    }
    const double t = tan(0.5 * theta);
    const Cx R = rational_map(Cx{cos(ph) * t, sin(ph) * t}, B);
    const double f = map_profile(r / L.r0, B, L.m0);
    const double a = R.re * R.re + R.im * R.im, den = 1.0 + a;
    double n[3] = {2.0 * R.re / den, 2.0 * R.im / den, (1.0 - a) / den};
    rot_euler(n, L.beta);
    const double sf = sin(f);
    out[0] = cos(f), out[1] = n[0] * sf, out[2] = n[1] * sf, out[3] = n[2] * sf;
}

__device__ __forceinline__ void normalise4(double (&v)[4]) {
    double s = 0.0;
    for (int a = 0; a < 4; ++a) s += v[a] * v[a];
    s = sqrt(s);
    if (s == 0.0) return;
    for (int a = 0; a < 4; ++a) v[a] /= s;
}

// One launch composes up to kLumpsPerLaunch lumps into the field.  `start`: 0 = the field
// holds the running product; 1 = start from the vacuum (1, 0, 0, 0); 2 = start from the
// first lump of the list (normalised, not composed).  The first launch also zeroes
// components 4.. of the field.
__global__ void k_init_lumps(Params p, LumpList list, int start, double* __restrict__ field) {
    const int64_t N = n_sites(p);
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N; s += (int64_t)gridDim.x * blockDim.x) {
        const int iz = (int)(s % p.Z);
        const int64_t rr = s / p.Z;
        const int iy = (int)(rr % p.Y);
        const int ix = (int)(rr / p.Y);
        const double gx = p.hx * (double)ix, gy = p.hy * (double)iy, gz = p.hz * (double)iz;
        double acc[4];
        int k0 = 0;
        if (start == 0) {
            for (int c = 0; c < 4; ++c) acc[c] = field[c * N + s];
        } else if (start == 1 || list.n == 0) {
            acc[0] = 1.0, acc[1] = acc[2] = acc[3] = 0.0;
        } else {
            lump_field(list.l[0], gx, gy, gz, acc);
            normalise4(acc);
            k0 = 1;
        }
        for (int k = k0; k < list.n; ++k) {
            double v[4];
            lump_field(list.l[k], gx, gy, gz, v);
            normalise4(v);
            double o[4];
            qmul(acc, v, o);
            normalise4(o);
            for (int c = 0; c < 4; ++c) acc[c] = o[c];
        }
        for (int c = 0; c < 4; ++c) field[c * N + s] = acc[c];
        if (start != 0)
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

int sky_init_lumps(const int32_t* p_i, int32_t n_pi, const double* p_f, int32_t n_pf, int32_t n_lumps,
                   const double* lumps, int32_t from_vacuum, double* field, void* stream) {
    Params p;
    int rc = pack_core(p_i, n_pi, p_f, n_pf, &p, true);
    if (rc) return rc;
    if (!field) return invalid("null field buffer");
    if (n_lumps < 0) return invalid("number of lumps must be >= 0");
    if (n_lumps > 0 && !lumps) return invalid("null lump list");
    if (p.C < 4) return invalid("the initial configurations need four Skyrme components");
    for (int k = 0; k < n_lumps; ++k) {
        const double* q = lumps + (int64_t)k * kLumpStride;
        if (q[0] != 0.0 && q[0] != 1.0) return invalid("lump kind must be 0 (hedgehog) or 1 (rational map)");
        if (!(q[11] > 0.0)) return invalid("lump profile length must be > 0");
        for (int i = 0; i < kLumpStride; ++i)
            if (!isfinite(q[i])) return invalid("lump entries must be finite");
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int64_t N = n_sites(p);
    int done = 0, launch = 0;
    do {
        LumpList list;
        memset(&list, 0, sizeof(list));
        list.n = n_lumps - done < kLumpsPerLaunch ? n_lumps - done : kLumpsPerLaunch;
        for (int k = 0; k < list.n; ++k) {
            const double* q = lumps + (int64_t)(done + k) * kLumpStride;
            Lump& L = list.l[k];
            L.kind = (int)q[0];
            L.B = q[1];
            for (int d = 0; d < 3; ++d) L.c[d] = q[2 + d], L.alpha[d] = q[5 + d], L.beta[d] = q[8 + d];
            L.r0 = q[11];
            L.m0 = q[12];
        }
        const int start = launch > 0 ? 0 : (from_vacuum ? 1 : 2);
        k_init_lumps<<<ew_blocks(N), 256, 0, st>>>(p, list, start, field);
        rc = check_cuda(cudaGetLastError(), "launch init lumps", __LINE__);
        if (rc) return rc;
        done += list.n;
        ++launch;
    } while (done < n_lumps);
    return 0;
}

}  // extern "C"
