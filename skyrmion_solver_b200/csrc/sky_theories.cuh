// Per-site physics of each Skyrme-type theory: energy gradient, energy density
// and baryon density, given the field value phi[C] and its first derivatives
// D[i][a] = d_i phi_a and second derivatives S[k][a] at one lattice site
// (k = 0:xx 1:yy 2:zz 3:xy 4:xz 5:yz).
//
// The formulas restate the reference's per-site device functions; each
// function names the reference lines (paths relative to the skyrmion_solver
// project root).  Templated on the arithmetic type T: double for the plain
// FP64 path, float for the mixed-precision engine.
#pragma once

#include "sky_common.cuh"

namespace sky {

__host__ __device__ constexpr int sidx(int i, int j) { return i == j ? i : 2 + i + j; }

// c_mu = det[e_mu, a, u, v] for mu = 0..3: the 4-D cross product of a, u, v,
// from the six 2x2 minors of (u, v) (24 multiply-adds instead of four 3x3
// cofactor expansions).
template <typename T>
__device__ __forceinline__ void cross4(const T* a, const T* u, const T* v, T (&c)[4]) {
    const T p01 = u[0] * v[1] - u[1] * v[0], p02 = u[0] * v[2] - u[2] * v[0], p03 = u[0] * v[3] - u[3] * v[0];
    const T p12 = u[1] * v[2] - u[2] * v[1], p13 = u[1] * v[3] - u[3] * v[1], p23 = u[2] * v[3] - u[3] * v[2];
    c[0] = a[1] * p23 - a[2] * p13 + a[3] * p12;
    c[1] = -(a[0] * p23 - a[2] * p03 + a[3] * p02);
    c[2] = a[0] * p13 - a[1] * p03 + a[3] * p01;
    c[3] = -(a[0] * p12 - a[1] * p02 + a[2] * p01);
}

// -det[phi, d_x phi, d_y phi, d_z phi] = sum_mu det[e_mu, phi, d_y phi, d_z phi] d_x phi_mu
// (expansion along the d_x phi column, th/nuclear_skyrme/kernels.py:155-194);
// baryon density = this * h^3 / (2 pi^2).
template <typename T, int C>
__device__ __forceinline__ T neg_det_b(const T* phi, const T (&D)[3][C]) {
    T c[4];
    cross4<T>(phi, D[1], D[2], c);
    return c[0] * D[0][0] + c[1] * D[0][1] + c[2] * D[0][2] + c[3] * D[0][3];
}

// Projection of the first nsky components of g orthogonal to phi
// (project_orthogonal_skyrme_field, th/nuclear_skyrme/kernels.py:236-272).
template <typename T, int C>
__device__ __forceinline__ void project(T* g, const T* phi, int nsky) {
    T lm = T(0);
#pragma unroll
    for (int a = 0; a < C; ++a)
        if (a < nsky) lm += g[a] * phi[a];
#pragma unroll
    for (int a = 0; a < C; ++a)
        if (a < nsky) g[a] -= lm * phi[a];
}

// Quartic Skyrme variation summed over ordered pairs i != j
// (th/nuclear_skyrme/kernels.py:1109-1138):
//   g_a -= coef sum_{i != j} [ 2 (F_j.S_ij) F_ia + n_j S_ii,a - (S_ii.F_j + F_i.S_ij) F_ja - (F_i.F_j) S_ij,a ]
// regrouped per unordered pair {i, j} (k = ij):
//   (F_j.S_k - S_jj.F_i) F_ia + (F_i.S_k - S_ii.F_j) F_ja - 2 (F_i.F_j) S_k,a
// plus sum_i (sum_j n_j - n_i) S_ii,a.  Same sum, fewer operations; only the
// rounding order differs from the reference.
template <typename T, int C>
__device__ __forceinline__ void skyrme_quartic(T* g, const T (&D)[3][C], const T (&S)[6][C], T coef) {
    T nrm[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) nrm[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
    const T ntot = nrm[0] + nrm[1] + nrm[2];
    T acc[4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
        acc[a] = (ntot - nrm[0]) * S[0][a] + (ntot - nrm[1]) * S[1][a] + (ntot - nrm[2]) * S[2][a];
    const int pi[3] = {0, 0, 1}, pj[3] = {1, 2, 2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int i = pi[q], j = pj[q], k = sidx(i, j);
        T dot = T(0), tij = T(0), tji = T(0), sij = T(0), sji = T(0);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            dot += D[i][b] * D[j][b];
            tij += D[j][b] * S[k][b];
            tji += D[i][b] * S[k][b];
            sij += S[i][b] * D[j][b];
            sji += S[j][b] * D[i][b];
        }
        const T ci = tij - sji, cj = tji - sij, ck = T(2) * dot;
#pragma unroll
        for (int a = 0; a < 4; ++a) acc[a] += ci * D[i][a] + cj * D[j][a] - ck * S[k][a];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) g[a] -= coef * acc[a];
}

// sum_{ijk} eps_ijk d_i(aux) det[e_mu, phi, d_j phi, d_k phi] for mu = 0..3, and
// (into *negdet) -det[phi, d_x phi, d_y phi, d_z phi], which shares the (y, z)
// cross product.  Used by the omega (th/omega_skyrme/kernels.py:633-690) and
// Coulomb (th/coulomb_skyrme/kernels.py:697-749) couplings.
template <typename T, int C>
__device__ __forceinline__ void cs_coupling(T* out, const T* phi, const T (&D)[3][C], const T* daux, T* negdet) {
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) out[mu] = T(0);
    // ordered triples (i,j,k) with sign; det[e_mu,phi,Dj,Dk] is antisymmetric in (j,k),
    // so eps_ijk det(..Dj,Dk) + eps_ikj det(..Dk,Dj) = 2 eps_ijk det(..Dj,Dk).
    const int tri[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int i = tri[t][0], j = tri[t][1], k = tri[t][2];
        T c[4];
        cross4<T>(phi, D[j], D[k], c);
        const T w = T(2) * daux[i];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) out[mu] += w * c[mu];
        if (t == 0) *negdet = c[0] * D[0][0] + c[1] * D[0][1] + c[2] * D[0][2] + c[3] * D[0][3];
    }
}

// ===========================================================================
// Nuclear (pion-only) Skyrme model, C = 4.  c0 = m_pi, c1 = kappa.
// ===========================================================================
template <typename T>
struct Nuclear {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = true;
    static constexpr int C = 4;
    static constexpr int kId = SKY_THEORY_NUCLEAR;
    // th/nuclear_skyrme/kernels.py:1035-1150
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mpi2 = T(p.c0 * p.c0);
        const T k2 = T(p.c1 * p.c1);
#pragma unroll
        for (int a = 0; a < 4; ++a) g[a] = -(S[0][a] + S[1][a] + S[2][a]);
        skyrme_quartic<T, C>(g, D, S, k2);
        g[0] -= mpi2;
        project<T, C>(g, phi, p.nsky);
    }
    // th/nuclear_skyrme/kernels.py:277-347
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T n[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) n[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
        T dxy = D[0][0] * D[1][0] + D[0][1] * D[1][1] + D[0][2] * D[1][2] + D[0][3] * D[1][3];
        T dxz = D[0][0] * D[2][0] + D[0][1] * D[2][1] + D[0][2] * D[2][2] + D[0][3] * D[2][3];
        T dyz = D[1][0] * D[2][0] + D[1][1] * D[2][1] + D[1][2] * D[2][2] + D[1][3] * D[2][3];
        T e = T(0.5) * (n[0] + n[1] + n[2]);
        e += T(0.5) * T(p.c1 * p.c1) * ((n[0] * n[1] - dxy * dxy) + (n[0] * n[2] - dxz * dxz) + (n[1] * n[2] - dyz * dyz));
        e += T(p.c0 * p.c0) * (T(1) - phi[0]);
        return e * T(p.vol);
    }
    // th/nuclear_skyrme/kernels.py:385-447
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return neg_det_b<T, C>(phi, D) * T(p.vol / (2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// Omega-meson variant, C = 5 (phi0..3, omega).  c0 = m_pi/m_omega, c1 = c_omega.
// ===========================================================================
template <typename T>
struct Omega {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = false;
    static constexpr int C = 5;
    static constexpr int kId = SKY_THEORY_OMEGA;
    // th/omega_skyrme/kernels.py:587-743
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mass2 = T(p.c0 * p.c0);
        const T cw = T(p.c1);
        const T daux[3] = {D[0][4], D[1][4], D[2][4]};
        T cs[4], nd;
        cs_coupling<T, C>(cs, phi, D, daux, &nd);
        const T k = cw / T(4.0 * M_PI * M_PI);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) g[mu] = -T(0.25) * (S[0][mu] + S[1][mu] + S[2][mu]) + k * cs[mu];
        g[0] -= T(0.25) * mass2;
        project<T, C>(g, phi, p.nsky);
        const T b0 = nd / T(2.0 * M_PI * M_PI);
        g[4] = phi[4] - (S[0][4] + S[1][4] + S[2][4]) + cw * b0;
    }
    // th/omega_skyrme/kernels.py:231-302 (no -c_omega*omega*B0 term, :301)
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T n = T(0);
#pragma unroll
        for (int i = 0; i < 3; ++i) n += D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
        T e = T(0.125) * n;
        e += T(p.c0 * p.c0) * T(0.25) * (T(1) - phi[0]);
        e += T(0.5) * phi[4] * phi[4];
        e += T(0.5) * (D[0][4] * D[0][4] + D[1][4] * D[1][4] + D[2][4] * D[2][4]);
        return e * T(p.vol);
    }
    // th/omega_skyrme/kernels.py:444-500
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return T(p.vol) * (neg_det_b<T, C>(phi, D) / T(2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// Coulomb variant, C = 5 (phi0..3, A0 = V).  c0 = mass, c1 = kappa.
// ===========================================================================
template <typename T>
struct Coulomb {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = true;
    static constexpr int C = 5;
    static constexpr int kId = SKY_THEORY_COULOMB;
    // th/coulomb_skyrme/kernels.py:585-767.  The 2*g store at :684-685 is
    // overwritten at :751-752, so the pion part is the un-doubled variation.
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mass2 = T(p.c0 * p.c0);
        const T kap = T(p.c1);
#pragma unroll
        for (int a = 0; a < 4; ++a) g[a] = -(S[0][a] + S[1][a] + S[2][a]);
        skyrme_quartic<T, C>(g, D, S, T(1));
        g[0] -= mass2;
        const T daux[3] = {D[0][4], D[1][4], D[2][4]};
        T cs[4], nd;
        cs_coupling<T, C>(cs, phi, D, daux, &nd);
        const T k = kap / T(4.0 * M_PI * M_PI);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) g[mu] -= k * cs[mu];
        project<T, C>(g, phi, p.nsky);
        const T b0 = nd / T(2.0 * M_PI * M_PI);
        g[4] = -(kap * (S[0][4] + S[1][4] + S[2][4]) + kap * b0);
    }
    // th/coulomb_skyrme/kernels.py:231-306 (no A0*B0 term, :305)
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T n[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) n[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
        T dxy = D[0][0] * D[1][0] + D[0][1] * D[1][1] + D[0][2] * D[1][2] + D[0][3] * D[1][3];
        T dxz = D[0][0] * D[2][0] + D[0][1] * D[2][1] + D[0][2] * D[2][2] + D[0][3] * D[2][3];
        T dyz = D[1][0] * D[2][0] + D[1][1] * D[2][1] + D[1][2] * D[2][2] + D[1][3] * D[2][3];
        T e = n[0] + n[1] + n[2];
        e += (n[0] * n[1] - dxy * dxy) + (n[0] * n[2] - dxz * dxz) + (n[1] * n[2] - dyz * dyz);
        e += T(2) * T(p.c0 * p.c0) * (T(1) - phi[0]);
        e += T(0.5) * T(p.c1) * (D[0][4] * D[0][4] + D[1][4] * D[1][4] + D[2][4] * D[2][4]);
        return e * T(p.vol);
    }
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return T(p.vol) * (neg_det_b<T, C>(phi, D) / T(2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// Rho-meson variant, C = 13: rho_i^a at component 4 + 3 i + a
// (th/rho_skyrme/kernels.py:84-89).  c0 = m_pi, c1 = m_rho, c2 = c_alpha.
// ===========================================================================
__host__ __device__ constexpr int ridx(int i, int a) { return 4 + 3 * i + a; }

__host__ __device__ constexpr int eps3(int i, int j, int k) {
    return (i == j || j == k || i == k) ? 0 : (((i == 0 && j == 1) || (i == 1 && j == 2) || (i == 2 && j == 0)) ? 1 : -1);
}

template <typename T>
struct Rho {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = true;
    static constexpr int C = 13;
    static constexpr int kId = SKY_THEORY_RHO;

    // d_l R^a_{jk} = S[j,l, rho(k,a)] - S[k,l, rho(j,a)]  (th/rho_skyrme/kernels.py:137-150)
    __device__ static __forceinline__ T dR(const T (&S)[6][C], int a, int j, int k, int l) {
        return S[sidx(j, l)][ridx(k, a)] - S[sidx(k, l)][ridx(j, a)];
    }
    // th/rho_skyrme/kernels.py:151-171
    __device__ static __forceinline__ T dOmega(const T (&D)[3][C], const T (&S)[6][C], int a, int j, int k, int l) {
        T t = S[sidx(j, l)][0] * D[k][a + 1] + D[j][0] * S[sidx(k, l)][a + 1] - S[sidx(j, l)][a + 1] * D[k][0] -
              D[j][a + 1] * S[sidx(k, l)][0];
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int e = eps3(a, b, c);
                if (e != 0) t += T(e) * (S[sidx(j, l)][b + 1] * D[k][c + 1] + D[j][b + 1] * S[sidx(k, l)][c + 1]);
            }
        return t;
    }
    // th/rho_skyrme/kernels.py:119-136
    __device__ static __forceinline__ T Om(const T (&D)[3][C], int a, int i, int j) {
        T t = D[i][0] * D[j][a + 1] - D[i][a + 1] * D[j][0];
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int e = eps3(a, b, c);
                if (e != 0) t += T(e) * D[i][b + 1] * D[j][c + 1];
            }
        return t;
    }

    // th/rho_skyrme/kernels.py:597-683
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mpi2 = T(p.c0 * p.c0);
        const T mrho2 = T(p.c1 * p.c1);
        const T ca16 = T(16.0 * p.c2);
        T nn[3], fs[3][3];
#pragma unroll
        for (int j = 0; j < 3; ++j) nn[j] = D[j][0] * D[j][0] + D[j][1] * D[j][1] + D[j][2] * D[j][2] + D[j][3] * D[j][3];
        // fs[i][j] = sum_nu S_ij,nu F_j,nu ; ss[i][j] = sum_nu S_jj,nu F_i,nu ; ff = F_i . F_j
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                fs[i][j] = S[sidx(i, j)][0] * D[j][0] + S[sidx(i, j)][1] * D[j][1] + S[sidx(i, j)][2] * D[j][2] +
                           S[sidx(i, j)][3] * D[j][3];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            T acc = T(0);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                acc += T(2) * S[i][mu];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const T sjf = S[j][0] * D[i][0] + S[j][1] * D[i][1] + S[j][2] * D[i][2] + S[j][3] * D[i][3];
                    const T ff = D[i][0] * D[j][0] + D[i][1] * D[j][1] + D[i][2] * D[j][2] + D[i][3] * D[j][3];
                    acc += T(2) * (S[i][mu] * nn[j] + (D[i][mu] * (fs[i][j] - sjf) - S[sidx(i, j)][mu] * ff));
                }
            }
            g[mu] = -acc;
        }
        g[0] -= T(2) * mpi2;
        // rho back-reaction on the Skyrme field (th/rho_skyrme/kernels.py:648-657)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const T r = dR(S, a, i, j, i);
                    g[0] += ca16 * D[j][a + 1] * r;
                    g[a + 1] -= ca16 * D[j][0] * r;
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const int e = eps3(b, a, c);
                            if (e != 0) g[a + 1] += ca16 * T(e) * D[j][c + 1] * dR(S, b, i, j, i);
                        }
                }
        // rho field gradient (th/rho_skyrme/kernels.py:659-667)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                T val = T(8) * mrho2 * phi[ridx(i, a)];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    val += T(8) * dR(S, a, i, j, j);
                    val -= ca16 * dOmega(D, S, a, i, j, j);
                }
                g[ridx(i, a)] = val;
            }
        project<T, C>(g, phi, 4);
    }
    // th/rho_skyrme/kernels.py:293-348
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T e = T(0);
        T n[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            n[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
            e += n[i];
        }
        // 0.5 sum_{ij} (n_i n_j - d_ij^2)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const T dij = D[i][0] * D[j][0] + D[i][1] * D[j][1] + D[i][2] * D[j][2] + D[i][3] * D[j][3];
                e += T(0.5) * (n[i] * n[j] - dij * dij);
            }
        e += T(2) * T(p.c0 * p.c0) * (T(1) - phi[0]);
        const T mrho2 = T(p.c1 * p.c1);
        const T ca8 = T(8.0 * p.c2);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T r = phi[ridx(i, a)];
                e += T(4) * mrho2 * r * r;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const T Rij = D[i][ridx(j, a)] - D[j][ridx(i, a)];
                    e += T(2) * Rij * Rij;
                    e -= ca8 * Rij * Om(D, a, i, j);
                }
            }
        return e * T(p.vol);
    }
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return neg_det_b<T, C>(phi, D) * T(p.vol / (2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// Berger-deformed Skyrme model, C = 4.  c0 = m_pi, c1 = kappa, c2 = alpha.
// omega(a, b) = a0 b3 + a1 b2 - a2 b1 - a3 b0 (th/berger_skyrme/kernels.py:81-111)
// ===========================================================================
template <typename T>
__device__ __forceinline__ T oc(const T* a, const T* b) { return a[0] * b[3] + a[1] * b[2] - a[2] * b[1] - a[3] * b[0]; }

template <typename T>
struct Berger {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = true;
    static constexpr int C = 4;
    static constexpr int kId = SKY_THEORY_BERGER;
    // th/berger_skyrme/kernels.py:554-736
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mpi2 = T(p.c0 * p.c0);
        const T k2 = T(p.c1 * p.c1);
        const T beta = T(p.c2 * p.c2 - 1.0);
#pragma unroll
        for (int a = 0; a < 4; ++a) g[a] = -(S[0][a] + S[1][a] + S[2][a]);
        const T u[3] = {oc<T>(D[0], phi), oc<T>(D[1], phi), oc<T>(D[2], phi)};
        const T div_u = oc<T>(S[0], phi) + oc<T>(S[1], phi) + oc<T>(S[2], phi);
        const T om_phi[4] = {phi[3], phi[2], -phi[1], -phi[0]};
        T om_f[3][4];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            om_f[i][0] = D[i][3];
            om_f[i][1] = D[i][2];
            om_f[i][2] = -D[i][1];
            om_f[i][3] = -D[i][0];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
            g[a] -= beta * (T(2) * u[0] * om_f[0][a] + T(2) * u[1] * om_f[1][a] + T(2) * u[2] * om_f[2][a] + div_u * om_phi[a]);
        skyrme_quartic<T, C>(g, D, S, k2);
        const T dwxy_dx = oc<T>(S[0], D[1]) + oc<T>(D[0], S[3]);
        const T dwxy_dy = oc<T>(S[3], D[1]) + oc<T>(D[0], S[1]);
        const T dwxz_dx = oc<T>(S[0], D[2]) + oc<T>(D[0], S[4]);
        const T dwxz_dz = oc<T>(S[4], D[2]) + oc<T>(D[0], S[2]);
        const T dwyz_dy = oc<T>(S[1], D[2]) + oc<T>(D[1], S[5]);
        const T dwyz_dz = oc<T>(S[5], D[2]) + oc<T>(D[1], S[2]);
        const T kb = k2 * beta;
#pragma unroll
        for (int a = 0; a < 4; ++a)
            g[a] -= kb * (dwxy_dx * om_f[1][a] - dwxy_dy * om_f[0][a] + dwxz_dx * om_f[2][a] - dwxz_dz * om_f[0][a] +
                          dwyz_dy * om_f[2][a] - dwyz_dz * om_f[1][a]);
        g[0] -= mpi2;
        project<T, C>(g, phi, p.nsky);
    }
    // th/berger_skyrme/kernels.py:251-337
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T n[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) n[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
        T dxy = D[0][0] * D[1][0] + D[0][1] * D[1][1] + D[0][2] * D[1][2] + D[0][3] * D[1][3];
        T dxz = D[0][0] * D[2][0] + D[0][1] * D[2][1] + D[0][2] * D[2][2] + D[0][3] * D[2][3];
        T dyz = D[1][0] * D[2][0] + D[1][1] * D[2][1] + D[1][2] * D[2][2] + D[1][3] * D[2][3];
        const T beta = T(p.c2 * p.c2 - 1.0);
        const T k2 = T(p.c1 * p.c1);
        const T ux = oc<T>(D[0], phi), uy = oc<T>(D[1], phi), uz = oc<T>(D[2], phi);
        const T wxy = oc<T>(D[0], D[1]), wxz = oc<T>(D[0], D[2]), wyz = oc<T>(D[1], D[2]);
        T e = T(0.5) * (n[0] + n[1] + n[2]);
        e += T(0.5) * beta * (ux * ux + uy * uy + uz * uz);
        e += T(0.5) * k2 * ((n[0] * n[1] - dxy * dxy) + (n[0] * n[2] - dxz * dxz) + (n[1] * n[2] - dyz * dyz));
        e += T(0.5) * k2 * beta * (wxy * wxy + wxz * wxz + wyz * wyz);
        e += T(p.c0 * p.c0) * (T(1) - phi[0]);
        return e * T(p.vol);
    }
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return neg_det_b<T, C>(phi, D) * T(p.vol / (2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// Lightly-bound Skyrme model, C = 4.  c0 = m_pi, c1 = alpha.
// ===========================================================================
template <typename T>
struct LightlyBound {
    // whether gradient() reads the mixed second derivatives S[3..5]
    static constexpr bool kMixed = true;
    static constexpr int C = 4;
    static constexpr int kId = SKY_THEORY_LIGHTLY_BOUND;
    // th/lightly_bound_skyrme/kernels.py:567-684
    __device__ static void gradient(const T* phi, const T (&D)[3][C], const T (&S)[6][C], const Params& p, T* g) {
        const T mpi2 = T(p.c0 * p.c0);
        const T al = T(p.c1);
        const T w = T(2) * (T(1) - al);
#pragma unroll
        for (int a = 0; a < 4; ++a) g[a] = -(w * (S[0][a] + S[1][a] + S[2][a]));
        skyrme_quartic<T, C>(g, D, S, T(1));
        const T om = T(1) - phi[0];
        g[0] -= (T(1) - al) * T(2) * mpi2;
        g[0] -= T(4) * al * om * om * om;
        project<T, C>(g, phi, p.nsky);
    }
    // th/lightly_bound_skyrme/kernels.py:275-346
    __device__ static T energy(const T* phi, const T (&D)[3][C], const Params& p) {
        T n[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) n[i] = D[i][0] * D[i][0] + D[i][1] * D[i][1] + D[i][2] * D[i][2] + D[i][3] * D[i][3];
        T dxy = D[0][0] * D[1][0] + D[0][1] * D[1][1] + D[0][2] * D[1][2] + D[0][3] * D[1][3];
        T dxz = D[0][0] * D[2][0] + D[0][1] * D[2][1] + D[0][2] * D[2][2] + D[0][3] * D[2][3];
        T dyz = D[1][0] * D[2][0] + D[1][1] * D[2][1] + D[1][2] * D[2][2] + D[1][3] * D[2][3];
        const T al = T(p.c1);
        const T om = T(1) - phi[0];
        T e = (T(1) - al) * (n[0] + n[1] + n[2]);
        e += T(0.5) * ((n[0] * n[1] - dxy * dxy) + (n[0] * n[2] - dxz * dxz) + (n[1] * n[2] - dyz * dyz));
        e += (T(1) - al) * T(2) * T(p.c0 * p.c0) * om;
        e += al * om * om * om * om;
        return e * T(p.vol);
    }
    __device__ static T baryon(const T* phi, const T (&D)[3][C], const Params& p) {
        return neg_det_b<T, C>(phi, D) * T(p.vol / (2.0 * M_PI * M_PI));
    }
};

// ===========================================================================
// What the RK4 dynamics (killkinen = 0) conserves.  The kernels integrate
// phi_c'' = -g_c.  H = (1/2) h^3 sum_c s_c |phi_c'|^2 + Phi is conserved when
// g_c = s_c dPhi/dphi_c, up to the O(h^4) gap between the force stencils and
// the energy stencils.  For the pure Skyrme variants and rho, Phi is the coded
// energy and every s_c = +1.  The omega and Coulomb auxiliary fields are time
// components of vector fields: their forces are anti-gradients (s_4 = -1) of
//   omega:   Phi = E_pion - E_omega - c_omega omega B0
//   Coulomb: Phi = E_pion / 2 - (kappa / 2) |grad V|^2 + kappa V B0
// (E_pion: the coded energy without the auxiliary field's terms; the Coulomb
// pion force is half the variation of its coded energy).  Signs and factors
// were fixed by central differences of these potentials against the coded
// forces.  Densities include the cell volume h^3, like the energies.
// ===========================================================================
template <template <typename> class Th>
struct Dynamics {
    static constexpr int C = Th<double>::C;
    __device__ static double potential(const double* phi, const double (&D)[3][C], const Params& p) {
        return Th<double>::energy(phi, D, p);
    }
    __host__ __device__ static constexpr double kinetic_sign(int) { return 1.0; }
};

template <>
struct Dynamics<Omega> {
    static constexpr int C = 5;
    __device__ static double potential(const double* phi, const double (&D)[3][C], const Params& p) {
        const double ew = p.vol * (0.5 * phi[4] * phi[4] + 0.5 * (D[0][4] * D[0][4] + D[1][4] * D[1][4] +
                                                                   D[2][4] * D[2][4]));
        const double e_pion = Omega<double>::energy(phi, D, p) - ew;
        return e_pion - ew - p.c1 * phi[4] * Omega<double>::baryon(phi, D, p);
    }
    __host__ __device__ static constexpr double kinetic_sign(int c) { return c == 4 ? -1.0 : 1.0; }
};

template <>
struct Dynamics<Coulomb> {
    static constexpr int C = 5;
    __device__ static double potential(const double* phi, const double (&D)[3][C], const Params& p) {
        const double ev = p.vol * 0.5 * p.c1 * (D[0][4] * D[0][4] + D[1][4] * D[1][4] + D[2][4] * D[2][4]);
        const double e_pion = Coulomb<double>::energy(phi, D, p) - ev;
        return 0.5 * e_pion - ev + p.c1 * phi[4] * Coulomb<double>::baryon(phi, D, p);
    }
    __host__ __device__ static constexpr double kinetic_sign(int c) { return c == 4 ? -1.0 : 1.0; }
};

}  // namespace sky
