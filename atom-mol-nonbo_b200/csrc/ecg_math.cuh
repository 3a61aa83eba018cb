// ecg_math.cuh -- register-resident FP64 complex algebra for one ECG pair term.
//
// One pair term is one call of the reference's MatrixElements
// (src/matelem.f90:12-750): bra function k, ket function l acted on by one
// Y^+Y permutation matrix P.  Everything here is n x n with n a template
// parameter (2..5), so every loop unrolls and every matrix lives in
// registers.  All arithmetic is FP64; complex square roots take the
// principal branch exactly as Fortran's intrinsic sqrt does.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace ecg {

constexpr int NMAX = 5;     // Glob_MaxAllowedNumOfPseudoParticles
constexpr int TMAX = 64;    // largest Y^+Y term count the kernels accept

struct cd {
    double x, y;
};

__host__ __device__ __forceinline__ cd mk(double x, double y) { return cd{x, y}; }
__device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cd operator-(cd a) { return cd{-a.x, -a.y}; }
__device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__device__ __forceinline__ cd operator*(cd a, double s) { return cd{s * a.x, s * a.y}; }
__device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
__device__ __forceinline__ cd cmul(cd a, cd b)
{
    return cd{fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)};
}
__device__ __forceinline__ cd operator*(cd a, cd b) { return cmul(a, b); }
// c + a*b
__device__ __forceinline__ cd cfma(cd a, cd b, cd c)
{
    return cd{fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y))};
}
// c - a*b
__device__ __forceinline__ cd cfms(cd a, cd b, cd c)
{
    return cd{fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y))};
}
// c + s*a, s real
__device__ __forceinline__ cd rfma(double s, cd a, cd c) { return cd{fma(s, a.x, c.x), fma(s, a.y, c.y)}; }
__device__ __forceinline__ double cnorm2(cd a) { return fma(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ cd crcp(cd b)
{
    const double d = 1.0 / cnorm2(b);
    return cd{b.x * d, -b.y * d};
}
__device__ __forceinline__ cd cdiv(cd a, cd b)
{
    const double d = 1.0 / cnorm2(b);
    return cd{fma(a.x, b.x, a.y * b.y) * d, fma(a.y, b.x, -a.x * b.y) * d};
}
// real / complex
__device__ __forceinline__ cd rdiv(double r, cd b)
{
    const double d = r / cnorm2(b);
    return cd{b.x * d, -b.y * d};
}
// Principal square root (branch cut on the negative real axis, as the
// Fortran intrinsic): Kahan's formulation, "Branch cuts for complex
// elementary functions" (1987): t = sqrt((|x| + |z|)/2), then the other
// component y/(2t).  One sqrt for |z| and one reciprocal square root give
// both t and 1/t.  Also returns |z| (= |sqrt z|^2).
__device__ __forceinline__ cd csqrt_r(cd z, double& absz)
{
    const double r = sqrt(fma(z.x, z.x, z.y * z.y));
    absz = r;
    if (r == 0.0) return cd{0.0, z.y};
    const double u = 0.5 * (fabs(z.x) + r);
    const double ri = rsqrt(u);
    const double t = u * ri;
    const double h = 0.5 * z.y * ri;
    if (z.x >= 0.0) return cd{t, h};
    return cd{fabs(h), copysign(t, z.y)};
}
__device__ __forceinline__ cd csqrt(cd z)
{
    double r;
    return csqrt_r(z, r);
}

// Physical constants of one system: the n x n mass matrix
// Glob_MassMatrix (src/workproc.f90:606-610), pseudo-charges q0, q_i and
// 2^(3n/2) (src/globvars.f90:69).
struct SysParams {
    double M[NMAX * NMAX];  // row-major M[i*NMAX+j]
    double q[NMAX];
    double q0;
    double two_r3n2;
    int n;
    int T;
};

constexpr double SQRTPI = 1.77245385090551602729816748334115;
constexpr double TWO_OVER_SQRTPI = 2.0 / SQRTPI;
constexpr double ONE_OVER_SQRTPI = 1.0 / SQRTPI;

template <int N>
struct Sym {
    static constexpr int NP = N * (N + 1) / 2;
};

// vech index of element (j,i), j >= i, in the column-order vech used by the
// reference (src/matelem.f90:109-122): i outer, j = i..n inner.
__host__ __device__ constexpr int vech_index(int N, int i, int j)
{
    return i * N - i * (i - 1) / 2 + (j - i);
}

// Per-term energy quantities shared by the energy, plain-gradient and
// adjoint kernels.  Inputs: Ck = A_k - iB_k (bra, conjugated), tCl =
// P'A_lP + iP'B_lP (permuted ket), absdet = |det L_k det L_l|.
// Outputs: inv = C^-1 (symmetric), S, T, V as in src/matelem.f90:182-299,
// and with CUBE the Coulomb cubes tr32[i][j] = tr[C^-1 J_ij]^(-3/2) of
// src/matelem.f90:284-296 (diagonal: (C^-1_ii)^(-3/2)).
// Divisions are folded into reciprocals: each pseudo-Cholesky pivot is
// inverted once and reused by the factor and by its inverse, and
// 1/sqrt(a) = conj(sqrt a)/|a|.
template <int N>
struct TermEnergy {
    cd inv[N][N];
    cd S, T, V;
    cd tr32[N][N];
};

template <int N, bool CUBE>
__device__ __forceinline__ void term_energy(const cd (&Ck)[N][N], const cd (&tCl)[N][N], double absdet,
                                            const SysParams& sp, TermEnergy<N>& o)
{
    cd G[N][N], rg[N];
    // pseudo-Cholesky C = G G^T of C = Ck + tCl (matelem.f90:203-217)
    cd det = mk(1.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) {
        {
            cd s = Ck[i][i] + tCl[i][i];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = cfms(G[i][k], G[i][k], s);
            G[i][i] = csqrt(s);
            det = det * s;
            rg[i] = crcp(G[i][i]);
        }
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            cd s = Ck[i][j] + tCl[i][j];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = cfms(G[i][k], G[j][k], s);
            G[j][i] = cmul(s, rg[i]);
        }
    }
    // X = G^-1 (lower) in place, then inv = X^T X (matelem.f90:221-241)
#pragma unroll
    for (int i = 0; i < N; i++) {
        G[i][i] = rg[i];
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = i; k <= j - 1; k++) s = cfms(G[j][k], G[k][i], s);
            G[j][i] = cmul(s, rg[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < N; i++) {
#pragma unroll
        for (int j = i; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = j; k < N; k++) s = cfma(G[k][i], G[k][j], s);
            o.inv[i][j] = s;
            o.inv[j][i] = s;
        }
    }
    // overlap (matelem.f90:244-245)
    const cd c = rdiv(absdet, det);
    o.S = sp.two_r3n2 * (c * csqrt(c));
    // kinetic: T = 6 S tr[M tCl C^-1 Ck] (matelem.f90:248-274)
    cd W1[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = cfma(o.inv[i][k], Ck[k][j], s);
            W1[i][j] = s;
        }
    cd tr = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int k = 0; k < N; k++) {
            cd w2 = mk(0.0, 0.0);
#pragma unroll
            for (int m = 0; m < N; m++) w2 = cfma(tCl[k][m], W1[m][i], w2);
            tr = rfma(sp.M[i * NMAX + k], w2, tr);
        }
    o.T = 6.0 * (o.S * tr);
    // Coulomb (matelem.f90:280-299): cn / sqrt(a) = cn conj(sqrt a) / |a|
    const cd cn = TWO_OVER_SQRTPI * o.S;
    cd v = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) {
        const cd a = o.inv[i][i];
        double r;
        const cd sq = csqrt_r(a, r);
        const double ir = 1.0 / r;
        const cd is = mk(sq.x * ir, -sq.y * ir);  // 1/sqrt(a)
        v = rfma(sp.q[i], cmul(cn, is), v);
        if (CUBE) o.tr32[i][i] = cmul(is, mk(a.x * ir * ir, -a.y * ir * ir));  // a^(-1/2) a^(-1)
    }
    v = sp.q0 * v;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            const cd a = o.inv[i][i] + o.inv[j][j] - o.inv[j][i] - o.inv[j][i];
            double r;
            const cd sq = csqrt_r(a, r);
            const double ir = 1.0 / r;
            const cd is = mk(sq.x * ir, -sq.y * ir);
            v = rfma(sp.q[i] * sp.q[j], cmul(cn, is), v);
            if (CUBE) {
                o.tr32[j][i] = cmul(is, mk(a.x * ir * ir, -a.y * ir * ir));
                o.tr32[i][j] = o.tr32[j][i];
            }
        }
    o.V = v;
}

// Coulomb weights for the gradient: cnumb_ij = q_i q_j tr[C^-1 J_ij]^(-3/2)
// (i != j) and q0 q_i (C^-1_ii)^(-3/2) on the diagonal, as cnumb of
// src/matelem.f90:677-681, from the cubes kept by term_energy<N, true>.
template <int N>
__device__ __forceinline__ void coulomb_weights(const TermEnergy<N>& te, const SysParams& sp, cd (&Qw)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++) Qw[i][i] = (sp.q0 * sp.q[i]) * te.tr32[i][i];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            Qw[j][i] = (sp.q[i] * sp.q[j]) * te.tr32[j][i];
            Qw[i][j] = Qw[j][i];
        }
}

}  // namespace ecg
