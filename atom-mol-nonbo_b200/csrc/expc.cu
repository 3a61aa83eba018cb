// expc.cu -- expectation values over an eigenvector: the pair terms of
// MatrixElementsForExpcVals (src/matelem.f90:949-1983) and the weighted
// sums of ExpectationValuesG's main loop (src/workproc.f90:8159-8366).
//
// One thread evaluates one pair (row i >= column j) for every symmetry term
// of the list, and adds each value's weight  factor * coef * Re(c_i^* c_j O)
// and its rounding-error bound (the reference's MEkl_s / MEkl_e) into
// per-thread shared-memory accumulators as the value is produced, so no
// pair term is stored.  Blocks then sum their threads in a fixed order and
// a second kernel sums the blocks in a fixed order: the result does not
// depend on scheduling.  Correlation functions and particle densities
// (the grid parts) run as a second pair kernel whose blocks also split the
// grid, with the same two-level reduction.
//
// The n x n algebra is restated with vectors: for a pair index P = (a, b),
// u_P = e_a (a = b) or e_a - e_b, d_P = C^-1 u_P and TrCJ_P = u_P' C^-1 u_P;
// then tr[C^-1 X C^-1 J_P] = d_P' X d_P, which is what the reference's
// ME_rXr_over_rij / ME_rXr_rYr_over_rij (src/matelem.f90:753-945) sum
// element by element.  Most matrices the reference builds for these traces
// are rank one or sums of rank-one terms (J C, C J_ii C in the
// mass-velocity terms, the Wc1..Wc3 of the orbit-orbit loops, E_ii / E_jj
// and the all-ones matrix of the Drachmanised Darwin term), so their traces
// are taken as dot products.  Results agree with the reference's to
// rounding.
//
// TrCJCJ(i,j,p,q) of src/matelem.f90:1270-1300 is never assigned for
// i = j < p < q (n >= 3) but is read by the 1/(r_ij r_pq) loop; the
// reference's ifort build keeps local arrays in zero-initialised static
// storage, so those entries are zero there.  pair_pair() reproduces that.
#include <float.h>
#include <algorithm>
#include "ecg_internal.h"

namespace ecg {

namespace {

constexpr int EXPC_BLK = 64;
constexpr double PI_D = 3.14159265358979323846264338327950;

__device__ __forceinline__ cd cexp_(cd z)
{
    double s, c;
    sincos(z.y, &s, &c);
    const double e = exp(z.x);
    return mk(e * c, e * s);
}
// principal branch, as Fortran's log of a complex argument
__device__ __forceinline__ cd clog_(cd z) { return mk(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }

template <int N>
__device__ __forceinline__ void mm(const cd (&A)[N][N], const cd (&B)[N][N], cd (&C)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = cfma(A[i][k], B[k][j], s);
            C[i][j] = s;
        }
}
// tr(A B)
template <int N>
__device__ __forceinline__ cd trmm(const cd (&A)[N][N], const cd (&B)[N][N])
{
    cd s = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) s = cfma(A[i][j], B[j][i], s);
    return s;
}
template <int N>
__device__ __forceinline__ cd trace(const cd (&A)[N][N])
{
    cd s = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) s = s + A[i][i];
    return s;
}
// u' A v
template <int N>
__device__ __forceinline__ cd quad(const cd (&u)[N], const cd (&A)[N][N], const cd (&v)[N])
{
    cd s = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) {
        cd t = mk(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < N; j++) t = cfma(A[i][j], v[j], t);
        s = cfma(u[i], t, s);
    }
    return s;
}
template <int N>
__device__ __forceinline__ cd dot(const cd (&u)[N], const cd (&v)[N])
{
    cd s = mk(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) s = cfma(u[i], v[i], s);
    return s;
}

// v[k] for a runtime k, by selects (keeps v in registers)
template <int N>
__device__ __forceinline__ cd pick(const cd (&v)[N], int k)
{
    cd r = v[0];
#pragma unroll
    for (int m = 1; m < N; m++)
        if (k == m) r = v[m];
    return r;
}
template <int N>
__device__ __forceinline__ double pickd(const double (&v)[N], int k)
{
    double r = v[0];
#pragma unroll
    for (int m = 1; m < N; m++)
        if (k == m) r = v[m];
    return r;
}

// Per pair index P = (a, b) in vech order: d_P = C^-1 u_P and TrCJ_P.
template <int N>
struct PairVecs {
    static constexpr int NP = N * (N + 1) / 2;
    cd d[NP][N];
    cd tr[NP];
};

template <int N>
__device__ __forceinline__ void pair_vecs(const cd (&inv)[N][N], PairVecs<N>& pv)
{
    int P = 0;
#pragma unroll
    for (int a = 0; a < N; a++)
#pragma unroll
        for (int b = a; b < N; b++, P++) {
            if (a == b) {
#pragma unroll
                for (int m = 0; m < N; m++) pv.d[P][m] = inv[m][a];
                pv.tr[P] = inv[a][a];
            } else {
#pragma unroll
                for (int m = 0; m < N; m++) pv.d[P][m] = inv[m][a] - inv[m][b];
                // inv(i,i) + inv(j,j) - inv(j,i) - inv(j,i), src/matelem.f90:1252
                pv.tr[P] = inv[a][a] + inv[b][b] - inv[b][a] - inv[b][a];
            }
        }
}

// tCl X tCl and tr(tCl X) (the products of ME_dXd / ME_dXd_over_rij)
template <int N>
__device__ __forceinline__ cd clxcl(const cd (&X)[N][N], const cd (&tCl)[N][N], cd (&M)[N][N])
{
    cd T1[N][N];
    mm(X, tCl, T1);
    mm(tCl, T1, M);
    return trmm(tCl, X);
}

struct ExpcArgs {
    SysParams sp;
    double mass[NMAX + 1];       // Glob_Mass: m0, m1..mn
    double bvc[NMAX][NMAX + 1];  // Glob_bvc
    double energy;               // Glob_CurrEnergy
    double err_mult;             // 2 (SymmAdaptMethod 1) or 3 (2)
    int nterms;
    int nv;                      // 6 np + 9
    long long npairs;
};

// Weighted accumulation of one value (src/workproc.f90:8218-8225).
struct Acc {
    double* s;
    double* e;
    double p1, p2;                 // Re(c_i^* c_j), -Im(c_i^* c_j)
    double rci, ici, rcj, icj;
    double w, em;
    __device__ __forceinline__ void add(int a, cd O) const
    {
        const double beta = p1 * O.x + p2 * O.y;
        const double mu = fabs(rci * (rcj * O.x - icj * O.y)) + fabs(rcj * (rci * O.x + ici * O.y)) +
                          fabs(ici * (icj * O.x + rcj * O.y)) + fabs(icj * (ici * O.x - rci * O.y));
        s[a * EXPC_BLK] += w * beta;
        e[a * EXPC_BLK] += fabs(w * (mu + em * fabs(beta)));
    }
};

__device__ __forceinline__ void pair_of(long long p, int& i, int& j)
{
    long long r = (long long)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > p) r--;
    while ((r + 1) * (r + 2) / 2 <= p) r++;
    i = (int)r;
    j = (int)(p - r * (r + 1) / 2);
}

// Unpacked bra / ket of one pair: L L' and B (src/matelem.f90:1038-1072).
template <int N>
__device__ __forceinline__ void unpack(const double* __restrict__ par, double (&A)[N][N], double (&B)[N][N],
                                       double& det)
{
    constexpr int NP = N * (N + 1) / 2;
    double L[N][N];
    int idx = 0;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++, idx++) {
            L[i][j] = 0.0;
            L[j][i] = __ldg(par + idx);
            B[i][j] = __ldg(par + NP + idx);
            B[j][i] = B[i][j];
        }
    det = 1.0;
#pragma unroll
    for (int i = 0; i < N; i++) det *= L[i][i];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k <= j; k++) s = fma(L[i][k], L[j][k], s);
            A[i][j] = s;
            A[j][i] = s;
        }
}

// P' X P for an integer-valued matrix P (src/matelem.f90:1074-1125)
template <int N>
__device__ __forceinline__ void congruence(const double (&X)[N][N], const double* __restrict__ P, double (&R)[N][N])
{
    double W[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; k++) s = fma(__ldg(P + k * NMAX + i), X[k][j], s);
            W[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; k++) s = fma(W[i][k], __ldg(P + k * NMAX + j), s);
            R[i][j] = s;
            R[j][i] = s;
        }
}

// Pseudo-Cholesky C = G G' of C = tCk + tCl, its inverse and the overlap
// (src/matelem.f90:1152-1201).
template <int N>
__device__ __forceinline__ void inverse_overlap(const cd (&C)[N][N], double absdet, double two_r3n2,
                                                cd (&inv)[N][N], cd& S)
{
    cd G[N][N], rg[N];
    cd det = mk(1.0, 0.0);
#pragma unroll
    for (int i = 0; i < N; i++) {
        {
            cd s = C[i][i];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = cfms(G[i][k], G[i][k], s);
            G[i][i] = csqrt(s);
            det = det * s;
            rg[i] = crcp(G[i][i]);
        }
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            cd s = C[i][j];
#pragma unroll
            for (int k = i - 1; k >= 0; k--) s = cfms(G[i][k], G[j][k], s);
            G[j][i] = cmul(s, rg[i]);
        }
    }
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
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = j; k < N; k++) s = cfma(G[k][i], G[k][j], s);
            inv[i][j] = s;
            inv[j][i] = s;
        }
    const cd c = rdiv(absdet, det);
    S = two_r3n2 * (c * csqrt(c));
}

// The permuted bra tCk = tAk - i tBk and ket tCl = tAl + i tBl of one term.
template <int N>
__device__ __forceinline__ void term_matrices(const double (&Ak)[N][N], const double (&Bk)[N][N],
                                              const double (&Al)[N][N], const double (&Bl)[N][N],
                                              const double* __restrict__ Pb, const double* __restrict__ Pk,
                                              cd (&tCk)[N][N], cd (&tCl)[N][N])
{
    double R1[N][N], R2[N][N];
    congruence(Ak, Pb, R1);
    congruence(Bk, Pb, R2);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) tCk[i][j] = mk(R1[i][j], -R2[i][j]);
    congruence(Al, Pk, R1);
    congruence(Bl, Pk, R2);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) tCl[i][j] = mk(R1[i][j], R2[i][j]);
}

// 1/(r_P r_Q) for pair indices P = (a,b) before Q = (c,d) in vech order
// (src/matelem.f90:1302-1339), from dP = C^-1 u_P and the two TrCJ:
// TrCJCJ is the square of u_Q' C^-1 u_P, zero where the reference leaves it
// unassigned (a = b < c < d).
template <int N>
__device__ __forceinline__ cd pair_pair(const cd (&dP)[N], cd trP, cd trQ, bool same, int a, int b, int c, int d,
                                        cd S)
{
    const cd cnumb = (4.0 / PI_D) * S;
    if (same) return cdiv(2.0 * S, trP);
    cd x;
    if (c == d)
        x = pick(dP, c);
    else if (a == b && a < c)
        x = mk(0.0, 0.0);
    else
        x = pick(dP, c) - pick(dP, d);
    const cd tt = x * x;
    const cd caux = csqrt(tt);
    const cd sq = csqrt(trP * trQ);
    if (caux.x != 0.0 || caux.y != 0.0) {
        const cd caux1 = cdiv(caux, sq);
        const cd w = mk(1.0, 0.0) - caux1 * caux1;
        const cd lg = clog_(mk(-caux1.y, caux1.x) + csqrt(w));  // log(i caux1 + sqrt(1 - caux1^2))
        const cd csum = mk(lg.y, -lg.x);                          // -i log(...)
        return cdiv(cnumb * csum, caux);
    }
    return cdiv(cnumb, sq);
}

// (a, b) of vech index P, a <= b
template <int N>
__device__ __forceinline__ void vech_pair(int P, int& a, int& b)
{
    a = 0;
    while (P >= N - a) {
        P -= N - a;
        a++;
    }
    b = a + P;
}

// The pass is split into four kernels by the values they produce, each
// recomputing the short common part (matrices, inverse, overlap): 0 = T, V,
// H, S, the pair quantities and Darwin; 1 = orbit-orbit; 2 = mass-velocity
// and its Drachmanised form; 3 = Drachmanised Darwin.  Smaller kernels keep
// their code in the instruction cache and their matrices in registers.
constexpr int EXPC_SECTIONS = 4;

// values of section SEC (local index order), and local -> MEkl index
template <int N, int SEC>
__host__ __device__ constexpr int sec_nv()
{
    return SEC == 0 ? 6 * (N * (N + 1) / 2) + 5 : (SEC == 2 ? 2 : 1);
}
template <int N, int SEC>
__device__ __forceinline__ int sec_global(int l)
{
    constexpr int B = 6 * (N * (N + 1) / 2);
    if (SEC == 0) return l < B + 4 ? l : B + 6;  // ..., H, S, T, V, then Darwin
    if (SEC == 1) return B + 8;                   // OO
    if (SEC == 2) return B + 4 + l;               // MV, drach_MV
    return B + 7;                                 // drach_Darwin
}

template <int N, int SEC>
__global__ void __launch_bounds__(EXPC_BLK) k_expc(const double* __restrict__ params, int npt,
                                                   const cd* __restrict__ cvec, const double* __restrict__ diagS,
                                                   const double* __restrict__ terms, ExpcArgs ea,
                                                   double* __restrict__ partial)
{
    constexpr int NP = N * (N + 1) / 2;
    constexpr int nvs = sec_nv<N, SEC>();
    extern __shared__ double sacc[];
    const int tid = threadIdx.x;
    const int nv = ea.nv;
    for (int a = 0; a < 2 * nvs; a++) sacc[a * EXPC_BLK + tid] = 0.0;
    const SysParams& sp = ea.sp;
    const double(&mass)[NMAX + 1] = ea.mass;
    for (long long pidx = (long long)blockIdx.x * EXPC_BLK + tid; pidx < ea.npairs;
         pidx += (long long)gridDim.x * EXPC_BLK) {
        int pi, pj;
        pair_of(pidx, pi, pj);
        double Ak[N][N], Bk[N][N], Al[N][N], Bl[N][N], dk, dl;
        unpack<N>(params + (size_t)pi * npt, Ak, Bk, dk);
        unpack<N>(params + (size_t)pj * npt, Al, Bl, dl);
        const double absdet = fabs(dl * dk);
        const cd ci = cvec[pi], cj = cvec[pj];
        const double factor = (pi == pj) ? 1.0 / sqrt(diagS[pi] * diagS[pi]) : 2.0 / sqrt(diagS[pi] * diagS[pj]);
        Acc acc;
        acc.s = sacc + tid;
        acc.e = sacc + nvs * EXPC_BLK + tid;
        acc.rci = ci.x; acc.ici = ci.y; acc.rcj = cj.x; acc.icj = cj.y;
        acc.p1 = ci.x * cj.x + ci.y * cj.y;
        acc.p2 = ci.y * cj.x - ci.x * cj.y;
        acc.em = ea.err_mult;
        for (int t = 0; t < ea.nterms; t++) {
            const double* tp = terms + (size_t)t * (2 * NMAX * NMAX + 2);
            acc.w = factor * __ldg(tp + 2 * NMAX * NMAX) * __ldg(tp + 2 * NMAX * NMAX + 1);
            cd tCk[N][N], tCl[N][N], tCkl[N][N], inv[N][N], S;
            term_matrices<N>(Ak, Bk, Al, Bl, tp, tp + NMAX * NMAX, tCk, tCl);
#pragma unroll
            for (int i = 0; i < N; i++)
#pragma unroll
                for (int j = 0; j < N; j++) tCkl[i][j] = tCk[i][j] + tCl[i][j];
            inverse_overlap<N>(tCkl, absdet, sp.two_r3n2, inv, S);
            PairVecs<N> pv;
            pair_vecs<N>(inv, pv);
            cd rm[NP];  // <1/r_P>
            if constexpr (SEC != 0) {
                const cd cn = TWO_OVER_SQRTPI * S;
#pragma unroll
                for (int P = 0; P < NP; P++) rm[P] = cdiv(cn, csqrt(pv.tr[P]));
            }

            if constexpr (SEC == 0) {
            // kinetic energy, src/matelem.f90:1203-1229
            cd T;
            {
                cd W1[N][N], W2[N][N];
                mm(inv, tCk, W1);
                mm(tCl, W1, W2);
                cd tr = mk(0.0, 0.0);
#pragma unroll
                for (int i = 0; i < N; i++)
#pragma unroll
                    for (int k = 0; k < N; k++) tr = rfma(sp.M[i * NMAX + k], W2[k][i], tr);
                T = 6.0 * (S * tr);
            }
            // 1/r, r, r^2, delta(r), V, src/matelem.f90:1231-1268
            cd V = mk(0.0, 0.0), V0 = mk(0.0, 0.0);
            {
                const cd cn = TWO_OVER_SQRTPI * S;
                const cd c15 = 1.5 * S;
                const cd cdl = (1.0 / (PI_D * SQRTPI)) * S;
                int P = 0;
#pragma unroll
                for (int a = 0; a < N; a++)
#pragma unroll
                    for (int b = a; b < N; b++, P++) {
                        const cd tr = pv.tr[P];
                        const cd sq = csqrt(tr);
                        rm[P] = cdiv(cn, sq);
                        acc.add(NP + P, rm[P]);
                        acc.add(2 * NP + P, cn * sq);
                        acc.add(3 * NP + P, c15 * tr);
                        acc.add(4 * NP + P, cdiv(cdl, sq * tr));
                        acc.add(P, cdiv(2.0 * S, tr));  // 1/r^2: the P == Q term of pair_pair
                        if (a == b)
                            V0 = rfma(sp.q[a], rm[P], V0);
                        else
                            V = rfma(sp.q[a] * sp.q[b], rm[P], V);
                    }
                V = sp.q0 * V0 + V;
            }
            acc.add(6 * NP + 0, T + V);
            acc.add(6 * NP + 1, S);
            acc.add(6 * NP + 2, T);
            acc.add(6 * NP + 3, V);

            // Darwin, src/matelem.f90:1850-1873, from delta(r_P)
            {
                const cd cdl = (1.0 / (PI_D * SQRTPI)) * S;
                cd dw = mk(0.0, 0.0);
                int P = 0;
#pragma unroll
                for (int a = 0; a < N; a++)
#pragma unroll
                    for (int b = a; b < N; b++, P++) {
                        const cd dr = cdiv(cdl, csqrt(pv.tr[P]) * pv.tr[P]);
                        if (a == b) {
                            const double f = (1.0 / (mass[0] * mass[0]) + 1.0 / (mass[a + 1] * mass[a + 1])) *
                                             sp.q0 * sp.q[a];
                            dw = rfma(f, dr, dw);
                        } else {
                            // delta(r_ab) enters twice: weights 1/m_a^2 and 1/m_b^2
                            const double f = (1.0 / (mass[a + 1] * mass[a + 1]) + 1.0 / (mass[b + 1] * mass[b + 1])) *
                                             sp.q[a] * sp.q[b];
                            dw = rfma(f, dr, dw);
                        }
                    }
                acc.add(6 * NP + 4, (-0.5 * PI_D) * dw);
            }

            // Drachmanised delta(r_P), src/matelem.f90:1349-1392
            {
                cd sumq[NP];
#pragma unroll
                for (int P = 0; P < NP; P++) sumq[P] = mk(0.0, 0.0);
                // charge weights per pair index, q0 q_a or q_a q_b
                double wq[NP];
                {
                    int P = 0;
#pragma unroll
                    for (int a = 0; a < N; a++)
#pragma unroll
                        for (int b = a; b < N; b++, P++) wq[P] = (a == b) ? sp.q0 * sp.q[a] : sp.q[a] * sp.q[b];
                }
                // one loop over the pairs (P, Q >= P); each R adds to both
                // sums, so every sum runs over Q in ascending order
#pragma unroll 1
                for (int P = 0; P < NP; P++) {
                    int a, b;
                    vech_pair<N>(P, a, b);
                    cd dP[N];
#pragma unroll
                    for (int m = 0; m < N; m++) {
                        cd r = pv.d[0][m];
#pragma unroll
                        for (int X = 1; X < NP; X++)
                            if (X == P) r = pv.d[X][m];
                        dP[m] = r;
                    }
                    const cd trP = pick(pv.tr, P);
                    const double wP = pickd(wq, P);
#pragma unroll 1
                    for (int Q = P; Q < NP; Q++) {
                        int c, d;
                        vech_pair<N>(Q, c, d);
                        const cd R = pair_pair<N>(dP, trP, pick(pv.tr, Q), Q == P, a, b, c, d, S);
                        const double wQ = pickd(wq, Q);
#pragma unroll
                        for (int X = 0; X < NP; X++) {
                            if (X == P) sumq[X] = rfma(wQ, R, sumq[X]);
                            if (X == Q && Q != P) sumq[X] = rfma(wP, R, sumq[X]);
                        }
                    }
                }
                int P = 0;
                cd W1[N][N], W2[N][N], Mc[N][N];
#pragma unroll
                for (int i = 0; i < N; i++)
#pragma unroll
                    for (int j = 0; j < N; j++) Mc[i][j] = mk(sp.M[i * NMAX + j], 0.0);
                mm(Mc, tCl, W1);
                mm(tCk, W1, W2);  // Wc2 = tCk M tCl, src/matelem.f90:1351-1366
                const cd trcx = trmm(inv, W2);
                P = 0;
#pragma unroll
                for (int a = 0; a < N; a++)
#pragma unroll
                    for (int b = a; b < N; b++, P++) {
                        const double cm = (a == b) ? 2.0 * PI_D * sp.M[a * NMAX + a]
                                                   : 2.0 * PI_D *
                                                         (sp.M[a * NMAX + a] + sp.M[b * NMAX + b] -
                                                          sp.M[a * NMAX + b] - sp.M[a * NMAX + b]);
                        const cd t = quad(pv.d[P], W2, pv.d[P]);
                        const cd rxr = rm[P] * (0.5 * (3.0 * trcx - cdiv(t, pv.tr[P])));
                        const cd num = ea.energy * rm[P] - sumq[P] - 4.0 * rxr;
                        acc.add(5 * NP + P, (1.0 / cm) * num);
                    }
            }

            }

            if constexpr (SEC == 1) {
            // orbit-orbit, src/matelem.f90:1394-1485
            // Each iteration's matrices are rank one or sums of rank-one
            // terms: Wc2 = x y', Wc3 = u z' and Wc1 = z y' + y z' + t x u'
            // + u v' with x = tCkl(:,j), y = tCl(:,j), z = tCl(:,i),
            // t = tCl(j,i), v = tCl(i,j) y + 3 tCl(j,j) z, u = e_j (first
            // loop) or e_j - e_i (second loop), so the traces of
            // ME_rXr_over_rij / ME_rXr_rYr_over_rij reduce to dot products
            // with C^-1 u, C^-1 x and C^-1 z.  The iterations run as one
            // loop; columns are picked with selects, so the matrices stay in
            // registers.
            {
                const cd cn = TWO_OVER_SQRTPI * S;
                double qv[N], mv[N];
#pragma unroll
                for (int p = 0; p < N; p++) {
                    qv[p] = sp.q[p];
                    mv[p] = mass[p + 1];
                }
                cd oo1 = mk(0.0, 0.0), oo2 = mk(0.0, 0.0);
#pragma unroll 1
                for (int it = 0; it < N * N + N * (N - 1) / 2; it++) {
                    int i, j;
                    const bool second = it >= N * N;
                    if (!second) {
                        i = it / N;
                        j = it - i * N;
                    } else {
                        int r = it - N * N;
                        i = 0;
                        while (r >= N - 1 - i) {
                            r -= N - 1 - i;
                            i++;
                        }
                        j = i + 1 + r;
                    }
                    cd x[N], y[N], z[N], iu[N];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        x[p] = pick(tCkl[p], j);
                        y[p] = pick(tCl[p], j);
                        z[p] = pick(tCl[p], i);
                        iu[p] = pick(inv[p], j);
                        if (second) iu[p] = iu[p] - pick(inv[p], i);
                    }
                    auto udot = [&](const cd (&w)[N]) -> cd {
                        cd r = pick(w, j);
                        if (second) r = r - pick(w, i);
                        return r;
                    };
                    const cd t = pick(z, j);           // tCl(j,i)
                    const cd tr3 = 3.0 * pick(y, j);   // 3 tCl(j,j)
                    cd v[N], ix[N], iz[N];
#pragma unroll
                    for (int p = 0; p < N; p++) v[p] = t * y[p] + tr3 * z[p];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        cd a = mk(0.0, 0.0), b = mk(0.0, 0.0);
#pragma unroll
                        for (int q = 0; q < N; q++) {
                            a = cfma(inv[p][q], x[q], a);
                            b = cfma(inv[p][q], z[q], b);
                        }
                        ix[p] = a;
                        iz[p] = b;
                    }
                    // d = C^-1 u_P (up to sign, which cancels) = iu; TrCJ = u' C^-1 u
                    const cd trcj = udot(iu);
                    const cd me1 = cdiv(cn, csqrt(trcj));
                    const cd yiz = dot(y, iz), xiu = dot(x, iu), viu = dot(v, iu), yiu = dot(y, iu);
                    const cd xiz = dot(x, iz), ziu = dot(z, iu), yix = dot(y, ix);
                    const cd dx = xiu, dy = yiu, dz = ziu, dv = viu, du = trcj;
                    // <r'Wc1 r / r_P>
                    const cd trw = 2.0 * yiz + t * xiu + viu;
                    const cd dwd = 2.0 * (dz * dy) + t * (dx * du) + du * dv;
                    const cd cnumb = me1 * (0.5 * (3.0 * trw - cdiv(dwd, trcj)));
                    // <(r'Wc2 r)(r'Wc3 r) / r_P>
                    const cd trcx = yix, trcy = ziu;
                    const cd trcxcy = 0.5 * (yiu * xiz + yiz * xiu);
                    const cd txj = dx * dy, tyj = du * dz;
                    const cd txyj = 0.25 * ((dy * dz) * xiu + (dy * du) * xiz + (dx * dz) * yiu + (dx * du) * yiz);
                    const cd r = 9.0 * (trcy * trcx) + 6.0 * trcxcy -
                                 cdiv(3.0 * (trcy * txj + trcx * tyj) + 4.0 * txyj, trcj) +
                                 cdiv(3.0 * (txj * tyj), trcj * trcj);
                    const cd ctemp = me1 * (0.25 * r);
                    const cd caux = -6.0 * ((t + t) * me1) + 4.0 * cnumb - 8.0 * ctemp;
                    const double qj = pickd(qv, j), mj = pickd(mv, j);
                    if (!second)
                        oo1 = oo1 - (qj / mj) * caux;
                    else
                        oo2 = oo2 + (pickd(qv, i) * qj / (pickd(mv, i) * mj)) * caux;
                }
                oo1 = (sp.q0 / mass[0]) * oo1;
                acc.add(0, 0.5 * (oo1 + oo2));
            }

            }

            if constexpr (SEC == 2) {
            // mass-velocity, src/matelem.f90:1487-1597: tCk J tCk = s_k s_k',
            // tCk J_ii tCk = tCk(:,i) tCk(i,:) (rank one), so every trace is a
            // quadratic form in C^-1.
            {
                auto mv_term = [&](const cd (&a)[N], const cd (&b)[N], cd tr1, cd tr2) -> cd {
                    const cd tr4 = quad(a, inv, a);  // tr[C^-1 a a']
                    const cd tr5 = quad(b, inv, b);
                    const cd x = quad(a, inv, b);
                    const cd caux = tr1 * tr5 + tr2 * tr4;
                    return tr4 * tr5 + (2.0 / 3.0) * (x * x) - caux + tr1 * tr2;
                };
                cd sk[N], sl[N];
                cd t1 = mk(0.0, 0.0), t2 = mk(0.0, 0.0);
#pragma unroll
                for (int p = 0; p < N; p++) {
                    cd u = mk(0.0, 0.0), v = mk(0.0, 0.0);
#pragma unroll
                    for (int q = 0; q < N; q++) {
                        u = u + tCk[q][p];
                        v = v + tCl[q][p];
                    }
                    sk[p] = u;
                    sl[p] = v;
                    t1 = t1 + u;
                    t2 = t2 + v;
                }
                cd mv = (1.0 / (mass[0] * mass[0] * mass[0])) * mv_term(sk, sl, t1, t2);
#pragma unroll
                for (int i = 0; i < N; i++) {
                    cd a[N], b[N];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        a[p] = tCk[p][i];
                        b[p] = tCl[p][i];
                    }
                    mv = mv + (1.0 / (mass[i + 1] * mass[i + 1] * mass[i + 1])) * mv_term(a, b, tCk[i][i], tCl[i][i]);
                }
                acc.add(0, (-36.0 / 8.0) * (S * mv));
            }

            // Drachmanised mass-velocity, src/matelem.f90:1675-1848
            {
                cd W1[N][N], W3[N][N];
                const double im0 = 1.0 / (mass[0] * mass[0]);
#pragma unroll
                for (int p = 0; p < N; p++)
#pragma unroll
                    for (int q = 0; q < N; q++)
                        W1[p][q] = mk(p == q ? im0 + 1.0 / (mass[p + 1] * mass[p + 1]) : im0, 0.0);
                const cd tr1 = clxcl(W1, tCl, W3);  // W3 = tCl W1 tCl
                const cd tr2 = trmm(inv, W3);
                cd dmv = (6.0 / 4.0) * (ea.energy * (S * (tr2 - tr1)));
                // second term: sum over pairs of 4 <r'W3r / r_P> - 6 tr1 <1/r_P>
                {
                    cd s = mk(0.0, 0.0);
                    int P = 0;
#pragma unroll
                    for (int a = 0; a < N; a++)
#pragma unroll
                        for (int b = a; b < N; b++, P++) {
                            const double wq = (a == b) ? sp.q0 * sp.q[a] : sp.q[a] * sp.q[b];
                            const cd t = quad(pv.d[P], W3, pv.d[P]);
                            const cd rxr = rm[P] * (0.5 * (3.0 * tr2 - cdiv(t, pv.tr[P])));
                            s = rfma(wq, 4.0 * rxr - 6.0 * (tr1 * rm[P]), s);
                        }
                    dmv = dmv - 0.25 * s;
                }
                // third term: J tCk = 1 s_k', so C^-1 tCk J tCk... = (C^-1 s_k) s_k'
                auto third = [&](const cd (&a)[N], cd t1, const double (&cw)[N]) -> cd {
                    // Wc2 = tCl diag(cw), Wc4 = C^-1 Wc2 tCl
                    cd W2[N][N], W4[N][N], Ti[N][N];
                    cd t2 = mk(0.0, 0.0);
#pragma unroll
                    for (int q = 0; q < N; q++)
#pragma unroll
                        for (int p = 0; p < N; p++) W2[q][p] = cw[p] * tCl[q][p];
#pragma unroll
                    for (int p = 0; p < N; p++) t2 = t2 + W2[p][p];
                    mm(inv, W2, Ti);
                    mm(Ti, tCl, W4);
                    const cd t4 = trace(W4);
                    cd ia[N];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        cd s = mk(0.0, 0.0);
#pragma unroll
                        for (int q = 0; q < N; q++) s = cfma(inv[p][q], a[q], s);
                        ia[p] = s;
                    }
                    const cd t3 = dot(a, ia);
                    const cd t5 = quad(a, W4, ia);
                    return 36.0 * (t3 * t4) + 24.0 * t5 - 36.0 * (t1 * t4) - 36.0 * (t2 * t3) + 36.0 * (t1 * t2);
                };
                {
                    cd sk[N];
                    cd t1 = mk(0.0, 0.0);
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        cd u = mk(0.0, 0.0);
#pragma unroll
                        for (int q = 0; q < N; q++) u = u + tCk[q][p];
                        sk[p] = u;
                        t1 = t1 + u;
                    }
                    double cw[N];
#pragma unroll
                    for (int p = 0; p < N; p++)
                        cw[p] = (mass[0] + mass[p + 1]) / (mass[0] * mass[0] * mass[p + 1] * mass[p + 1]);
                    dmv = dmv + 0.125 * (S * third(sk, t1, cw));
                }
#pragma unroll
                for (int k = 0; k < N - 1; k++) {
                    cd a[N];
                    double cw[N];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        a[p] = tCk[p][k];
                        cw[p] = p <= k ? 0.0
                                       : (mass[k + 1] + mass[p + 1]) /
                                             (mass[k + 1] * mass[k + 1] * mass[p + 1] * mass[p + 1]);
                    }
                    dmv = dmv + 0.125 * (S * third(a, tCk[k][k], cw));
                }
                acc.add(1, dmv);
            }

            }

            if constexpr (SEC == 3) {
            // Drachmanised Darwin, src/matelem.f90:1875-1929
            // ME_dXd_dYd with X = E_ii, Y = E_jj is rank one on both sides:
            // tCk E_ii tCk = a a', tCl E_jj tCl = b b' (a = tCk(:,i),
            // b = tCl(:,j)), so tr3 = a'C^-1 a, tr4 = b'C^-1 b and
            // tr5 = (a'C^-1 b)^2; with X = ones, tCk X tCk = s s' (s the
            // column sums of tCk).
            {
                cd W1[N][N], M3[N][N];
                const double im0 = 1.0 / (mass[0] * mass[0]);
#pragma unroll
                for (int p = 0; p < N; p++)
#pragma unroll
                    for (int q = 0; q < N; q++)
                        W1[p][q] = mk(p == q ? im0 + 1.0 / (mass[p + 1] * mass[p + 1]) : im0, 0.0);
                const cd trx = clxcl(W1, tCl, M3);  // M3 = tCl W1 tCl, trx = tr(tCl W1)
                const cd trm = trmm(inv, M3);
                // first and second terms: E ME_dXd(W1)/4 and the sum of ME_dXd_over_rij(W1)
                cd dd = 0.25 * (ea.energy * (6.0 * ((trm - trx) * S)));
                int P = 0;
#pragma unroll
                for (int a = 0; a < N; a++)
#pragma unroll
                    for (int b = a; b < N; b++, P++) {
                        const double wq = (a == b) ? sp.q0 * sp.q[a] : sp.q[a] * sp.q[b];
                        const cd rxr = rm[P] * (0.5 * (3.0 * trm - cdiv(quad(pv.d[P], M3, pv.d[P]), pv.tr[P])));
                        dd = dd - (0.25 * wq) * (4.0 * rxr - 6.0 * (trx * rm[P]));
                    }
                // C^-1 tCk and C^-1 tCl
                cd Vk[N][N], Vl[N][N];
                mm(inv, tCk, Vk);
                mm(inv, tCl, Vl);
                // third term: X = ones, Y = diag((m0 + m_j) / (m0^2 m_j^2))
                {
                    cd s[N], is[N];
                    cd t1 = mk(0.0, 0.0), t2 = mk(0.0, 0.0);
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        cd u = mk(0.0, 0.0), w = mk(0.0, 0.0);
#pragma unroll
                        for (int q = 0; q < N; q++) {
                            u = u + tCk[q][p];
                            w = w + Vk[p][q];  // (C^-1 tCk 1)_p = (C^-1 s)_p
                        }
                        s[p] = u;
                        is[p] = w;
                        t1 = t1 + u;
                    }
                    cd MM[N][N];  // C^-1 tCl D tCl = Vl D tCl
                    double w[N];
#pragma unroll
                    for (int p = 0; p < N; p++) {
                        w[p] = (mass[0] + mass[p + 1]) / (mass[0] * mass[0] * mass[p + 1] * mass[p + 1]);
                        t2 = rfma(w[p], tCl[p][p], t2);
                    }
#pragma unroll
                    for (int p = 0; p < N; p++)
#pragma unroll
                        for (int q = 0; q < N; q++) {
                            cd a = mk(0.0, 0.0);
#pragma unroll
                            for (int k = 0; k < N; k++) a = cfma(w[k] * Vl[p][k], tCl[k][q], a);
                            MM[p][q] = a;
                        }
                    const cd t3 = dot(s, is);
                    const cd t4 = trace(MM);
                    const cd t5 = quad(s, MM, is);
                    dd = dd + 0.125 * ((36.0 * (t3 * t4) + 24.0 * t5 - 36.0 * (t1 * t4) - 36.0 * (t2 * t3) +
                                        36.0 * (t1 * t2)) * S);
                }
                // fourth term: pairs i < j with X = E_ii, Y = E_jj
#pragma unroll
                for (int i = 0; i < N; i++) {
                    cd a[N];
#pragma unroll
                    for (int p = 0; p < N; p++) a[p] = tCk[p][i];
                    cd t3 = mk(0.0, 0.0);
#pragma unroll
                    for (int p = 0; p < N; p++) t3 = cfma(a[p], Vk[p][i], t3);  // a' C^-1 a
#pragma unroll
                    for (int j = i + 1; j < N; j++) {
                        cd t4 = mk(0.0, 0.0), x = mk(0.0, 0.0);
#pragma unroll
                        for (int p = 0; p < N; p++) {
                            t4 = cfma(tCl[p][j], Vl[p][j], t4);  // b' C^-1 b
                            x = cfma(a[p], Vl[p][j], x);         // a' C^-1 b
                        }
                        const cd t1 = tCk[i][i], t2 = tCl[j][j];
                        const cd t5 = x * x;
                        const double cw = (mass[i + 1] + mass[j + 1]) /
                                          (mass[i + 1] * mass[i + 1] * mass[j + 1] * mass[j + 1]);
                        dd = dd + (0.125 * cw) * ((36.0 * (t3 * t4) + 24.0 * t5 - 36.0 * (t1 * t4) -
                                                   36.0 * (t2 * t3) + 36.0 * (t1 * t2)) * S);
                    }
                }
                acc.add(0, dd);
            }
            }
        }
    }
    __syncthreads();
    // block sums in a fixed order; the section's slice of partial holds zero
    // for the values of the other sections
    double* out = partial + ((size_t)SEC * gridDim.x + blockIdx.x) * 2 * nv;
    for (int a = tid; a < 2 * nv; a += EXPC_BLK) out[a] = 0.0;
    __syncthreads();
    for (int l = tid; l < 2 * nvs; l += EXPC_BLK) {
        double s = 0.0;
        for (int t = 0; t < EXPC_BLK; t++) s += sacc[l * EXPC_BLK + t];
        const int li = l < nvs ? l : l - nvs;
        out[sec_global<N, SEC>(li) + (l < nvs ? 0 : nv)] = s;
    }
}

// Correlation functions (np per grid point) and particle densities (n+1
// per grid point), src/matelem.f90:1931-1960; blockIdx.y selects a chunk
// of `gchunk` grid entries (grid points times values).
template <int N>
__global__ void __launch_bounds__(EXPC_BLK) k_expc_grid(const double* __restrict__ params, int npt,
                                                        const cd* __restrict__ cvec, const double* __restrict__ diagS,
                                                        const double* __restrict__ terms, ExpcArgs ea,
                                                        const double* __restrict__ cf_grid, int ncf,
                                                        const double* __restrict__ dens_grid, int ndens, int gchunk,
                                                        double* __restrict__ partial, int ngrid)
{
    constexpr int NP = N * (N + 1) / 2;
    extern __shared__ double sacc[];
    const int tid = threadIdx.x;
    const int g0 = blockIdx.y * gchunk;
    const int g1 = min(ngrid, g0 + gchunk);
    for (int g = g0; g < g1; g++) sacc[(g - g0) * EXPC_BLK + tid] = 0.0;
    const SysParams& sp = ea.sp;
    for (long long pidx = (long long)blockIdx.x * EXPC_BLK + tid; pidx < ea.npairs;
         pidx += (long long)gridDim.x * EXPC_BLK) {
        int pi, pj;
        pair_of(pidx, pi, pj);
        double Ak[N][N], Bk[N][N], Al[N][N], Bl[N][N], dk, dl;
        unpack<N>(params + (size_t)pi * npt, Ak, Bk, dk);
        unpack<N>(params + (size_t)pj * npt, Al, Bl, dl);
        const double absdet = fabs(dl * dk);
        const cd ci = cvec[pi], cj = cvec[pj];
        const double factor = (pi == pj) ? 1.0 / sqrt(diagS[pi] * diagS[pi]) : 2.0 / sqrt(diagS[pi] * diagS[pj]);
        const double p1 = ci.x * cj.x + ci.y * cj.y, p2 = ci.y * cj.x - ci.x * cj.y;
        for (int t = 0; t < ea.nterms; t++) {
            const double* tp = terms + (size_t)t * (2 * NMAX * NMAX + 2);
            const double w = factor * __ldg(tp + 2 * NMAX * NMAX) * __ldg(tp + 2 * NMAX * NMAX + 1);
            cd tCk[N][N], tCl[N][N], inv[N][N], S;
            term_matrices<N>(Ak, Bk, Al, Bl, tp, tp + NMAX * NMAX, tCk, tCl);
#pragma unroll
            for (int i = 0; i < N; i++)
#pragma unroll
                for (int j = 0; j < N; j++) tCk[i][j] = tCk[i][j] + tCl[i][j];
            inverse_overlap<N>(tCk, absdet, sp.two_r3n2, inv, S);
            const cd pre = (1.0 / (PI_D * SQRTPI)) * S;
            // TrCJ in vech order, then the density quadratic forms
            cd x[NP + N + 1];
            {
                int P = 0;
#pragma unroll
                for (int a = 0; a < N; a++)
#pragma unroll
                    for (int b = a; b < N; b++, P++)
                        x[P] = (a == b) ? inv[a][a] : inv[a][a] + inv[b][b] - inv[b][a] - inv[b][a];
            }
#pragma unroll
            for (int i = 0; i <= N; i++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int p = 0; p < N; p++) {
                    s = rfma(ea.bvc[p][i] * ea.bvc[p][i], inv[p][p], s);
#pragma unroll
                    for (int q = p + 1; q < N; q++) s = rfma(2.0 * ea.bvc[q][i] * ea.bvc[p][i], inv[q][p], s);
                }
                x[NP + i] = s;
            }
            cd xr[NP + N + 1], px[NP + N + 1];  // 1/x and pre/(sqrt(x) x)
#pragma unroll
            for (int v = 0; v < NP + N + 1; v++) {
                xr[v] = crcp(x[v]);
                px[v] = cdiv(pre, csqrt(x[v]) * x[v]);
            }
            for (int g = g0; g < g1; g++) {
                int v, k;
                double r;
                if (g < ncf * NP) {
                    k = g / NP;
                    v = g - k * NP;
                    r = cf_grid[k];
                } else {
                    const int gd = g - ncf * NP;
                    k = gd / (N + 1);
                    v = NP + (gd - k * (N + 1));
                    r = dens_grid[k];
                }
                cd O = mk(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < NP + N + 1; u++)
                    if (u == v) O = px[u] * cexp_((-r * r) * xr[u]);
                sacc[(g - g0) * EXPC_BLK + tid] += w * (p1 * O.x + p2 * O.y);
            }
        }
    }
    __syncthreads();
    for (int g = g0 + tid; g < g1; g += EXPC_BLK) {
        double s = 0.0;
        for (int t = 0; t < EXPC_BLK; t++) s += sacc[(g - g0) * EXPC_BLK + t];
        partial[(size_t)blockIdx.x * ngrid + g] = s;
    }
}

// out[a] = sum over blocks of partial[b][a]; the second half (the error
// bounds) times epsilon when `eps_from` < count.
__global__ void k_expc_sum(const double* __restrict__ partial, int nblocks, int count, int eps_from,
                           double* __restrict__ out)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= count) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; b++) s += partial[(size_t)b * count + a];
    out[a] = a >= eps_from ? s * DBL_EPSILON : s;
}

template <int N, int SEC>
int launch_sec(Ctx& c, const ExpcArgs& ea, const double* terms, const cd* cvec, double* partial, int nblocks)
{
    const size_t smem = (size_t)2 * sec_nv<N, SEC>() * EXPC_BLK * sizeof(double);
    if (cudaFuncSetAttribute(k_expc<N, SEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -2;
    k_expc<N, SEC><<<nblocks, EXPC_BLK, smem, c.stream>>>(c.params, c.npt, cvec, c.diagS, terms, ea, partial);
    c.launches += 1;
    return 0;
}

template <int N>
int launch_n(Ctx& c, const ExpcArgs& ea, const double* terms, const cd* cvec, const double* cfg, int ncf,
             const double* dg, int ndens, double* partial, int nblocks, double* out, double* gpartial, int gblocks,
             int gchunk, int ngrid, double* gout)
{
    if (launch_sec<N, 0>(c, ea, terms, cvec, partial, nblocks) || launch_sec<N, 1>(c, ea, terms, cvec, partial, nblocks) ||
        launch_sec<N, 2>(c, ea, terms, cvec, partial, nblocks) || launch_sec<N, 3>(c, ea, terms, cvec, partial, nblocks))
        return -2;
    k_expc_sum<<<(2 * ea.nv + 127) / 128, 128, 0, c.stream>>>(partial, EXPC_SECTIONS * nblocks, 2 * ea.nv, ea.nv,
                                                               out);
    c.launches += 1;
    if (ngrid > 0) {
        const size_t gsm = (size_t)gchunk * EXPC_BLK * sizeof(double);
        if (cudaFuncSetAttribute(k_expc_grid<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm) !=
            cudaSuccess)
            return -2;
        dim3 grid(gblocks, (ngrid + gchunk - 1) / gchunk);
        k_expc_grid<N><<<grid, EXPC_BLK, gsm, c.stream>>>(c.params, c.npt, cvec, c.diagS, terms, ea, cfg, ncf, dg,
                                                          ndens, gchunk, gpartial, ngrid);
        k_expc_sum<<<(ngrid + 127) / 128, 128, 0, c.stream>>>(gpartial, gblocks, ngrid, ngrid, gout);
        c.launches += 2;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace

int expectation_values(Ctx& c, int nbasis, const double* masses, int nterms, const int* pbra, const int* pket,
                       const double* coef1, const double* coef2, int err_mult, double energy, const cd* c_host,
                       int ncf, const double* cf_grid, int ndens, const double* dens_grid, double* values,
                       double* errors, double* cf, double* dens)
{
    const int n = c.n, np = c.np;
    if (nbasis < 1 || nbasis > c.ld || nterms < 1 || ncf < 0 || ndens < 0) return -1;
    ExpcArgs ea{};
    ea.sp = c.sp;
    double mtot = 0.0;
    for (int i = 0; i <= n; i++) {
        ea.mass[i] = masses[i];
        mtot += masses[i];
    }
    // Glob_bvc, src/workproc.f90:612-621
    for (int i = 0; i <= n; i++)
        for (int p = 0; p < n; p++) ea.bvc[p][i] = -masses[p + 1] / mtot;
    for (int i = 1; i <= n; i++) ea.bvc[i - 1][i] += 1.0;
    ea.energy = energy;
    ea.err_mult = err_mult;
    ea.nterms = nterms;
    ea.nv = 6 * np + 9;
    ea.npairs = (long long)nbasis * (nbasis + 1) / 2;

    // term list: Pbra, Pket (row-major NMAX x NMAX doubles), coef1, coef2
    const int tstride = 2 * NMAX * NMAX + 2;
    std::vector<double> th((size_t)nterms * tstride, 0.0);
    for (int t = 0; t < nterms; t++) {
        double* d = th.data() + (size_t)t * tstride;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                d[i * NMAX + j] = pbra[(size_t)t * n * n + i + j * n];
                d[NMAX * NMAX + i * NMAX + j] = pket[(size_t)t * n * n + i + j * n];
            }
        d[2 * NMAX * NMAX] = coef1[t];
        d[2 * NMAX * NMAX + 1] = coef2 ? coef2[t] : 1.0;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.dev);
    const long long blocks_needed = (ea.npairs + EXPC_BLK - 1) / EXPC_BLK;
    const int nblocks = (int)std::min<long long>(blocks_needed, (long long)sms * 8);
    const int ngrid = ncf * np + ndens * (n + 1);
    const int gchunk = 48;  // 48 x 64 doubles of shared memory per block
    const int gblocks = (int)std::min<long long>(blocks_needed, (long long)sms * 2);

    double *d_terms = nullptr, *d_part = nullptr, *d_out = nullptr, *d_gpart = nullptr, *d_gout = nullptr,
           *d_cfg = nullptr, *d_dg = nullptr;
    cd* d_c = nullptr;
    int rc = 0;
    auto alloc = [&](void** p, size_t bytes) {
        if (bytes == 0) return true;
        if (cudaMalloc(p, bytes) != cudaSuccess) {
            cudaGetLastError();
            rc = -3;
            return false;
        }
        return true;
    };
    const size_t nv = ea.nv;
    if (alloc((void**)&d_terms, th.size() * sizeof(double)) &&
        alloc((void**)&d_part, (size_t)EXPC_SECTIONS * nblocks * 2 * nv * sizeof(double)) &&
        alloc((void**)&d_out, 2 * nv * sizeof(double)) &&
        alloc((void**)&d_gpart, (size_t)gblocks * ngrid * sizeof(double)) &&
        alloc((void**)&d_gout, (size_t)ngrid * sizeof(double)) &&
        alloc((void**)&d_cfg, (size_t)ncf * sizeof(double)) && alloc((void**)&d_dg, (size_t)ndens * sizeof(double)) &&
        (c_host == nullptr || alloc((void**)&d_c, (size_t)nbasis * sizeof(cd)))) {
        cudaStream_t s = c.stream;
        bool ok = cudaMemcpyAsync(d_terms, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, s) ==
                  cudaSuccess;
        if (ncf) ok = ok && cudaMemcpyAsync(d_cfg, cf_grid, ncf * sizeof(double), cudaMemcpyHostToDevice, s) ==
                                cudaSuccess;
        if (ndens)
            ok = ok && cudaMemcpyAsync(d_dg, dens_grid, ndens * sizeof(double), cudaMemcpyHostToDevice, s) ==
                           cudaSuccess;
        if (c_host) ok = ok && cudaMemcpyAsync(d_c, c_host, nbasis * sizeof(cd), cudaMemcpyHostToDevice, s) ==
                                   cudaSuccess;
        c.bytes_h2d += th.size() * sizeof(double) + (ncf + ndens) * sizeof(double) +
                       (c_host ? nbasis * sizeof(cd) : 0);
        const cd* cv = c_host ? d_c : c.c;
        if (!ok) rc = -2;
        if (rc == 0) {
            switch (n) {
                case 2: rc = launch_n<2>(c, ea, d_terms, cv, d_cfg, ncf, d_dg, ndens, d_part, nblocks, d_out, d_gpart,
                                         gblocks, gchunk, ngrid, d_gout); break;
                case 3: rc = launch_n<3>(c, ea, d_terms, cv, d_cfg, ncf, d_dg, ndens, d_part, nblocks, d_out, d_gpart,
                                         gblocks, gchunk, ngrid, d_gout); break;
                case 4: rc = launch_n<4>(c, ea, d_terms, cv, d_cfg, ncf, d_dg, ndens, d_part, nblocks, d_out, d_gpart,
                                         gblocks, gchunk, ngrid, d_gout); break;
                case 5: rc = launch_n<5>(c, ea, d_terms, cv, d_cfg, ncf, d_dg, ndens, d_part, nblocks, d_out, d_gpart,
                                         gblocks, gchunk, ngrid, d_gout); break;
                default: rc = -1;
            }
        }
        if (rc == 0) {
            std::vector<double> h(2 * nv), hg(ngrid);
            ok = cudaMemcpyAsync(h.data(), d_out, 2 * nv * sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess;
            if (ngrid)
                ok = ok && cudaMemcpyAsync(hg.data(), d_gout, ngrid * sizeof(double), cudaMemcpyDeviceToHost, s) ==
                               cudaSuccess;
            ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
            c.bytes_d2h += (2 * nv + ngrid) * sizeof(double);
            if (!ok) {
                rc = -2;
            } else {
                for (size_t a = 0; a < nv; a++) {
                    if (values) values[a] = h[a];
                    if (errors) errors[a] = h[nv + a];
                }
                if (cf)
                    for (int g = 0; g < ncf * np; g++) cf[g] = hg[g];
                if (dens)
                    for (int g = 0; g < ndens * (n + 1); g++) dens[g] = hg[ncf * np + g];
            }
        }
        if (rc != 0) cudaStreamSynchronize(s);
    }
    cudaFree(d_terms);
    cudaFree(d_part);
    cudaFree(d_out);
    cudaFree(d_gpart);
    cudaFree(d_gout);
    cudaFree(d_cfg);
    cudaFree(d_dg);
    cudaFree(d_c);
    cudaGetLastError();
    return rc;
}

}  // namespace ecg
