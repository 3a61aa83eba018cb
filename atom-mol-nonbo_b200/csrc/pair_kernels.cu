// pair_kernels.cu -- symmetry-projected pair elements over the lower
// triangle of the basis, fused with their normalised store.
//
//   k_prep          per-function data: Ck = A - iB (bra), P'AP + iP'BP per
//                   Y^+Y term (ket), det L           (src/matelem.f90:109-194)
//   k_pair_diag     diagonal pairs + StoreHS/StoreHSD diagonal branch
//                   (src/matform.f90:22-25, 36-39, 84-88)
//   k_pair_energy   off-diagonal pairs, sum over Y^+Y terms, StoreHS
//                   (src/matform.f90:119-230 with :26-35, :40-49)
//   k_pair_grad     off-diagonal pairs with derivatives, StoreHSD
//                   (src/matform.f90:234-360 with :89-114)
//   k_adjoint       dE/dp contracted per pair and reduced per function,
//                   replacing Glob_D and the loop of src/workproc.f90:2127-2142
//   k_contract      the loop of src/workproc.f90:2127-2142 over Glob_D
//
// Grid shape: one CTA per 32 x 32 tile of the lower triangle; lanes run
// along the row index k (the contiguous index of the column-major H and S),
// warps along the column index l.
#include <string.h>
#include "ecg_internal.h"
#include "ecg_grad.cuh"

namespace ecg {

__device__ __forceinline__ cd ldcd(const cd* p)
{
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}
__device__ __forceinline__ void stcd(cd* p, cd v) { *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y); }

template <int N>
__device__ __forceinline__ void load_sym(const cd* __restrict__ p, cd (&M)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            const cd v = ldcd(p + vech_index(N, i, j));
            M[j][i] = v;
            M[i][j] = v;
        }
}

template <int N>
__device__ __forceinline__ void load_L(const double* __restrict__ p, double (&L)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            L[i][j] = 0.0;
            L[j][i] = __ldg(p + vech_index(N, i, j));
        }
}

template <int N>
__device__ __forceinline__ void load_P(const double* __restrict__ Pd, int t, double (&P)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) P[i][j] = Pd[(t * NMAX + i) * NMAX + j];
}

// L L' exactly as src/matelem.f90:124-139 (sum over k = 1..j).
template <int N>
__device__ __forceinline__ void gram(const double (&L)[N][N], double (&A)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            double r = 0.0;
#pragma unroll
            for (int k = 0; k <= j; k++) r = fma(L[i][k], L[j][k], r);
            A[i][j] = r;
            A[j][i] = r;
        }
}

template <int N>
__device__ __forceinline__ void sym_from_vech(const double* __restrict__ p, double (&B)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            const double v = __ldg(p + vech_index(N, i, j));
            B[i][j] = v;
            B[j][i] = v;
        }
}

// P' X P for symmetric X (src/matelem.f90:144-169); products with the 0/+-1
// entries of P are exact, so the result does not depend on FMA contraction.
template <int N>
__device__ __forceinline__ void perm_sym(const double (&P)[N][N], const double (&X)[N][N], double (&Y)[N][N])
{
    double W[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            double r = 0.0;
#pragma unroll
            for (int k = 0; k < N; k++) r = fma(P[k][i], X[k][j], r);
            W[i][j] = r;
        }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            double r = 0.0;
#pragma unroll
            for (int k = 0; k < N; k++) r = fma(W[i][k], P[k][j], r);
            Y[i][j] = r;
            Y[j][i] = r;
        }
}

// bra data of one function: Ck = A - iB and det L
template <int N>
__device__ __forceinline__ void make_bra(const double* __restrict__ p, cd (&Ck)[N][N], double& det)
{
    constexpr int NP = Sym<N>::NP;
    double L[N][N], A[N][N], B[N][N];
    load_L<N>(p, L);
    gram<N>(L, A);
    sym_from_vech<N>(p + NP, B);
    det = 1.0;
#pragma unroll
    for (int i = 0; i < N; i++) det *= L[i][i];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) Ck[i][j] = mk(A[i][j], -B[i][j]);
}

// ket data of one function under one permutation: tCl = P'AP + iP'BP
template <int N>
__device__ __forceinline__ void make_ket(const double* __restrict__ p, const double (&P)[N][N], cd (&tCl)[N][N],
                                         double& det)
{
    constexpr int NP = Sym<N>::NP;
    double L[N][N], A[N][N], B[N][N], tA[N][N], tB[N][N];
    load_L<N>(p, L);
    gram<N>(L, A);
    sym_from_vech<N>(p + NP, B);
    perm_sym<N>(P, A, tA);
    perm_sym<N>(P, B, tB);
    det = 1.0;
#pragma unroll
    for (int i = 0; i < N; i++) det *= L[i][i];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) tCl[i][j] = mk(tA[i][j], tB[i][j]);
}

template <int N>
__device__ __forceinline__ void store_sym(cd* p, const cd (&M)[N][N])
{
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) stcd(p + vech_index(N, i, j), M[j][i]);
}

// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(128) k_prep(const double* __restrict__ params, const double* __restrict__ Pd,
                                              int T, int nfun, cd* __restrict__ bra, cd* __restrict__ ket,
                                              double* __restrict__ detL)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NPT = 2 * NP;
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfun) return;
    const double* p = params + (size_t)f * NPT;
    cd Ck[N][N];
    double det;
    make_bra<N>(p, Ck, det);
    store_sym<N>(bra + (size_t)f * NP, Ck);
    detL[f] = det;
    for (int t = 0; t < T; t++) {
        double P[N][N];
        load_P<N>(Pd, t, P);
        cd tCl[N][N];
        double d2;
        make_ket<N>(p, P, tCl, d2);
        store_sym<N>(ket + ((size_t)f * T + t) * NP, tCl);
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void tile_rc(long long b, int Rlo, int& R, int& C)
{
    const long long bb = b + (long long)Rlo * (Rlo + 1) / 2;
    long long r = (long long)((sqrt(8.0 * (double)bb + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > bb) r--;
    while ((r + 1) * (r + 2) / 2 <= bb) r++;
    R = (int)r;
    C = (int)(bb - r * (r + 1) / 2);
}

// Diagonal pairs k = l for k in [r0, r1).  deriv: also Glob_D(:,k-nfru,k).
template <int N, bool DERIV>
__global__ void __launch_bounds__(128) k_pair_diag(SysParams sp, const double* __restrict__ coef,
                                                   const double* __restrict__ Pd, const double* __restrict__ params,
                                                   const cd* __restrict__ bra, const cd* __restrict__ ket,
                                                   const double* __restrict__ detL, double* __restrict__ diagS,
                                                   double* __restrict__ diagH, cd* __restrict__ H, cd* __restrict__ S,
                                                   int ld, int r0, int r1, char method, double approx_e,
                                                   cd* __restrict__ D, int ldo, int nfru)
{
    constexpr int NP = Sym<N>::NP;
    const int k = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= r1) return;
    cd Ck[N][N];
    load_sym<N>(bra + (size_t)k * NP, Ck);
    const double dk = detL[k];
    const double absdet = fabs(dk * dk);
    cd Hs = mk(0.0, 0.0), Ss = mk(0.0, 0.0);
    cd Dks[4 * NP];
    double Lk[N][N];
    if (DERIV) {
        load_L<N>(params + (size_t)k * 2 * NP, Lk);
#pragma unroll
        for (int m = 0; m < 4 * NP; m++) Dks[m] = mk(0.0, 0.0);
    }
    for (int t = 0; t < sp.T; t++) {
        cd tCl[N][N];
        load_sym<N>(ket + ((size_t)k * sp.T + t) * NP, tCl);
        TermEnergy<N> te;
        term_energy<N, DERIV>(Ck, tCl, absdet, sp, te);
        const double cf = coef[t];
        Hs = rfma(cf, te.T + te.V, Hs);
        Ss = rfma(cf, te.S, Ss);
        if (DERIV) {
            double P[N][N];
            load_P<N>(Pd, t, P);
            cd Dk[4 * NP], Dl[1];
            term_grad_plain<N, true, false>(Lk, Lk, P, Ck, tCl, te, sp, Dk, Dl);
#pragma unroll
            for (int m = 0; m < 4 * NP; m++) Dks[m] = rfma(cf, Dk[m], Dks[m]);
        }
    }
    const double dS = Ss.x;
    diagS[k] = dS;
    const size_t kk = (size_t)k + (size_t)k * ld;
    if (method == 'I') {
        S[kk] = mk(1.0, 0.0);
        H[kk] = mk(Hs.x / dS - approx_e, 0.0);
    } else {
        diagH[k] = Hs.x / dS;
    }
    if (DERIV) {
        cd* d = D + ((size_t)(k - nfru) + (size_t)k * ldo) * (4 * NP);
#pragma unroll
        for (int m = 0; m < 4 * NP; m++) d[m] = mk(2.0 * Dks[m].x / dS, 0.0);
    }
}

// Off-diagonal pairs k > l, k in [r0, r1): H, S only.  One CTA per 32 x 32
// tile, NW warps (lanes along k, warps along l, 32 / NW columns each); the
// shape (NW, MINB) is chosen by timing (PAIR_SHAPES); every shape computes
// each element with the same instructions, so results do not depend on it.
template <int N, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_pair_energy(SysParams sp, const double* __restrict__ coef,
                                                     const cd* __restrict__ bra, const cd* __restrict__ ket,
                                                     const double* __restrict__ detL,
                                                     const double* __restrict__ diagS, cd* __restrict__ H,
                                                     cd* __restrict__ S, int ld, int r0, int r1, int Rlo,
                                                     char method, double approx_e, long long t0)
{
    constexpr int NP = Sym<N>::NP;
    int R, C;
    tile_rc(t0 + blockIdx.x, Rlo, R, C);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = R * TILE + lane;
    if (k < r0 || k >= r1) return;
    cd Ck[N][N];
    load_sym<N>(bra + (size_t)k * NP, Ck);
    const double dk = detL[k];
    const double dSk = diagS[k];
#pragma unroll 1
    for (int j = 0; j < TILE / NW; j++) {
        const int l = C * TILE + w + NW * j;
        if (l >= k) break;
        const double absdet = fabs(detL[l] * dk);
        cd Hs = mk(0.0, 0.0), Ss = mk(0.0, 0.0);
#pragma unroll 1
        for (int t = 0; t < sp.T; t++) {
            cd tCl[N][N];
            load_sym<N>(ket + ((size_t)l * sp.T + t) * NP, tCl);
            TermEnergy<N> te;
            term_energy<N, false>(Ck, tCl, absdet, sp, te);
            const double cf = __ldg(coef + t);
            Hs = rfma(cf, te.T + te.V, Hs);
            Ss = rfma(cf, te.S, Ss);
        }
        const double f = 1.0 / sqrt(dSk * diagS[l]);
        const size_t kl = (size_t)k + (size_t)l * ld;
        const cd s = f * Ss;
        S[kl] = s;
        if (method == 'I') {
            S[(size_t)l + (size_t)k * ld] = conj(s);
            H[kl] = f * (Hs - approx_e * Ss);
        } else {
            H[kl] = f * Hs;
        }
    }
}

// Off-diagonal pairs with derivatives, one pair per thread at a time; the
// per-term derivative sums live in shared memory ([value][thread]).
template <int N, int NT>
__global__ void __launch_bounds__(NT) k_pair_grad(SysParams sp, const double* __restrict__ coef,
                                                  const double* __restrict__ Pd,
                                                  const double* __restrict__ params, const cd* __restrict__ bra,
                                                  const cd* __restrict__ ket, const double* __restrict__ detL,
                                                  const double* __restrict__ diagS, cd* __restrict__ H,
                                                  cd* __restrict__ S, int ld, int r0, int r1, int Rlo, char method,
                                                  double approx_e, cd* __restrict__ D, int ldo, int nfru)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = 8 * NP;  // complex values: Dk (4NP) + Dl (4NP)
    extern __shared__ double acc[];
    int R, C;
    tile_rc(blockIdx.x, Rlo, R, C);
    const int tid = threadIdx.x;
    const int lane = tid & 31, w = tid >> 5;
    constexpr int NW = NT / 32;
    const int k = R * TILE + lane;
    if (k < r0 || k >= r1) return;
    cd Ck[N][N];
    load_sym<N>(bra + (size_t)k * NP, Ck);
    double Lk[N][N];
    load_L<N>(params + (size_t)k * 2 * NP, Lk);
    const double dk = detL[k];
    const double dSk = diagS[k];
    auto A = [&](int v) -> double& { return acc[v * NT + tid]; };
#pragma unroll 1
    for (int j = 0; j < TILE / NW; j++) {
        const int l = C * TILE + w + NW * j;
        if (l >= k) break;
        const bool gl = (l >= nfru);
        double Ll[N][N];
        load_L<N>(params + (size_t)l * 2 * NP, Ll);
        const double absdet = fabs(detL[l] * dk);
        for (int v = 0; v < 2 * NV; v++) A(v) = 0.0;
        cd Hs = mk(0.0, 0.0), Ss = mk(0.0, 0.0);
#pragma unroll 1
        for (int t = 0; t < sp.T; t++) {
            cd tCl[N][N];
            load_sym<N>(ket + ((size_t)l * sp.T + t) * NP, tCl);
            TermEnergy<N> te;
            term_energy<N, true>(Ck, tCl, absdet, sp, te);
            const double cf = __ldg(coef + t);
            Hs = rfma(cf, te.T + te.V, Hs);
            Ss = rfma(cf, te.S, Ss);
            double P[N][N];
            load_P<N>(Pd, t, P);
            cd Dk[4 * NP], Dl[4 * NP];
            if (gl) {
                term_grad_plain<N, true, true>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
#pragma unroll
                for (int m = 0; m < 4 * NP; m++) {
                    A(2 * (4 * NP + m)) = fma(cf, Dl[m].x, A(2 * (4 * NP + m)));
                    A(2 * (4 * NP + m) + 1) = fma(cf, Dl[m].y, A(2 * (4 * NP + m) + 1));
                }
            } else {
                term_grad_plain<N, true, false>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
            }
#pragma unroll
            for (int m = 0; m < 4 * NP; m++) {
                A(2 * m) = fma(cf, Dk[m].x, A(2 * m));
                A(2 * m + 1) = fma(cf, Dk[m].y, A(2 * m + 1));
            }
        }
        const double f = 1.0 / sqrt(dSk * diagS[l]);
        const size_t kl = (size_t)k + (size_t)l * ld;
        const cd s = f * Ss;
        S[kl] = s;
        if (method == 'I') {
            S[(size_t)l + (size_t)k * ld] = conj(s);
            H[kl] = f * (Hs - approx_e * Ss);
        } else {
            H[kl] = f * Hs;
        }
        cd* dkl = D + ((size_t)(k - nfru) + (size_t)l * ldo) * (4 * NP);
        for (int m = 0; m < 4 * NP; m++) stcd(dkl + m, mk(f * A(2 * m), f * A(2 * m + 1)));
        if (gl) {
            cd* dlk = D + ((size_t)(l - nfru) + (size_t)k * ldo) * (4 * NP);
            for (int m = 0; m < 4 * NP; m++)
                stcd(dlk + m, mk(f * A(2 * (4 * NP + m)), -f * A(2 * (4 * NP + m) + 1)));
        }
    }
}

// ---------------------------------------------------------------------------
// Adjoint gradient.  For pair (k >= l) with weight w = conj(c_k) c_l f_kl:
//   row function k   gets  w * sum_t coef_t Z_k(t)        and Re(w a)
//   column function l gets conj(w * sum_t coef_t Z_l(t))  and Re(w a)
//   (column part only for k != l and l > nfru).
// Per tile, rows are reduced over the 8 warps and columns over the 32 lanes
// (butterfly), and written to part[tile][side][slot][NV] in a fixed order.
// ---------------------------------------------------------------------------
template <int N>
struct AdjNV {
    static constexpr int value = 2 * Sym<N>::NP + 1;
};

template <int N, int MINB>
__global__ void __launch_bounds__(256, MINB) k_adjoint(SysParams sp, const double* __restrict__ coef,
                                                 const double* __restrict__ Pd, const cd* __restrict__ bra,
                                                 const cd* __restrict__ ket, const double* __restrict__ detL,
                                                 const double* __restrict__ diagS, const cd* __restrict__ cvec,
                                                 double E, int nfru, int nfa, int Rlo, double* __restrict__ part,
                                                 long long t0)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = AdjNV<N>::value;
    extern __shared__ double red[];  // [8][32][NV]
    int R, C;
    tile_rc(t0 + blockIdx.x, Rlo, R, C);
    const long long tile = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int k = R * TILE + lane;
    const bool krow = (k >= nfru && k < nfa);
    cd Ck[N][N];
    double dk = 1.0, dSk = 1.0;
    cd ck = mk(0.0, 0.0);
    if (krow) {
        load_sym<N>(bra + (size_t)k * NP, Ck);
        dk = detL[k];
        dSk = diagS[k];
        ck = ldcd(cvec + k);
    }
    cd Ak[NP];
    double dl_k = 0.0;
#pragma unroll
    for (int x = 0; x < NP; x++) Ak[x] = mk(0.0, 0.0);
#pragma unroll 1
    for (int j = 0; j < TILE / 8; j++) {
        const int l = C * TILE + w + 8 * j;
        const bool valid = krow && (l <= k);
        const bool ketw = (l >= nfru);  // warp-uniform
        cd Zk[NP], Zl[NP], a = mk(0.0, 0.0);
#pragma unroll
        for (int x = 0; x < NP; x++) {
            Zk[x] = mk(0.0, 0.0);
            Zl[x] = mk(0.0, 0.0);
        }
        cd wkl = mk(0.0, 0.0);
        if (valid) {
            const double absdet = fabs(detL[l] * dk);
#pragma unroll 1
            for (int t = 0; t < sp.T; t++) {
                cd tCl[N][N];
                load_sym<N>(ket + ((size_t)l * sp.T + t) * NP, tCl);
                TermEnergy<N> te;
                term_energy<N, true>(Ck, tCl, absdet, sp, te);
                double P[N][N];
                load_P<N>(Pd, t, P);
                const double cf = __ldg(coef + t);
                if (ketw)
                    term_adjoint<N, true>(P, Ck, tCl, te, sp, E, cf, Zk, Zl, a);
                else
                    term_adjoint<N, false>(P, Ck, tCl, te, sp, E, cf, Zk, Zl, a);
            }
            const double f = 1.0 / sqrt(dSk * diagS[l]);
            wkl = f * cmul(conj(ck), ldcd(cvec + l));
        }
        const double ra = cmul(wkl, a).x;
#pragma unroll
        for (int x = 0; x < NP; x++) Ak[x] = cfma(wkl, Zk[x], Ak[x]);
        dl_k += ra;
        if (ketw) {
            const bool kc = valid && (l != k);
            double v[NV];
#pragma unroll
            for (int x = 0; x < NP; x++) {
                const cd z = kc ? conj(cmul(wkl, Zl[x])) : mk(0.0, 0.0);
                v[2 * x] = z.x;
                v[2 * x + 1] = z.y;
            }
            v[NV - 1] = kc ? ra : 0.0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1)
#pragma unroll
                for (int x = 0; x < NV; x++) v[x] += __shfl_xor_sync(0xffffffffu, v[x], s);
            if (lane == 0) {
                double* dst = part + ((tile * 2 + 1) * TILE + (w + 8 * j)) * NV;
#pragma unroll
                for (int x = 0; x < NV; x++) dst[x] = v[x];
            }
        }
    }
    double* r = red + ((size_t)w * TILE + lane) * NV;
#pragma unroll
    for (int x = 0; x < NP; x++) {
        r[2 * x] = Ak[x].x;
        r[2 * x + 1] = Ak[x].y;
    }
    r[NV - 1] = dl_k;
    __syncthreads();
    if (w == 0) {
        double* dst = part + ((tile * 2 + 0) * TILE + lane) * NV;
        for (int x = 0; x < NV; x++) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 8; q++) s += red[((size_t)q * TILE + lane) * NV + x];
            dst[x] = s;
        }
    }
}

// dE/d(vech L, vech B) of one function from its summed adjoint values v
// (NP complex sums of w Z, then the sum of Re(w a)) and its parameters p;
// lane x < NP writes entry x of both halves of g.
template <int N>
__device__ __forceinline__ void adj_gradient(const double (&v)[AdjNV<N>::value], const double* __restrict__ p,
                                             int lane, double* __restrict__ g)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = AdjNV<N>::value;
    if (lane < NP) {
        // vech entry x = (column i, row j >= i)
        int i = 0, x = lane;
        while (x >= N - i) {
            x -= N - i;
            i++;
        }
        const int j = i + x;
        double acc = 0.0;
        for (int m = i; m < N; m++) {
            // A(j,m) from the packed lower triangle, L(m,i) = vech(i,m)
            const int a = (j >= m) ? vech_index(N, m, j) : vech_index(N, j, m);
            acc += v[2 * a] * p[vech_index(N, i, m)];
        }
        double gL = -4.0 * acc;
        if (i == j) gL += 2.0 * v[NV - 1] / p[vech_index(N, i, i)];
        const int a = vech_index(N, i, j);
        const double gB = -2.0 * ((i == j) ? 1.0 : 2.0) * v[2 * a + 1];
        g[lane] = gL;
        g[NP + lane] = gB;
    }
}

// One warp per function f in [nfru, nfa): sum its row and column partials
// in a fixed order and form dE/d(vech L_f, vech B_f).
template <int N>
__global__ void __launch_bounds__(256) k_adjoint_final(const double* __restrict__ part,
                                                       const double* __restrict__ params, int nfru, int nfa,
                                                       int Rlo, int nR, double* __restrict__ grad)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = AdjNV<N>::value;
    const int lane = threadIdx.x & 31;
    const int f = nfru + (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    if (f >= nfa) return;
    const int Rf = f / TILE, slot = f % TILE;
    const long long base = (long long)Rlo * (Rlo + 1) / 2;
    double v[NV];
#pragma unroll
    for (int x = 0; x < NV; x++) v[x] = 0.0;
    for (int Cc = lane; Cc <= Rf; Cc += 32) {
        const long long t = (long long)Rf * (Rf + 1) / 2 - base + Cc;
        const double* src = part + ((t * 2 + 0) * TILE + slot) * NV;
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += src[x];
    }
    for (int Rr = Rf + lane; Rr < nR; Rr += 32) {
        const long long t = (long long)Rr * (Rr + 1) / 2 - base + Rf;
        const double* src = part + ((t * 2 + 1) * TILE + slot) * NV;
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += src[x];
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1)
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += __shfl_xor_sync(0xffffffffu, v[x], s);
    adj_gradient<N>(v, params + (size_t)f * 2 * NP, lane, grad + (size_t)(f - nfru) * 2 * NP);
}

// Contraction of Glob_D, src/workproc.f90:2127-2142: one CTA per function.
__global__ void __launch_bounds__(256) k_contract(const cd* __restrict__ D, int ldo, int npt,
                                                  const cd* __restrict__ cvec, double E, int nfo, int nfa,
                                                  int nfru, double* __restrict__ grad)
{
    __shared__ double sw[8][32][2];
    const int k = blockIdx.x;  // 0-based row of Glob_D's second index
    if (k >= nfo) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n2 = 2 * npt;
    cd W = mk(0.0, 0.0);
    if (lane < npt) {
        for (int l = w; l < nfa; l += 8) {
            const cd* d = D + ((size_t)k + (size_t)l * ldo) * n2;
            const cd t = ldcd(cvec + l);
            const cd dh = ldcd(d + lane), ds = ldcd(d + npt + lane);
            W = cfma(t, dh - E * ds, W);
        }
    }
    sw[w][lane][0] = W.x;
    sw[w][lane][1] = W.y;
    __syncthreads();
    if (w == 0 && lane < npt) {
        cd s = mk(0.0, 0.0);
        for (int q = 0; q < 8; q++) s = s + mk(sw[q][lane][0], sw[q][lane][1]);
        const cd t = ldcd(cvec + k + nfru);
        const cd* d = D + ((size_t)k + (size_t)(k + nfru) * ldo) * n2;
        const cd dd = ldcd(d + lane) - E * ldcd(d + npt + lane);
        double g = 2.0 * cmul(conj(t), s).x;
        g = g - cmul(cmul(t, conj(t)), dd).x;
        grad[(size_t)k * npt + lane] = g;
    }
}

// One MatrixElements call per thread (explicit bra/ket parameters, term t).
template <int N>
__global__ void __launch_bounds__(128) k_term_batch(SysParams sp, const double* __restrict__ Pd, int count,
                                                    const double* __restrict__ pk, const double* __restrict__ pl,
                                                    const int* __restrict__ term, int gradflag, cd* __restrict__ hs,
                                                    cd* __restrict__ dko, cd* __restrict__ dlo)
{
    constexpr int NP = Sym<N>::NP;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double* a = pk + (size_t)i * 2 * NP;
    const double* b = pl + (size_t)i * 2 * NP;
    double P[N][N];
    load_P<N>(Pd, term[i], P);
    cd Ck[N][N], tCl[N][N];
    double dk, dl;
    make_bra<N>(a, Ck, dk);
    make_ket<N>(b, P, tCl, dl);
    TermEnergy<N> te;
    term_energy<N, true>(Ck, tCl, fabs(dl * dk), sp, te);
    hs[2 * (size_t)i] = te.T + te.V;
    hs[2 * (size_t)i + 1] = te.S;
    if (gradflag < 1 || gradflag > 3) return;
    double Lk[N][N], Ll[N][N];
    load_L<N>(a, Lk);
    load_L<N>(b, Ll);
    cd Dk[4 * NP], Dl[4 * NP];
    if (gradflag == 1)
        term_grad_plain<N, true, false>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
    else if (gradflag == 2)
        term_grad_plain<N, false, true>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
    else
        term_grad_plain<N, true, true>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
    if (gradflag & 1)
        for (int m = 0; m < 4 * NP; m++) dko[(size_t)i * 4 * NP + m] = Dk[m];
    if (gradflag & 2)
        for (int m = 0; m < 4 * NP; m++) dlo[(size_t)i * 4 * NP + m] = Dl[m];
}

// ---------------------------------------------------------------------------
// Candidate rows (the BasisEnlI trial loop, src/workproc.f90:4054-4070, where
// each trial function becomes row nbase+1 of H and S).  Candidate j is the
// bra, base function q the permuted ket, as for row k = nbase+1 of
// ComputeMatElem (src/matform.f90:160-177); the StoreHS 'I' normalisation
// (src/matform.f90:22-35) is applied and the row is kept as the upper column
// it mirrors into: Mcol(q, j) = conj(M(K, q)), Scol(q, j) = conj(S(K, q)).
// ---------------------------------------------------------------------------

// Diagonal pair (K, K) of every candidate: diagS and M(K, K).
template <int N>
__global__ void __launch_bounds__(128) k_cand_diag(SysParams sp, const double* __restrict__ coef,
                                                   const cd* __restrict__ cbra, const cd* __restrict__ cket,
                                                   const double* __restrict__ cdet, int count, double approx_e,
                                                   double* __restrict__ cdS, double* __restrict__ cmu)
{
    constexpr int NP = Sym<N>::NP;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    cd Ck[N][N];
    load_sym<N>(cbra + (size_t)j * NP, Ck);
    const double dj = cdet[j];
    const double absdet = fabs(dj * dj);
    cd Hs = mk(0.0, 0.0), Ss = mk(0.0, 0.0);
    for (int t = 0; t < sp.T; t++) {
        cd tCl[N][N];
        load_sym<N>(cket + ((size_t)j * sp.T + t) * NP, tCl);
        TermEnergy<N> te;
        term_energy<N, false>(Ck, tCl, absdet, sp, te);
        const double cf = coef[t];
        Hs = rfma(cf, te.T + te.V, Hs);
        Ss = rfma(cf, te.S, Ss);
    }
    cdS[j] = Ss.x;
    cmu[j] = Hs.x / Ss.x - approx_e;
}

// Off-diagonal pairs (K, q), q < nbase, for all candidates.  Lanes run along
// q (the contiguous index of the stored columns), the W warps of a CTA over
// candidates, CPW candidates per warp.
template <int N, int W, int CPW>
__global__ void __launch_bounds__(W * 32) k_cand_row(SysParams sp, const double* __restrict__ coef,
                                                     const cd* __restrict__ cbra, const double* __restrict__ cdet,
                                                     const double* __restrict__ cdS, const cd* __restrict__ ket,
                                                     const double* __restrict__ detL,
                                                     const double* __restrict__ diagS, int nbase, int count,
                                                     double approx_e, cd* __restrict__ Mcol, cd* __restrict__ Scol,
                                                     int ldv)
{
    constexpr int NP = Sym<N>::NP;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int q = blockIdx.x * 32 + lane;
    if (q >= nbase) return;
    const double dq = detL[q];
    const double dSq = diagS[q];
#pragma unroll 1
    for (int u = 0; u < CPW; u++) {
        const int j = (blockIdx.y * W + w) * CPW + u;
        if (j >= count) break;
        cd Ck[N][N];
        load_sym<N>(cbra + (size_t)j * NP, Ck);
        const double absdet = fabs(dq * cdet[j]);
        cd Hs = mk(0.0, 0.0), Ss = mk(0.0, 0.0);
#pragma unroll 1
        for (int t = 0; t < sp.T; t++) {
            cd tCl[N][N];
            load_sym<N>(ket + ((size_t)q * sp.T + t) * NP, tCl);
            TermEnergy<N> te;
            term_energy<N, false>(Ck, tCl, absdet, sp, te);
            const double cf = __ldg(coef + t);
            Hs = rfma(cf, te.T + te.V, Hs);
            Ss = rfma(cf, te.S, Ss);
        }
        const double f = 1.0 / sqrt(cdS[j] * dSq);
        const size_t o = (size_t)q + (size_t)j * ldv;
        const cd s = f * Ss;
        const cd m = f * (Hs - approx_e * Ss);
        stcd(Scol + o, conj(s));
        stcd(Mcol + o, conj(m));
    }
}

// Gradient of every candidate's energy with respect to its own parameters:
// what EnergyIB(nbase, nbase+1) (src/workproc.f90:2063-2154, nfo = 1) returns
// once candidate j is function K = nbase+1 and its eigenpair is (E_j, c),
// c = x / sqrt(x^H S x) (SpecifNorm 0).  Only the pairs (K, q), q <= nbase,
// hold derivatives with respect to function K; each is recomputed with the
// bra derivative contracted (term_adjoint) and weighted w = conj(c_K) c_q
// f_Kq, q = nbase being the diagonal pair (the candidate with itself).
// CTA (chunk, j): 128 threads over q, summed in a fixed order (butterflies,
// then warps in order) into part[(j * nchunk + chunk) * NV].
constexpr int CAND_ADJ_NT = 128;

template <int N>
__global__ void __launch_bounds__(CAND_ADJ_NT) k_cand_adjoint(
    SysParams sp, const double* __restrict__ coef, const double* __restrict__ Pd, const cd* __restrict__ cbra,
    const cd* __restrict__ cket, const double* __restrict__ cdet, const double* __restrict__ cdS,
    const cd* __restrict__ ket, const double* __restrict__ detL, const double* __restrict__ diagS, int nbase,
    const cd* __restrict__ V, int ldv, const cd* __restrict__ vK, const double* __restrict__ t1,
    const double* __restrict__ energy, const int* __restrict__ err, double* __restrict__ part)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = AdjNV<N>::value;
    __shared__ double red[CAND_ADJ_NT / 32][NV];
    const int j = blockIdx.y;
    const int q = blockIdx.x * CAND_ADJ_NT + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double v[NV];
#pragma unroll
    for (int x = 0; x < NV; x++) v[x] = 0.0;
    if (q <= nbase && err[j] != 1) {
        const double rs = 1.0 / sqrt(t1[j]);
        const double E = energy[j];
        const cd cK = rs * vK[j];
        const bool dg = (q == nbase);
        cd Ck[N][N];
        load_sym<N>(cbra + (size_t)j * NP, Ck);
        const cd* kq = dg ? cket + (size_t)j * sp.T * NP : ket + (size_t)q * sp.T * NP;
        const double dq = dg ? cdet[j] : detL[q];
        const double dSq = dg ? cdS[j] : diagS[q];
        const cd cq = dg ? cK : rs * ldcd(V + (size_t)j * ldv + q);
        const double absdet = fabs(dq * cdet[j]);
        cd Zk[NP], Zl[NP], a = mk(0.0, 0.0);
#pragma unroll
        for (int x = 0; x < NP; x++) Zk[x] = mk(0.0, 0.0);
#pragma unroll 1
        for (int t = 0; t < sp.T; t++) {
            cd tCl[N][N];
            load_sym<N>(kq + (size_t)t * NP, tCl);
            TermEnergy<N> te;
            term_energy<N, true>(Ck, tCl, absdet, sp, te);
            double P[N][N];
            load_P<N>(Pd, t, P);
            term_adjoint<N, false>(P, Ck, tCl, te, sp, E, __ldg(coef + t), Zk, Zl, a);
        }
        const cd wq = (1.0 / sqrt(cdS[j] * dSq)) * cmul(conj(cK), cq);
#pragma unroll
        for (int x = 0; x < NP; x++) {
            const cd z = cmul(wq, Zk[x]);
            v[2 * x] = z.x;
            v[2 * x + 1] = z.y;
        }
        v[NV - 1] = cmul(wq, a).x;
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1)
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += __shfl_xor_sync(0xffffffffu, v[x], s);
    if (lane == 0)
#pragma unroll
        for (int x = 0; x < NV; x++) red[w][x] = v[x];
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
#pragma unroll
        for (int u = 0; u < CAND_ADJ_NT / 32; u++) s += red[u][threadIdx.x];
        part[((size_t)j * gridDim.x + blockIdx.x) * NV + threadIdx.x] = s;
    }
}

// One warp per candidate: the chunk sums in order, then the gradient
// (NaN where the candidate's factorisation hit a zero pivot).
template <int N>
__global__ void __launch_bounds__(256) k_cand_adjoint_final(const double* __restrict__ part, int nchunk,
                                                            const double* __restrict__ cpar,
                                                            const int* __restrict__ err, int count,
                                                            double* __restrict__ grad)
{
    constexpr int NP = Sym<N>::NP;
    constexpr int NV = AdjNV<N>::value;
    const int lane = threadIdx.x & 31;
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    if (j >= count) return;
    double v[NV];
#pragma unroll
    for (int x = 0; x < NV; x++) v[x] = 0.0;
    for (int u = lane; u < nchunk; u += 32) {
        const double* src = part + ((size_t)j * nchunk + u) * NV;
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += src[x];
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1)
#pragma unroll
        for (int x = 0; x < NV; x++) v[x] += __shfl_xor_sync(0xffffffffu, v[x], s);
    double* g = grad + (size_t)j * 2 * NP;
    if (err[j] == 1) {
        if (lane < 2 * NP) g[lane] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    adj_gradient<N>(v, cpar + (size_t)j * 2 * NP, lane, g);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Overlap penalty, ComputeOverlapPenalty / ComputeOverlapPenaltyAndAddGradient
// (src/workproc.f90:1491-1693): P = sum over pairs i < j, j > nfru, of
// pc (|S~_ji|^2 - t2) where |S~_ji|^2 > t2, pc = b / (1 - t2).  One CTA per
// function r of the optimised range; its threads scan the partners p of r in
// the normalised overlap Glob_S (lower triangle).  The pair (j = max, i =
// min) adds to the penalty in the CTA of its larger index.  With a gradient
// mode, the derivatives the reference reads from Glob_D are recomputed here
// for the flagged pairs only (usually few): the S part of Glob_D(., r-nfru,
// p) (the pair's term sum times 1/sqrt(diagS_r diagS_p), conjugated when r
// is the column function) and of the diagonal Glob_D(., r-nfru, r) (2 Re of
// the term sum over diagS_r), so no derivative array is needed.  Mode 1 adds
// the reference's expression, mode 2 the derivative of the penalty (no
// sqrt(diagS_i/diagS_j) factor, |S~|^2 for the lower-index function).  Each
// CTA sums its partners in a fixed order.
// ---------------------------------------------------------------------------
constexpr int PEN_NT = 128;

template <int N>
__device__ void pen_pair_deriv(const SysParams& sp, const double* __restrict__ coef,
                               const double* __restrict__ Pd, const double* __restrict__ params,
                               const cd* __restrict__ bra, const cd* __restrict__ ket,
                               const double* __restrict__ detL, int k, int l, bool want_row, cd* out)
{
    // sum over terms of dS(k,l) w.r.t. the row function k (want_row) or the
    // column function l; out receives 2 NP complex values (vech L, vech B)
    constexpr int NP = Sym<N>::NP;
    cd Ck[N][N];
    load_sym<N>(bra + (size_t)k * NP, Ck);
    double Lk[N][N], Ll[N][N];
    load_L<N>(params + (size_t)k * 2 * NP, Lk);
    load_L<N>(params + (size_t)l * 2 * NP, Ll);
    const double absdet = fabs(detL[l] * detL[k]);
    for (int m = 0; m < 2 * NP; m++) out[m] = mk(0.0, 0.0);
    for (int t = 0; t < sp.T; t++) {
        cd tCl[N][N];
        load_sym<N>(ket + ((size_t)l * sp.T + t) * NP, tCl);
        TermEnergy<N> te;
        term_energy<N, true>(Ck, tCl, absdet, sp, te);
        double P[N][N];
        load_P<N>(Pd, t, P);
        cd Dk[4 * NP], Dl[4 * NP];
        term_grad_plain<N, true, true>(Lk, Ll, P, Ck, tCl, te, sp, Dk, Dl);
        const double cf = coef[t];
        const cd* d = want_row ? Dk : Dl;
#pragma unroll
        for (int m = 0; m < 2 * NP; m++) out[m] = rfma(cf, d[2 * NP + m], out[m]);
    }
}

template <int N>
__global__ void __launch_bounds__(PEN_NT) k_penalty(SysParams sp, const double* __restrict__ coef,
                                                    const double* __restrict__ Pd,
                                                    const double* __restrict__ params, const cd* __restrict__ bra,
                                                    const cd* __restrict__ ket, const double* __restrict__ detL,
                                                    const double* __restrict__ diagS, const cd* __restrict__ S,
                                                    int ld, int nfru, int nfa, double t2, double pc, int mode,
                                                    double* __restrict__ grad, double* __restrict__ part)
{
    constexpr int NP = Sym<N>::NP, NPT = 2 * NP;
    __shared__ double sg[NPT][PEN_NT];
    __shared__ double stp[PEN_NT];
    __shared__ double sdd[NPT];
    const int tid = threadIdx.x;
    const int r = nfru + blockIdx.x;
    const double dr = diagS[r];
    double tp = 0.0;
    bool flagged = false;
    for (int p = tid; p < nfa; p += PEN_NT) {
        if (p == r) continue;
        const int j = max(p, r), i = min(p, r);
        const cd s = S[(size_t)j + (size_t)i * ld];
        const double aux = s.x * s.x + s.y * s.y;
        if (aux > t2) {
            flagged = true;
            if (p < r) tp += pc * (aux - t2);
        }
    }
    stp[tid] = tp;
    const int any = __syncthreads_or(flagged ? 1 : 0);
    if (tid == 0) {
        double a = 0.0;
        for (int t = 0; t < PEN_NT; t++) a += stp[t];
        part[blockIdx.x] = a;
    }
    if (mode == 0 || !any) return;
    if (tid == 0) {
        // Glob_D(npt+m, r-nfru, r) = 2 Re(sum_t coef_t dS_rr/dp_m) / diagS_r
        cd d[NPT];
        pen_pair_deriv<N>(sp, coef, Pd, params, bra, ket, detL, r, r, true, d);
        for (int m = 0; m < NPT; m++) sdd[m] = 2.0 * d[m].x / dr;
    }
    for (int m = 0; m < NPT; m++) sg[m][tid] = 0.0;
    __syncthreads();
    const double temp1 = 2.0 * pc;
    for (int p = tid; p < nfa; p += PEN_NT) {
        if (p == r) continue;
        const int j = max(p, r), i = min(p, r);
        const cd s = S[(size_t)j + (size_t)i * ld];
        const double aux = s.x * s.x + s.y * s.y;
        if (!(aux > t2)) continue;
        cd d[NPT];
        const bool row = (r == j);
        pen_pair_deriv<N>(sp, coef, Pd, params, bra, ket, detL, j, i, row, d);
        const double f = 1.0 / sqrt(diagS[j] * diagS[i]);
        const double temp2 = (mode == 2) ? 1.0 : sqrt(diagS[i] / diagS[j]);
        for (int m = 0; m < NPT; m++) {
            cd g;
            if (row) {
                // Glob_D(npt+m, j-nfru, i) = f dS_ji/dp_j
                const cd dji = f * d[m];
                const cd x = dji - (0.5 * sdd[m] * temp2) * s;
                g = s * conj(x);
            } else {
                // Glob_D(npt+m, i-nfru, j) = conj(f dS_ji/dp_i)
                const cd dij = conj(f * d[m]);
                const cd sn = (mode == 2) ? conj(s) : s;
                const cd x = dij - (0.5 * sdd[m] / temp2) * sn;
                g = s * x;
            }
            sg[m][tid] += temp1 * g.x;
        }
    }
    __syncthreads();
    for (int m = tid; m < NPT; m += PEN_NT) {
        double a = 0.0;
        for (int t = 0; t < PEN_NT; t++) a += sg[m][t];
        grad[(size_t)(r - nfru) * NPT + m] += a;
    }
}

#define ECG_DISPATCH_N(n, FN, ...)              \
    switch (n) {                                \
        case 2: return FN<2>(__VA_ARGS__);      \
        case 3: return FN<3>(__VA_ARGS__);      \
        case 4: return FN<4>(__VA_ARGS__);      \
        case 5: return FN<5>(__VA_ARGS__);      \
        default: return -1;                     \
    }

static int last_err() { return cudaGetLastError() == cudaSuccess ? 0 : -2; }

template <int N>
static int prep_n(Ctx& c, int nfun)
{
    if (nfun <= 0) return 0;
    k_prep<N><<<(nfun + 127) / 128, 128, 0, c.stream>>>(c.params, c.Pd, c.T, nfun, c.bra, c.ket, c.detL);
    c.launches++;
    return last_err();
}
int launch_prep(Ctx& c, int nfun) { ECG_DISPATCH_N(c.n, prep_n, c, nfun) }

template <int N>
static int diag_n(Ctx& c, int r0, int r1, double approx_e, int deriv, int nfru)
{
    if (r1 <= r0) return 0;
    const int nb = (r1 - r0 + 127) / 128;
    if (deriv)
        k_pair_diag<N, true><<<nb, 128, 0, c.stream>>>(c.sp, c.coef, c.Pd, c.params, c.bra, c.ket, c.detL, c.diagS,
                                                       c.diagH, c.H, c.S, c.ld, r0, r1, c.method, approx_e, c.D,
                                                       c.max_nfo, nfru);
    else
        k_pair_diag<N, false><<<nb, 128, 0, c.stream>>>(c.sp, c.coef, c.Pd, c.params, c.bra, c.ket, c.detL,
                                                        c.diagS, c.diagH, c.H, c.S, c.ld, r0, r1, c.method,
                                                        approx_e, c.D, c.max_nfo, nfru);
    c.launches++;
    return last_err();
}
template <int N>
static int penalty_n(Ctx& c, int nfru, int nfa, double t2, double pc, int mode, double* part)
{
    k_penalty<N><<<nfa - nfru, PEN_NT, 0, c.stream>>>(c.sp, c.coef, c.Pd, c.params, c.bra, c.ket, c.detL, c.diagS,
                                                      c.S, c.ld, nfru, nfa, t2, pc, mode, c.grad, part);
    c.launches++;
    return last_err();
}
int launch_penalty(Ctx& c, int nfru, int nfa, double t2, double pc, int mode, double* part)
{
    ECG_DISPATCH_N(c.n, penalty_n, c, nfru, nfa, t2, pc, mode, part)
}

int launch_pair_diag(Ctx& c, int r0, int r1, double approx_e, int deriv, int nfru)
{
    ECG_DISPATCH_N(c.n, diag_n, c, r0, r1, approx_e, deriv, nfru)
}

// The pair-kernel shapes the autotuner chooses from: k_pair_energy (warps
// per tile, minimum CTAs per SM), k_adjoint (minimum CTAs per SM).
template <int N>
static void pair_energy_launch(Ctx& c, int v, unsigned grid, int r0, int r1, int Rlo, double approx_e, long long t0)
{
    switch (v) {
        case 0:
            k_pair_energy<N, 8, 2><<<grid, 256, 0, c.stream>>>(c.sp, c.coef, c.bra, c.ket, c.detL, c.diagS, c.H, c.S,
                                                               c.ld, r0, r1, Rlo, c.method, approx_e, t0);
            break;
        case 1:
            k_pair_energy<N, 8, 3><<<grid, 256, 0, c.stream>>>(c.sp, c.coef, c.bra, c.ket, c.detL, c.diagS, c.H, c.S,
                                                               c.ld, r0, r1, Rlo, c.method, approx_e, t0);
            break;
        case 2:
            k_pair_energy<N, 4, 2><<<grid, 128, 0, c.stream>>>(c.sp, c.coef, c.bra, c.ket, c.detL, c.diagS, c.H, c.S,
                                                               c.ld, r0, r1, Rlo, c.method, approx_e, t0);
            break;
        default:
            k_pair_energy<N, 4, 4><<<grid, 128, 0, c.stream>>>(c.sp, c.coef, c.bra, c.ket, c.detL, c.diagS, c.H, c.S,
                                                               c.ld, r0, r1, Rlo, c.method, approx_e, t0);
            break;
    }
}

// Time every shape once on this launch (the last run's results stand:
// all shapes write the same values) and keep the fastest for the context.
template <typename F>
static int tune(Ctx& c, int nshapes, int& choice, float* ms_out, F run)
{
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -2;
    float best = 1e30f;
    int bv = 0;
    for (int v = 0; v < nshapes; v++) {
        cudaEventRecord(e0, c.stream);
        run(v);
        cudaEventRecord(e1, c.stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return -2;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms_out) ms_out[v] = ms;
        if (ms < best) {
            best = ms;
            bv = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // rerun the chosen shape last unless it already was
    if (bv != nshapes - 1) run(bv);
    choice = bv;
    return last_err();
}

template <int N>
static int energy_n(Ctx& c, int r0, int r1, double approx_e)
{
    if (r1 <= r0) return 0;
    const int Rlo = r0 / TILE, Rhi = (r1 + TILE - 1) / TILE;
    const long long nt = tile_count(Rlo, Rhi);
    c.launches++;
    // shapes are tuned on the first launch with at least 256 tiles
    if (c.tune_pair < 0 && nt >= 256)
        return tune(c, PAIR_SHAPES, c.tune_pair, c.tune_pair_ms, [&](int v) {
            pair_energy_launch<N>(c, v, (unsigned)nt, r0, r1, Rlo, approx_e, 0LL);
        });
    pair_energy_launch<N>(c, c.tune_pair < 0 ? 0 : c.tune_pair, (unsigned)nt, r0, r1, Rlo, approx_e, 0LL);
    return last_err();
}
int launch_pair_energy(Ctx& c, int r0, int r1, double approx_e) { ECG_DISPATCH_N(c.n, energy_n, c, r0, r1, approx_e) }

// Tiles [t0, t0 + count) of the list k_pair_energy walks for rows [r0, r1).
template <int N>
static int energy_tiles_n(Ctx& c, int r0, int r1, double approx_e, long long t0, long long count)
{
    if (r1 <= r0 || count <= 0) return 0;
    const int Rlo = r0 / TILE;
    pair_energy_launch<N>(c, c.tune_pair < 0 ? 0 : c.tune_pair, (unsigned)count, r0, r1, Rlo, approx_e, t0);
    c.launches++;
    return last_err();
}
int launch_pair_energy_tiles(Ctx& c, int r0, int r1, double approx_e, long long t0, long long count)
{
    ECG_DISPATCH_N(c.n, energy_tiles_n, c, r0, r1, approx_e, t0, count)
}

// Pack (dir 0) or unpack (dir 1) the off-diagonal entries k > l, k in
// [r0, r1), of tiles [t0, t0 + count) of that list: buf holds per tile H
// then S as [l][k] 32 x 32 complex blocks; unpacking writes H(k,l), S(k,l)
// and, in 'I' storage, S(l,k) = conj(S(k,l)), as k_pair_energy stores them.
__global__ void __launch_bounds__(256) k_tiles_copy(cd* __restrict__ H, cd* __restrict__ S, int ld, int r0, int r1,
                                                    int Rlo, long long t0, cd* __restrict__ buf, int dir, char method)
{
    int R, C;
    tile_rc(t0 + blockIdx.x, Rlo, R, C);
    cd* tb = buf + (size_t)blockIdx.x * 2 * TILE * TILE;
    for (int e = threadIdx.x; e < TILE * TILE; e += blockDim.x) {
        const int lk = e & 31, ll = e >> 5;
        const int k = R * TILE + lk, l = C * TILE + ll;
        if (k < r0 || k >= r1 || l >= k) continue;
        const size_t kl = (size_t)k + (size_t)l * ld;
        if (dir == 0) {
            tb[e] = H[kl];
            tb[TILE * TILE + e] = S[kl];
        } else {
            const cd sv = tb[TILE * TILE + e];
            H[kl] = tb[e];
            S[kl] = sv;
            if (method == 'I') S[(size_t)l + (size_t)k * ld] = conj(sv);
        }
    }
}
int launch_tiles_copy(Ctx& c, int r0, int r1, long long t0, long long count, cd* buf, int dir)
{
    if (r1 <= r0 || count <= 0) return 0;
    k_tiles_copy<<<(unsigned)count, 256, 0, c.stream>>>(c.H, c.S, c.ld, r0, r1, r0 / TILE, t0, buf, dir, c.method);
    c.launches++;
    return last_err();
}

template <int N>
static int grad_n(Ctx& c, int r0, int r1, int nfru, double approx_e)
{
    if (r1 <= r0) return 0;
    constexpr int NT = (N <= 4) ? 128 : 64;
    constexpr int NP = Sym<N>::NP;
    const size_t smem = (size_t)16 * NP * NT * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_pair_grad<N, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    const int Rlo = r0 / TILE, Rhi = (r1 + TILE - 1) / TILE;
    const long long nt = tile_count(Rlo, Rhi);
    k_pair_grad<N, NT><<<(unsigned)nt, NT, smem, c.stream>>>(c.sp, c.coef, c.Pd, c.params, c.bra, c.ket, c.detL,
                                                             c.diagS, c.H, c.S, c.ld, r0, r1, Rlo, c.method,
                                                             approx_e, c.D, c.max_nfo, nfru);
    c.launches++;
    return last_err();
}
int launch_pair_plain_grad(Ctx& c, int r0, int r1, int nfru, double approx_e)
{
    ECG_DISPATCH_N(c.n, grad_n, c, r0, r1, nfru, approx_e)
}

template <int N>
static int adjoint_n(Ctx& c, int nfru, int nfa, double E)
{
    if (nfa <= nfru) return 0;
    constexpr int NV = AdjNV<N>::value;
    const int Rlo = nfru / TILE, Rhi = (nfa + TILE - 1) / TILE;
    const long long nt = tile_count(Rlo, Rhi);
    const size_t need = (size_t)nt * 2 * TILE * NV * sizeof(double);
    if (need > c.part_bytes) {
        if (c.part) cudaFree(c.part);
        c.part = nullptr;
        c.part_bytes = 0;
        if (cudaMalloc(&c.part, need) != cudaSuccess) return -3;
        c.part_bytes = need;
    }
    const size_t smem = (size_t)8 * TILE * NV * sizeof(double);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adjoint<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_adjoint<N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    auto run = [&](int v) {
        if (v == 0)
            k_adjoint<N, 1><<<(unsigned)nt, 256, smem, c.stream>>>(c.sp, c.coef, c.Pd, c.bra, c.ket, c.detL, c.diagS,
                                                                   c.c, E, nfru, nfa, Rlo, c.part, 0LL);
        else
            k_adjoint<N, 2><<<(unsigned)nt, 256, smem, c.stream>>>(c.sp, c.coef, c.Pd, c.bra, c.ket, c.detL, c.diagS,
                                                                   c.c, E, nfru, nfa, Rlo, c.part, 0LL);
    };
    c.launches++;
    if (c.tune_adj < 0 && nt >= 256) {
        const int r = tune(c, ADJ_SHAPES, c.tune_adj, c.tune_adj_ms, run);
        if (r) return r;
    } else {
        run(c.tune_adj < 0 ? 0 : c.tune_adj);
    }
    const int nf = nfa - nfru;
    k_adjoint_final<N><<<(nf * 32 + 255) / 256, 256, 0, c.stream>>>(c.part, c.params, nfru, nfa, Rlo, Rhi, c.grad);
    c.launches++;
    return last_err();
}
int launch_adjoint(Ctx& c, int nfru, int nfa, double E) { ECG_DISPATCH_N(c.n, adjoint_n, c, nfru, nfa, E) }

// The adjoint pass over tiles [t0, t0 + count) of its list only, with the
// eigenvector cvec; part receives their partials (count x 2 x 32 x NV),
// in the order the whole pass writes them.
template <int N>
static int adjoint_tiles_n(Ctx& c, int nfru, int nfa, double E, const cd* cvec, long long t0, long long count,
                           double* part)
{
    if (nfa <= nfru || count <= 0) return 0;
    constexpr int NV = AdjNV<N>::value;
    const size_t smem = (size_t)8 * TILE * NV * sizeof(double);
    if (cudaFuncSetAttribute(k_adjoint<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -2;
    k_adjoint<N, 1><<<(unsigned)count, 256, smem, c.stream>>>(c.sp, c.coef, c.Pd, c.bra, c.ket, c.detL, c.diagS,
                                                              cvec, E, nfru, nfa, nfru / TILE, part, t0);
    c.launches++;
    return last_err();
}
int launch_adjoint_tiles(Ctx& c, int nfru, int nfa, double E, const cd* cvec, long long t0, long long count,
                         double* part)
{
    ECG_DISPATCH_N(c.n, adjoint_tiles_n, c, nfru, nfa, E, cvec, t0, count, part)
}

// The gradient from the partials of every tile of the list, in list order.
template <int N>
static int adjoint_finish_n(Ctx& c, int nfru, int nfa, const double* part)
{
    if (nfa <= nfru) return 0;
    const int Rlo = nfru / TILE, Rhi = (nfa + TILE - 1) / TILE;
    const int nf = nfa - nfru;
    k_adjoint_final<N><<<(nf * 32 + 255) / 256, 256, 0, c.stream>>>(part, c.params, nfru, nfa, Rlo, Rhi, c.grad);
    c.launches++;
    return last_err();
}
int launch_adjoint_finish(Ctx& c, int nfru, int nfa, const double* part)
{
    ECG_DISPATCH_N(c.n, adjoint_finish_n, c, nfru, nfa, part)
}
int adjoint_nv(int n) { return 2 * (n * (n + 1) / 2) + 1; }

int launch_plain_contract(Ctx& c, int nfo, int nfa, int nfru, double E)
{
    if (nfo <= 0) return 0;
    k_contract<<<nfo, 256, 0, c.stream>>>(c.D, c.max_nfo, c.npt, c.c, E, nfo, nfa, nfru, c.grad);
    c.launches++;
    return last_err();
}

template <int N>
static int batch_n(Ctx& c, int count, const double* pk, const double* pl, const int* term, int gradflag, cd* hs,
                   cd* dk, cd* dl)
{
    if (count <= 0) return 0;
    k_term_batch<N><<<(count + 127) / 128, 128, 0, c.stream>>>(c.sp, c.Pd, count, pk, pl, term, gradflag, hs, dk,
                                                               dl);
    c.launches++;
    return last_err();
}
int launch_term_batch(Ctx& c, int count, const double* pk, const double* pl, const int* term, int gradflag, cd* hs,
                      cd* dk, cd* dl)
{
    ECG_DISPATCH_N(c.n, batch_n, c, count, pk, pl, term, gradflag, hs, dk, dl)
}

// Candidate rows.  variant = tile shape of k_cand_row (CAND_ROW_SHAPES):
// warps per CTA x candidates per warp.
template <int N, int W, int CPW>
static void cand_row_launch(Ctx& c, CandWork& cw, int nbase, int count, double approx_e)
{
    dim3 g((nbase + 31) / 32, (count + W * CPW - 1) / (W * CPW));
    k_cand_row<N, W, CPW><<<g, W * 32, 0, c.stream>>>(c.sp, c.coef, cw.bra, cw.det, cw.dS, c.ket, c.detL, c.diagS,
                                                      nbase, count, approx_e, cw.Mcol, cw.Scol, cw.ldv);
}

template <int N>
static int cand_rows_n(Ctx& c, CandWork& cw, int nbase, int count, double approx_e, int variant)
{
    if (count <= 0) return 0;
    k_prep<N><<<(count + 127) / 128, 128, 0, c.stream>>>(cw.par, c.Pd, c.T, count, cw.bra, cw.ket, cw.det);
    k_cand_diag<N><<<(count + 127) / 128, 128, 0, c.stream>>>(c.sp, c.coef, cw.bra, cw.ket, cw.det, count, approx_e,
                                                              cw.dS, cw.mu);
    c.launches += 2;
    if (nbase > 0) {
        switch (variant) {
            case 0: cand_row_launch<N, 4, 1>(c, cw, nbase, count, approx_e); break;
            case 1: cand_row_launch<N, 4, 2>(c, cw, nbase, count, approx_e); break;
            case 2: cand_row_launch<N, 8, 1>(c, cw, nbase, count, approx_e); break;
            case 3: cand_row_launch<N, 8, 2>(c, cw, nbase, count, approx_e); break;
            default: cand_row_launch<N, 8, 4>(c, cw, nbase, count, approx_e); break;
        }
        c.launches++;
    }
    return last_err();
}
int launch_cand_rows(Ctx& c, CandWork& cw, int nbase, int count, double approx_e, int variant)
{
    ECG_DISPATCH_N(c.n, cand_rows_n, c, cw, nbase, count, approx_e, variant)
}

template <int N>
static int cand_adjoint_n(Ctx& c, CandWork& cw, int nbase, int count, const cd* vK, const double* t1,
                          const double* energy, const int* err, double* grad)
{
    constexpr int NV = AdjNV<N>::value;
    const int nchunk = nbase / CAND_ADJ_NT + 1;  // q = 0..nbase
    if ((size_t)nchunk * count * NV > cw.gpart_n) return -1;
    k_cand_adjoint<N><<<dim3(nchunk, count), CAND_ADJ_NT, 0, c.stream>>>(c.sp, c.coef, c.Pd, cw.bra, cw.ket, cw.det,
                                                                         cw.dS, c.ket, c.detL, c.diagS, nbase, cw.V,
                                                                         cw.ldv, vK, t1, energy, err, cw.gpart);
    k_cand_adjoint_final<N><<<(count * 32 + 255) / 256, 256, 0, c.stream>>>(cw.gpart, nchunk, cw.par, err, count,
                                                                           grad);
    c.launches += 2;
    return last_err();
}
int launch_cand_adjoint(Ctx& c, CandWork& cw, int nbase, int count, const cd* vK, const double* t1,
                        const double* energy, const int* err, double* grad)
{
    ECG_DISPATCH_N(c.n, cand_adjoint_n, c, cw, nbase, count, vK, t1, energy, err, grad)
}

}  // namespace ecg

// ---------------------------------------------------------------------------
// Adjoint gradient without any device allocation (ecg_adjoint_gradient_noalloc).
//
// Some hosts cannot allocate device memory at the point where they need the
// gradient: an application that owns all GPU memory through its own pool and
// forbids stray allocations, an optimiser callback that must not fail or
// fragment memory in the middle of a long run, or a service with fixed
// per-tenant memory budgets.  This variant takes every input and output as a
// caller-owned device pointer and keeps all of its working data (per-function
// bra/ket matrices, the projector terms and the per-tile partial sums) in one
// fixed array compiled into the library.  Limits: at most NOALLOC_KMAX basis
// functions and NOALLOC_TMAX projector terms; every GPU that loads the
// library holds the array (about 4.3 MB) until the process exits.  All calls
// on a device share the array, so calls whose GPU work overlaps (different
// streams, other host threads) race on it; each call rewrites every part of
// it that the call reads, so nothing has to start at zero.  The projector
// terms reach the array through the arguments of a small kernel (copied at
// launch), so the call issues no host-to-device copy and does not wait for
// the stream.
// ---------------------------------------------------------------------------
#include <mutex>
#include "../../include/ecg_abi.h"

namespace ecg {
namespace noalloc {

constexpr int KMAX = 512;
constexpr int TMAXN = 16;
constexpr int NPMAX = 15;                  // n(n+1)/2 at n = 5
constexpr int NVMAX = 2 * NPMAX + 1;
constexpr long long TILES = (long long)(KMAX / TILE) * (KMAX / TILE + 1) / 2;

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t OFF_P = 0;
constexpr size_t OFF_COEF = OFF_P + align256(sizeof(double) * TMAXN * NMAX * NMAX);
constexpr size_t OFF_BRA = OFF_COEF + align256(sizeof(double) * TMAXN);
constexpr size_t OFF_KET = OFF_BRA + align256(sizeof(cd) * KMAX * NPMAX);
constexpr size_t OFF_DET = OFF_KET + align256(sizeof(cd) * KMAX * TMAXN * NPMAX);
constexpr size_t OFF_PART = OFF_DET + align256(sizeof(double) * KMAX);
constexpr size_t BYTES = OFF_PART + align256(sizeof(double) * TILES * 2 * TILE * NVMAX);

// The one scratch array.  Host code must not take its address directly (on
// the host the name denotes a stand-in, not device memory); device_base()
// obtains the device address with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[BYTES];

constexpr int MAX_DEVICES = 64;
static std::mutex g_mu;
static unsigned char* g_base[MAX_DEVICES] = {};

// Device address of g_scratch on the current device, looked up once per
// device: the first call on a device does this set-up, so that first call
// should come before any stream capture on the device.
static int device_base(unsigned char** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        cudaGetLastError();
        return ECG_ENODEV;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_base[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return ECG_ECUDA;
        }
        g_base[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_base[dev];
    return ECG_OK;
}

// Projector terms by value (row-major P[t][i][j], then the coefficients):
// 16 * 25 + 16 doubles, well inside the kernel-parameter limit.
struct Terms {
    double P[TMAXN * NMAX * NMAX];
    double coef[TMAXN];
};

__global__ void k_store_terms(const Terms t, int nterms, double* __restrict__ P, double* __restrict__ coef)
{
    for (int e = threadIdx.x; e < nterms * NMAX * NMAX; e += blockDim.x) P[e] = t.P[e];
    for (int e = threadIdx.x; e < nterms; e += blockDim.x) coef[e] = t.coef[e];
}

template <int N>
static int run(const SysParams& sp, const Terms& terms, unsigned char* base, const double* params, const cd* cvec, const double* diagS,
               double E, int nfru, int nfa, double* grad, cudaStream_t st)
{
    constexpr int NV = AdjNV<N>::value;
    double* Pd = reinterpret_cast<double*>(base + OFF_P);
    double* coef = reinterpret_cast<double*>(base + OFF_COEF);
    k_store_terms<<<1, 128, 0, st>>>(terms, sp.T, Pd, coef);
    cd* bra = reinterpret_cast<cd*>(base + OFF_BRA);
    cd* ket = reinterpret_cast<cd*>(base + OFF_KET);
    double* detL = reinterpret_cast<double*>(base + OFF_DET);
    double* part = reinterpret_cast<double*>(base + OFF_PART);
    k_prep<N><<<(nfa + 127) / 128, 128, 0, st>>>(params, Pd, sp.T, nfa, bra, ket, detL);
    const int Rlo = nfru / TILE, Rhi = (nfa + TILE - 1) / TILE;
    const long long nt = tile_count(Rlo, Rhi);
    const size_t smem = (size_t)8 * TILE * NV * sizeof(double);
    if (cudaFuncSetAttribute(k_adjoint<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return ECG_ECUDA;
    }
    k_adjoint<N, 1><<<(unsigned)nt, 256, smem, st>>>(sp, coef, Pd, bra, ket, detL, diagS, cvec, E, nfru, nfa, Rlo, part,
                                                     0LL);
    const int nf = nfa - nfru;
    k_adjoint_final<N><<<(nf * 32 + 255) / 256, 256, 0, st>>>(part, params, nfru, nfa, Rlo, Rhi, grad);
    return cudaGetLastError() == cudaSuccess ? ECG_OK : ECG_ECUDA;
}

}  // namespace noalloc
}  // namespace ecg

extern "C" int ecg_adjoint_gradient_noalloc(int n, const double* mass_matrix_host, const double* charges_host,
                                            int nterms, const int* yhy_mats_host, const int* yhy_coeffs_host,
                                            const double* params_dev, const double* c_dev, const double* diagS_dev,
                                            double energy, int nfru, int nfa, double* grad_dev, void* stream)
{
    using namespace ecg;
    if (n < 2 || n > NMAX || nterms < 1 || nfru < 0 || nfa <= nfru) return ECG_EARG;
    if (!mass_matrix_host || !charges_host || !yhy_mats_host || !yhy_coeffs_host || !params_dev || !c_dev ||
        !diagS_dev || !grad_dev)
        return ECG_EARG;
    if (nfa > noalloc::KMAX || nterms > noalloc::TMAXN) return ECG_ELIMIT;
    cudaGetLastError();  // an error left by the caller's own earlier work is not this call's
    unsigned char* base = nullptr;
    const int rb = noalloc::device_base(&base);
    if (rb != ECG_OK) return rb;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SysParams sp;
    memset(&sp, 0, sizeof(sp));
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) sp.M[i * NMAX + j] = mass_matrix_host[i + j * n];
    sp.q0 = charges_host[0];
    for (int i = 0; i < n; i++) sp.q[i] = charges_host[1 + i];
    sp.two_r3n2 = pow(2.0, (3 * n) / 2.0);
    sp.n = n;
    sp.T = nterms;
    // projector terms (double, row-major P[t][i][j]) travel as kernel arguments
    noalloc::Terms terms;
    memset(&terms, 0, sizeof(terms));
    for (int t = 0; t < nterms; t++) {
        for (int i = 0; i < NMAX; i++)
            for (int j = 0; j < NMAX; j++)
                terms.P[(t * NMAX + i) * NMAX + j] =
                    (i < n && j < n) ? yhy_mats_host[(size_t)t * n * n + i + j * n] : 0.0;
        terms.coef[t] = yhy_coeffs_host[t];
    }
    const cd* cv = reinterpret_cast<const cd*>(c_dev);
    switch (n) {
        case 2: return noalloc::run<2>(sp, terms, base, params_dev, cv, diagS_dev, energy, nfru, nfa, grad_dev, st);
        case 3: return noalloc::run<3>(sp, terms, base, params_dev, cv, diagS_dev, energy, nfru, nfa, grad_dev, st);
        case 4: return noalloc::run<4>(sp, terms, base, params_dev, cv, diagS_dev, energy, nfru, nfa, grad_dev, st);
        default: return noalloc::run<5>(sp, terms, base, params_dev, cv, diagS_dev, energy, nfru, nfa, grad_dev, st);
    }
}
