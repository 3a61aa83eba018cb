// cand.cu -- batched evaluation of candidate basis functions.
//
// The reference's basis enlargement (BasisEnlI, src/workproc.f90:4054-4070)
// tries NTrials candidate functions one after another: each trial writes
// its parameters into column nbase+1 of Glob_NonlinParam and calls
// EnergyIA(nbase+1, nbase+1), i.e. ComputeMatElem for row K = nbase+1 and
// GHEPIIS(K, K, ...) on the factor of the first nbase rows
// (src/linalg.f90:1781-1926).  Here all candidates of one call are
// evaluated together:
//
//   rows        k_cand_diag, k_cand_row (pair_kernels.cu): row K of H and
//               S for every candidate, normalised as StoreHS 'I' does
//   border      the bordered step of LDLHF for row K (src/linalg.f90:
//               359-391): a = L0^-1 M(1:nbase, K) (a multi-right-hand-side
//               forward solve), U(:, K) = invD o a and
//               d_K = conj(M(K, K) - sum_q conj(a_q) U(q, K))
//   iterations  the loop of GHEPIIS (src/linalg.f90:1892-1909) for all
//               candidates at once.  With V the iterates (one column per
//               candidate, rows < nbase) and v_K their border entries:
//                 W = S0 V + S(:,K) v_K,  w_K = S(K,:) V + v_K   (MHMV)
//                 Y = L0^-1 W,  y_K = w_K - U(:,K)^H Y           (LDLHS, L)
//                 Z = invD o Y,  z_K = invD_K y_K,  x_K = z_K     (LDLHS, D)
//                 X = U0^-1 (Z - U(:,K) x_K)                     (LDLHS, L^H)
//               then CMaxAbsReOrIm, CVScale, CDotProdQuotient and
//               CVDiffEucNorm per candidate.  S0 V is a complex GEMM on
//               the FP64 tensor cores; each triangular solve is one
//               cooperative launch over (panel, column block) work items;
//               the bordered row and column enter as rank-one terms.
//   Rayleigh    VMMHMV on S and on M (src/linalg.f90:1913-1917) as two
//               GEMMs (S0 V and the Hermitian M0 V) plus border terms.
//
// One iteration (GEMM, solves, norms) is captured once into a CUDA graph
// and replayed until every candidate has converged or MaxIter is reached;
// converged candidates keep their iterate, exactly as the reference stops
// iterating them.  Every candidate starts from the same vector (the
// context's Glob_LastEigvector(1:K)), so results do not depend on the
// order of the candidates.
#include <float.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include "../../include/ecg_abi.h"
#include "ecg_internal.h"
#include "zmma.cuh"

namespace ecg {

namespace {

__device__ __forceinline__ cd ldcd(const cd* p)
{
    const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// C = op(A) B (+ E1 o e2 per column): M x N complex, inner dimension Kd.
// Column j of B, C, E1 and e2 is physical column cmap[j] (j itself when
// cmap is null): the iterations run on the still-active candidates only.
//   AMODE 0: A(i, k) = A[i + k lda]
//   AMODE 1: A Hermitian, stored in its lower triangle (the lower triangle
//            of Glob_H holds M = H - lambda~ S): A(i, k) = A[i + k lda] for
//            i >= k, conj(A[k + i lda]) for i < k.
// 64 x 64 output tile per CTA, 8 warps as 2 x 4 (32 x 16 each), inner
// chunks of 32 staged by cp.async into two shared-memory stages.
// ---------------------------------------------------------------------------
constexpr int GM = 64, GN = 64, GK = 32;
constexpr int G_LDA = GM + 2;  // % 8 == 2
constexpr int G_LDB = GK + 4;  // % 8 == 4
constexpr int G_STAGE = GK * G_LDA + GN * G_LDB;
constexpr size_t G_SMEM = 2 * (size_t)G_STAGE * sizeof(double2);

template <int AMODE>
__global__ void __launch_bounds__(256) k_zgemm(const cd* __restrict__ A, int lda, int M, int Kd,
                                               const cd* __restrict__ B, int ldb, cd* __restrict__ C, int ldc,
                                               const cd* __restrict__ E1, const cd* __restrict__ e2,
                                               const int* __restrict__ cmap, cd* __restrict__ P, size_t pstride)
{
    extern __shared__ double2 gsm[];
    const int i0 = blockIdx.x * GM, j0 = blockIdx.y * GN;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int wm = (wp >> 2) * 32, wn = (wp & 3) * 16;
    ZAcc<4, 2> acc;
    acc.zero();
    // split K: slice blockIdx.z of gridDim.z takes chunks [kc0, kc1)
    const int nkt = (Kd + GK - 1) / GK;
    const int per = (nkt + gridDim.z - 1) / gridDim.z;
    const int kc0 = blockIdx.z * per, kc1 = min(nkt, kc0 + per);
    const int nk = kc1 > kc0 ? kc1 - kc0 : 0;
    auto stage = [&](int s, int kcl) {
        const int kc = kc0 + kcl;
        double2* As = gsm + s * G_STAGE;
        double2* Bs = As + GK * G_LDA;
        const int k0 = kc * GK;
        // a tile wholly above the diagonal reads A's transpose: walk k fastest
        const bool up = (AMODE == 1) && (i0 + GM <= k0);
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int e = tid + 256 * u;
            const int m = up ? (e >> 5) : (e & 63);
            const int k = up ? (e & 31) : (e >> 6);
            const int i = i0 + m, kk = k0 + k;
            const cd* src = A;
            int bytes = 0;
            if (i < M && kk < Kd) {
                bytes = 16;
                src = (AMODE == 1 && i < kk) ? A + kk + (size_t)i * lda : A + i + (size_t)kk * lda;
            }
            cp_async16(As + k * G_LDA + m, src, bytes);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int e = tid + 256 * u;
            const int k = e & 31, n = e >> 5;
            const int kk = k0 + k;
            const bool ok = kk < Kd;
            const int jp = cmap ? cmap[j0 + n] : j0 + n;
            cp_async16(Bs + n * G_LDB + k, ok ? B + kk + (size_t)jp * ldb : B, ok ? 16 : 0);
        }
        cp_async_commit();
    };
    if (nk > 0) stage(0, 0);
    for (int kcl = 0; kcl < nk; kcl++) {
        if (kcl + 1 < nk) {
            stage((kcl + 1) & 1, kcl + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        double2* As = gsm + (kcl & 1) * G_STAGE;
        const double2* Bs = As + GK * G_LDA;
        const int kc = kc0 + kcl;
        if (AMODE == 1 && i0 < (kc + 1) * GK) {
            // elements read from the upper triangle enter conjugated
            const int k0 = kc * GK;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int e = tid + 256 * u;
                const int m = e & 63, k = e >> 6;
                if (i0 + m < k0 + k) As[k * G_LDA + m].y = -As[k * G_LDA + m].y;
            }
            __syncthreads();
        }
#pragma unroll
        for (int kk = 0; kk < GK; kk += 4) zmma_k4<4, 2, G_LDA, G_LDB, false>(acc, As, Bs, wm, wn, kk, lane);
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 4; mt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int i = i0 + wm + mt * 8 + g;
                const int j = j0 + wn + nt * 8 + 2 * t + e;
                if (i >= M) continue;
                if (gridDim.z > 1) {  // partial sum of this K slice, by slot
                    *reinterpret_cast<double2*>(P + blockIdx.z * pstride + (size_t)i + (size_t)j * ldc) =
                        make_double2(acc.r[mt][nt][e], acc.i[mt][nt][e]);
                    continue;
                }
                const int jp = cmap ? cmap[j] : j;
                cd v = mk(acc.r[mt][nt][e], acc.i[mt][nt][e]);
                const size_t o = (size_t)i + (size_t)jp * ldc;
                if (E1) v = cfma(ldcd(E1 + o), ldcd(e2 + jp), v);
                *reinterpret_cast<double2*>(C + o) = make_double2(v.x, v.y);
            }
}

// ---------------------------------------------------------------------------
// Multi-right-hand-side triangular solves with the base factor, one
// cooperative launch each.  With Linv_p the inverse unit-lower diagonal
// blocks of the factor and the off-diagonal blocks premultiplied once per
// call (k_cand_gmat):
//   FWD (L y = w, then z = invD o y):
//     Y_p = Linv_p W_p - sum_{q<p} G_pq Y_q,           G_pq = Linv_p L_pq
//   BWD (L^H x = z - U(:,K) x_K):
//     X_p = Linv_p^H (Z_p - U(p,K) x_K) - sum_{q>p} G_pq X_q,  G_pq = Linv_p^H U_pq
// (L_pq(m, k) = conj(U(q0+k, p0+m)), U_pq(m, k) = U(p0+m, q0+k)).  The
// diagonal-block product needs no other panel, so it runs before the first
// wait; each dependency's G tile (static) is loaded while the CTA waits for
// that panel's flag, so a step of the panel chain is one flag hand-off, one
// 64 x 16 tile load and one 64 x 64 x 16 product.
// Work item (panel p, column block cb of CAND_NC columns); items are ordered
// so that every item depends only on items with smaller indices, and each
// CTA takes items blockIdx.x, blockIdx.x + gridDim.x, ... in order, so with
// all CTAs co-resident every wait ends.  Each wait is bounded
// (abort_word[1] polls, SOLVE_SPIN_LIMIT by default, or at once after any
// CTA gave up); a CTA that gives
// up records ST_SOLVE_TIMEOUT and publishes nothing.
// ---------------------------------------------------------------------------
constexpr int TS_LDA = 64 + 2;
constexpr int TS_LDB = 64 + 4;
constexpr size_t TS_SMEM = (size_t)(64 * TS_LDA + CAND_NC * TS_LDB) * sizeof(double2);

// G tiles: one CTA per ordered panel pair (p, q), p != q; FWD blocks (p > q)
// and BWD blocks (p < q) share the array, G(p0+m, q0+n) at Gm[(p0+m) + (q0+n) ld].
__global__ void __launch_bounds__(256) k_cand_gmat(const cd* __restrict__ H, int ld, const int* __restrict__ bstart,
                                                   int nb, const cd* __restrict__ linv, cd* __restrict__ Gm)
{
    extern __shared__ double2 gsm[];
    const int p = blockIdx.x, q = blockIdx.y;
    if (p == q || p >= nb || q >= nb) return;
    const bool fwd = p > q;
    const int p0 = bstart[p], bp = bstart[p + 1] - p0;
    const int q0 = bstart[q], bq = bstart[q + 1] - q0;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int wm = (wp >> 2) * 32, wn = (wp & 3) * 16;
    ZAcc<4, 2> acc;
    acc.zero();
    double2* As = gsm;               // [k][m]: Linv_p (FWD) / Linv_p^H before its conjugation (BWD)
    double2* Bs = gsm + GK * G_LDA;  // [n][k]: L_pq (FWD) / U_pq (BWD)
    for (int k0 = 0; k0 < LDL_NB; k0 += GK) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int e = tid + 256 * u;
            // A(m, k): FWD linv[(p0+m) 64 + k] (k contiguous); BWD conj(linv[(p0+k) 64 + m]) (m contiguous)
            const int m = fwd ? (e >> 5) : (e & 63), k = fwd ? (e & 31) : (e >> 6);
            const bool in = (m < bp) && (k0 + k < bp);
            const cd* src = fwd ? linv + (size_t)(p0 + m) * LDL_NB + k0 + k : linv + (size_t)(p0 + k0 + k) * LDL_NB + m;
            double2 v = make_double2(0.0, 0.0);
            if (in) v = __ldg(reinterpret_cast<const double2*>(src));
            As[k * G_LDA + m] = v;
            // B(k, n): FWD conj(H[(q0+n) + (p0+k) ld]) (n contiguous); BWD H[(p0+k) + (q0+n) ld] (k contiguous)
            const int n2 = fwd ? (e & 63) : (e >> 5), k2 = fwd ? (e >> 6) : (e & 31);
            const bool in2 = (n2 < bq) && (k0 + k2 < bp);
            double2 w = make_double2(0.0, 0.0);
            if (in2) {
                const cd* s2 = fwd ? H + (size_t)(q0 + n2) + (size_t)(p0 + k0 + k2) * ld
                                   : H + (size_t)(p0 + k0 + k2) + (size_t)(q0 + n2) * ld;
                w = __ldg(reinterpret_cast<const double2*>(s2));
                if (fwd) w.y = -w.y;
            }
            Bs[n2 * G_LDB + k2] = w;
        }
        __syncthreads();
        if (fwd) {
#pragma unroll
            for (int kk = 0; kk < GK; kk += 4) zmma_k4<4, 2, G_LDA, G_LDB, false>(acc, As, Bs, wm, wn, kk, lane);
        } else {
#pragma unroll
            for (int kk = 0; kk < GK; kk += 4) zmma_k4<4, 2, G_LDA, G_LDB, true>(acc, As, Bs, wm, wn, kk, lane);
        }
        __syncthreads();
    }
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 4; mt++)
#pragma unroll
        for (int nt = 0; nt < 2; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int m = wm + mt * 8 + g, n = wn + nt * 8 + 2 * t + e;
                if (m < bp && n < bq)
                    *reinterpret_cast<double2*>(Gm + (size_t)(p0 + m) + (size_t)(q0 + n) * ld) =
                        make_double2(acc.r[mt][nt][e], acc.i[mt][nt][e]);
            }
}

template <bool FWD>
__global__ void __launch_bounds__(256) k_cand_solve(const cd* __restrict__ Gm, int ld, const int* __restrict__ bstart,
                                                    int nb, const cd* __restrict__ linv, const cd* __restrict__ invD,
                                                    const cd* __restrict__ Win, cd* __restrict__ Yout,
                                                    cd* __restrict__ Zout, const cd* __restrict__ lcol,
                                                    const cd* __restrict__ xK, int ldv, int ncb,
                                                    const int* __restrict__ cmap, unsigned* __restrict__ flags,
                                                    int* __restrict__ status, int* __restrict__ abort_word)
{
    extern __shared__ double2 tsm[];
    double2* As = tsm;                // [k][m]
    double2* Bs = tsm + 64 * TS_LDA;  // [n][k]
    __shared__ int go;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int wm = (wp >> 1) * 16, wn = (wp & 1) * 8;  // 4 x 2 warps of 16 x 8
    const int g = lane >> 2, t = lane & 3;
    const int nitems = nb * ncb;
    bool ok = true;
    // G tile of dependency q into As (m contiguous in memory)
    auto load_g = [&](int p0, int bp, int q) {
        const int q0 = bstart[q], bq = bstart[q + 1] - q0;
#pragma unroll 4
        for (int u = 0; u < 16; u++) {
            const int e = tid + 256 * u;
            const int m = e & 63, k = e >> 6;
            const bool in = (m < bp) && (k < bq);
            cp_async16(As + k * TS_LDA + m, in ? Gm + (size_t)(p0 + m) + (size_t)(q0 + k) * ld : Gm, in ? 16 : 0);
        }
        cp_async_commit();
    };
    for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
        const int pi = item / ncb, cb = item % ncb;
        const int p = FWD ? pi : nb - 1 - pi;
        const int p0 = bstart[p], bp = bstart[p + 1] - p0;
        const int col0 = cb * CAND_NC;
        // (1) diagonal block: Linv_p rhs (FWD) / Linv_p^H (rhs - U(p,K) x_K) (BWD)
#pragma unroll 4
        for (int u = 0; u < 16; u++) {
            const int e = tid + 256 * u;
            const int m = FWD ? (e >> 6) : (e & 63);
            const int k = FWD ? (e & 63) : (e >> 6);
            const bool in = (m < bp) && (k < bp);
            const cd* src = FWD ? linv + (size_t)(p0 + m) * LDL_NB + k : linv + (size_t)(p0 + k) * LDL_NB + m;
            cp_async16(As + k * TS_LDA + m, in ? src : linv, in ? 16 : 0);
        }
        cp_async_commit();
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = tid + 256 * u;
            const int m = e & 63, n = e >> 6;
            cd v = mk(0.0, 0.0);
            if (m < bp) {
                const int jp = cmap ? cmap[col0 + n] : col0 + n;
                const size_t o = (size_t)(p0 + m) + (size_t)jp * ldv;
                v = ldcd(Win + o);
                if (!FWD) v = cfms(ldcd(lcol + o), ldcd(xK + jp), v);
            }
            Bs[n * TS_LDB + m] = make_double2(v.x, v.y);
        }
        cp_async_wait<0>();
        __syncthreads();
        ZAcc<2, 1> acc;
        acc.zero();
#pragma unroll
        for (int kk = 0; kk < 64; kk += 4) zmma_k4<2, 1, TS_LDA, TS_LDB, !FWD>(acc, As, Bs, wm, wn, kk, lane);
        __syncthreads();
        // (2) the panels this one depends on
        ZAcc<2, 1> dep;
        dep.zero();
        const int ndep = FWD ? p : nb - 1 - p;
        if (ndep > 0) load_g(p0, bp, FWD ? 0 : nb - 1);
        for (int d = 0; d < ndep; d++) {
            const int q = FWD ? d : nb - 1 - d;
            if (tid == 0) {
                int gg = 1;
                int spins = 0;
                const int limit = ((volatile int*)abort_word)[1];
                while (ld_acquire_u32(flags + q * ncb + cb) != 1u) {
                    if (++spins > limit || *((volatile int*)abort_word) != 0) {
                        gg = 0;
                        break;
                    }
                    __nanosleep(64);
                }
                if (!gg) {
                    atomicExch(status + ST_SOLVE_TIMEOUT, 1);
                    atomicExch(abort_word, 1);
                }
                go = gg;
            }
            __syncthreads();
            if (!go) {
                ok = false;
                break;
            }
            const int q0 = bstart[q], bq = bstart[q + 1] - q0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int e = tid + 256 * u;
                const int k = e & 63, n = e >> 6;
                const bool in = k < bq;
                const int jp = cmap ? cmap[col0 + n] : col0 + n;
                cp_async16(Bs + n * TS_LDB + k, in ? Yout + (size_t)(q0 + k) + (size_t)jp * ldv : Yout, in ? 16 : 0);
            }
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < 64; kk += 4) zmma_k4<2, 1, TS_LDA, TS_LDB, false>(dep, As, Bs, wm, wn, kk, lane);
            __syncthreads();
            if (d + 1 < ndep) load_g(p0, bp, FWD ? d + 1 : nb - 2 - d);  // overlaps the next wait
        }
        if (!ok) {
            cp_async_wait<0>();
            break;
        }
        // (3) publish this panel
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int m = wm + mt * 8 + g, n = wn + 2 * t + e;
                if (m < bp) {
                    const int jp = cmap ? cmap[col0 + n] : col0 + n;
                    const size_t o = (size_t)(p0 + m) + (size_t)jp * ldv;
                    const cd y = mk(acc.r[mt][0][e] - dep.r[mt][0][e], acc.i[mt][0][e] - dep.i[mt][0][e]);
                    *reinterpret_cast<double2*>(Yout + o) = make_double2(y.x, y.y);
                    if (FWD) {
                        const cd z = cmul(y, ldcd(invD + p0 + m));
                        *reinterpret_cast<double2*>(Zout + o) = make_double2(z.x, z.y);
                    }
                }
            }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release_u32(flags + p * ncb + cb, 1u);
    }
}

// Split-K partial sums of k_zgemm are added in a fixed order:
// C(:, slot j) = sum_z P[z](:, j) (+ E1 o e2), through the column map.
__global__ void __launch_bounds__(256) k_zsum(const cd* __restrict__ P, int nz, size_t pstride, int M, int ncols,
                                              int ldc, cd* __restrict__ C, const cd* __restrict__ E1,
                                              const cd* __restrict__ e2, const int* __restrict__ cmap)
{
    const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;
    if (idx >= (long long)M * ncols) return;
    const int i = (int)(idx % M), j = (int)(idx / M);
    cd v = mk(0.0, 0.0);
    for (int z = 0; z < nz; z++) v = v + ldcd(P + z * pstride + (size_t)i + (size_t)j * ldc);
    const int jp = cmap ? cmap[j] : j;
    const size_t o = (size_t)i + (size_t)jp * ldc;
    if (E1) v = cfma(ldcd(E1 + o), ldcd(e2 + jp), v);
    *reinterpret_cast<double2*>(C + o) = make_double2(v.x, v.y);
}

// ---------------------------------------------------------------------------
// Per-candidate kernels: one CTA of 256 threads per candidate j, fixed-order
// block reductions (results are reproducible run to run).
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum256(double (&v)[NV], double* sh)
{
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++)
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[wp * NV + k] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; q++) s += sh[q * NV + k];
        v[k] = s;
    }
}

__device__ __forceinline__ double block_max256(double v, double* sh)
{
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) sh[wp] = v;
    __syncthreads();
    double m = sh[0];
#pragma unroll
    for (int q = 1; q < 8; q++) m = fmax(m, sh[q]);
    return m;
}

// Per-column state, stride `bcap` in the kernels (CandWork::ccap):
// CandWork::st (ints): [0] active  [1] iterations  [2] ErrorCode, then the active count
// CandWork::nd (doubles): [0] NormOfDiff  [1] NormOfDiffPrev  [2] t1  [3] t2  [4] E
// border entries (CandWork::brd, complex): [0] v_K  [1] w_K  [2] invD_K  [3] x_K
enum { ST_ACTIVE = 0, ST_ITERS = 1, ST_ERR = 2 };
enum { ND_ND = 0, ND_PREV = 1, ND_T1 = 2, ND_T2 = 3, ND_E = 4 };
enum { BR_V = 0, BR_W = 1, BR_INVD = 2, BR_X = 3 };

// Bordered LDLHF step for row K (src/linalg.f90:359-383):
// x = M(K,K) - sum_q conj(a_q) U(q,K);  d_K = conj(x);  invD_K = 1/d_K,
// with the pivot's rounding-level imaginary part dropped (cplx = 0, as in
// k_ldl_diag<false>) or kept (cplx = 1, as the reference keeps it).
__global__ void __launch_bounds__(256) k_cand_border(const cd* __restrict__ Acol, const cd* __restrict__ Lcol,
                                                     const double* __restrict__ mu, int nbase, int ldv, int bcap,
                                                     cd* __restrict__ brd, int* __restrict__ st, int cplx)
{
    __shared__ double sh[8 * 2];
    const int j = blockIdx.x;
    const cd* a = Acol + (size_t)j * ldv;
    const cd* l = Lcol + (size_t)j * ldv;
    double v[2] = {0.0, 0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd s = cmul(conj(ldcd(a + q)), ldcd(l + q));
        v[0] += s.x;
        v[1] += s.y;
    }
    block_sum256<2>(v, sh);
    if (threadIdx.x == 0) {
        const double xr = mu[j] - v[0];
        const double xi = cplx ? v[1] : 0.0;  // d_K = conj(x): Im d_K = +Im(sum)
        if (xr == 0.0 && xi == 0.0) {
            st[ST_ERR * bcap + j] = 1;
            brd[BR_INVD * bcap + j] = mk(0.0, 0.0);
        } else if (!cplx) {
            brd[BR_INVD * bcap + j] = mk(1.0 / xr, 0.0);
        } else {
            const double m = 1.0 / fma(xr, xr, xi * xi);
            brd[BR_INVD * bcap + j] = mk(xr * m, -xi * m);
        }
    }
}

// v = Glob_LastEigvector(1:K) for every candidate; state reset.
__global__ void __launch_bounds__(256) k_cand_init(const cd* __restrict__ x0, int nbase, int count, int ldv, int bcap,
                                                   cd* __restrict__ V, cd* __restrict__ brd, double* __restrict__ nd,
                                                   int* __restrict__ st)
{
    const int j = blockIdx.y;
    const bool real_col = j < count;
    for (int q = blockIdx.x * 256 + threadIdx.x; q < nbase; q += gridDim.x * 256)
        V[(size_t)q + (size_t)j * ldv] = real_col ? x0[q] : mk(0.0, 0.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        brd[BR_V * bcap + j] = real_col ? x0[nbase] : mk(0.0, 0.0);
        if (real_col) {
            st[ST_ACTIVE * bcap + j] = (st[ST_ERR * bcap + j] == 0) ? 1 : 0;
            st[ST_ITERS * bcap + j] = 0;
            nd[ND_ND * bcap + j] = 0.0;
            nd[ND_PREV * bcap + j] = DBL_MAX;
        }
    }
}

// w_K = sum_q conj(S(q,K)) v_q + v_K  (row K of MHMV's B^H v)
__global__ void __launch_bounds__(256) k_cand_wk(const cd* __restrict__ Scol, const cd* __restrict__ V, int nbase,
                                                 int ldv, int bcap, cd* __restrict__ brd, const int* __restrict__ cmap,
                                                 int count)
{
    __shared__ double sh[8 * 2];
    const int j = cmap[blockIdx.x];
    if (j >= count) return;
    const cd* s = Scol + (size_t)j * ldv;
    const cd* v = V + (size_t)j * ldv;
    double a[2] = {0.0, 0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd p = cmul(conj(ldcd(s + q)), ldcd(v + q));
        a[0] += p.x;
        a[1] += p.y;
    }
    block_sum256<2>(a, sh);
    if (threadIdx.x == 0) brd[BR_W * bcap + j] = mk(a[0], a[1]) + brd[BR_V * bcap + j];
}

// y_K = w_K - sum_q conj(U(q,K)) y_q;  x_K = z_K = invD_K y_K
__global__ void __launch_bounds__(256) k_cand_mid(const cd* __restrict__ Lcol, const cd* __restrict__ Y, int nbase,
                                                  int ldv, int bcap, cd* __restrict__ brd, const int* __restrict__ cmap,
                                                  int count)
{
    __shared__ double sh[8 * 2];
    const int j = cmap[blockIdx.x];
    if (j >= count) return;
    const cd* l = Lcol + (size_t)j * ldv;
    const cd* y = Y + (size_t)j * ldv;
    double a[2] = {0.0, 0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd p = cmul(conj(ldcd(l + q)), ldcd(y + q));
        a[0] += p.x;
        a[1] += p.y;
    }
    block_sum256<2>(a, sh);
    if (threadIdx.x == 0) {
        const cd yk = brd[BR_W * bcap + j] - mk(a[0], a[1]);
        brd[BR_X * bcap + j] = cmul(yk, brd[BR_INVD * bcap + j]);
    }
}

// GHEPIIS iteration tail for an active candidate (src/linalg.f90:1894-1908):
// t = CMaxAbsReOrIm(x), x = x / t, tc = x^H v / v^H v,
// NormOfDiff = sqrt(2K) ||x - tc v||, convergence test; v <- x.
__global__ void __launch_bounds__(256) k_cand_norm(const cd* __restrict__ X, cd* __restrict__ V, int nbase, int ldv,
                                                   int bcap, cd* __restrict__ brd, double* __restrict__ nd,
                                                   int* __restrict__ st, double sqrtn, double tol,
                                                   const int* __restrict__ cmap, int count)
{
    __shared__ double sh[8 * 3];
    const int j = cmap[blockIdx.x];
    if (j >= count || st[ST_ACTIVE * bcap + j] == 0) return;
    const cd* x = X + (size_t)j * ldv;
    cd* v = V + (size_t)j * ldv;
    const cd xk = brd[BR_X * bcap + j], vk = brd[BR_V * bcap + j];
    double m = 0.0;
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd a = ldcd(x + q);
        m = fmax(m, fmax(fabs(a.x), fabs(a.y)));
    }
    if (threadIdx.x == 0) m = fmax(m, fmax(fabs(xk.x), fabs(xk.y)));
    m = block_max256(m, sh);
    const double s = 1.0 / m;
    // tc = (x^H v) / (v^H v)
    double a3[3] = {0.0, 0.0, 0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd a = s * ldcd(x + q), b = ldcd(v + q);
        const cd p = cmul(conj(a), b);
        a3[0] += p.x;
        a3[1] += p.y;
        a3[2] += cnorm2(b);
    }
    if (threadIdx.x == 0) {
        const cd p = cmul(conj(s * xk), vk);
        a3[0] += p.x;
        a3[1] += p.y;
        a3[2] += cnorm2(vk);
    }
    block_sum256<3>(a3, sh);
    const cd tc = mk(a3[0] / a3[2], a3[1] / a3[2]);
    // ||x - tc v||^2, then v <- x
    double d[1] = {0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd a = s * ldcd(x + q), b = ldcd(v + q);
        d[0] += cnorm2(a - cmul(tc, b));
        v[q] = a;
    }
    if (threadIdx.x == 0) d[0] += cnorm2(s * xk - cmul(tc, vk));
    block_sum256<1>(d, sh);
    if (threadIdx.x == 0) {
        const double ndv = sqrtn * sqrt(d[0]);
        bool conv;
        if (tol > 0.0) {
            conv = ndv <= tol;
        } else {
            conv = (ndv > nd[ND_PREV * bcap + j]) && (ndv <= fabs(tol));
            nd[ND_PREV * bcap + j] = ndv;
        }
        nd[ND_ND * bcap + j] = ndv;
        brd[BR_V * bcap + j] = s * xk;
        st[ST_ITERS * bcap + j] += 1;
        if (conv) st[ST_ACTIVE * bcap + j] = 0;
    }
}

// Column map of the next iteration: the slots of the still-active
// candidates first, in their current order (the order does not change any
// result: columns never mix), then spare columns bcap.. up to the next
// multiple of CAND_PAD (bcap here is the column stride, CAND_PAD beyond
// the candidate capacity); the active count goes to st[3 bcap].  init:
// start from candidates 0..count-1.
__global__ void k_cand_compact(int* __restrict__ cmap, int* __restrict__ st, int bcap, int count, int nslots,
                               int init)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int na = 0;
    const int n = init ? count : nslots;
    for (int s = 0; s < n; s++) {
        const int j = init ? s : cmap[s];
        if (j < count && st[ST_ACTIVE * bcap + j]) cmap[na++] = j;
    }
    const int pad = ((na + CAND_PAD - 1) / CAND_PAD) * CAND_PAD;
    for (int s = na; s < pad; s++) cmap[s] = bcap - CAND_PAD + (s - na);  // spare physical columns
    st[3 * bcap] = na;
}

// Rayleigh quotient (src/linalg.f90:1913-1917) of the final iterate:
// t1 = v^H S v, t2 = v^H M v with P = S0 V, Q = M0 V; E = t2 / t1 + lambda~.
__global__ void __launch_bounds__(256) k_cand_rayleigh(const cd* __restrict__ P, const cd* __restrict__ Q,
                                                       const cd* __restrict__ V, const cd* __restrict__ Scol,
                                                       const cd* __restrict__ Mcol, const double* __restrict__ mu,
                                                       int nbase, int ldv, int bcap, const cd* __restrict__ brd,
                                                       double* __restrict__ nd, const int* __restrict__ st,
                                                       double lam)
{
    __shared__ double sh[8 * 6];
    const int j = blockIdx.x;
    const size_t o = (size_t)j * ldv;
    double a[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = threadIdx.x; q < nbase; q += 256) {
        const cd v = ldcd(V + o + q);
        const cd cv = conj(v);
        a[0] += cmul(cv, ldcd(P + o + q)).x;
        a[1] += cmul(cv, ldcd(Q + o + q)).x;
        const cd s = cmul(conj(ldcd(Scol + o + q)), v);
        const cd m = cmul(conj(ldcd(Mcol + o + q)), v);
        a[2] += s.x;
        a[3] += s.y;
        a[4] += m.x;
        a[5] += m.y;
    }
    block_sum256<6>(a, sh);
    if (threadIdx.x == 0) {
        const cd vk = brd[BR_V * bcap + j];
        const double t1 = a[0] + 2.0 * cmul(conj(vk), mk(a[2], a[3])).x + cnorm2(vk);
        const double t2 = a[1] + 2.0 * cmul(conj(vk), mk(a[4], a[5])).x + mu[j] * cnorm2(vk);
        nd[ND_T1 * bcap + j] = t1;
        nd[ND_T2 * bcap + j] = t2;
        nd[ND_E * bcap + j] = (st[ST_ERR * bcap + j] == 1) ? __longlong_as_double(0x7ff8000000000000LL) : t2 / t1 + lam;
    }
}

template <typename T>
int dalloc_n(T** p, size_t count)
{
    *p = nullptr;
    if (cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return -3;
    }
    return 0;
}

void drop_graphs(CandWork& cw)
{
    for (auto& g : cw.graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    cw.graphs.clear();
}

int ensure_work(Ctx& c, int count)
{
    CandWork& cw = c.cand;
    const int need = ((count + CAND_PAD - 1) / CAND_PAD) * CAND_PAD;
    if (need <= cw.bcap) return 0;
    cand_free(cw);
    const int bcap = std::max(need, CAND_PAD);
    const int ccap = bcap + CAND_PAD;
    const int ldv = ((c.ld + 63) / 64) * 64;
    const size_t col = (size_t)ldv * ccap;
    cw.ldv = ldv;
    const int maxpanels = c.ld + 2;  // panel count never exceeds the row count
    cw.nflags = maxpanels * (ccap / CAND_NC);
    int r = 0;
    r |= dalloc_n(&cw.par, (size_t)c.npt * bcap);
    r |= dalloc_n(&cw.bra, (size_t)bcap * c.np);
    r |= dalloc_n(&cw.ket, (size_t)bcap * c.T * c.np);
    r |= dalloc_n(&cw.det, (size_t)bcap);
    r |= dalloc_n(&cw.dS, (size_t)bcap);
    r |= dalloc_n(&cw.mu, (size_t)bcap);
    r |= dalloc_n(&cw.Mcol, col);
    r |= dalloc_n(&cw.Scol, col);
    r |= dalloc_n(&cw.Acol, col);
    r |= dalloc_n(&cw.Lcol, col);
    r |= dalloc_n(&cw.V, col);
    r |= dalloc_n(&cw.W, col);
    r |= dalloc_n(&cw.Y, col);
    r |= dalloc_n(&cw.Z, col);
    r |= dalloc_n(&cw.X, col);
    r |= dalloc_n(&cw.X2, col);
    r |= dalloc_n(&cw.brd, (size_t)4 * ccap);
    r |= dalloc_n(&cw.nd, (size_t)5 * ccap);
    r |= dalloc_n(&cw.st, (size_t)3 * ccap + 1);
    r |= dalloc_n(&cw.cmap, (size_t)ccap);
    r |= dalloc_n(&cw.Gm, (size_t)c.ld * c.ld);
    r |= dalloc_n(&cw.Pk, (size_t)CAND_KSPLIT * ldv * 2 * CAND_PAD);
    r |= dalloc_n(&cw.flags, (size_t)cw.nflags);
    r |= dalloc_n(&cw.bstart, (size_t)maxpanels + 1);
    r |= dalloc_n(&cw.abort_word, 2);  // abort word, wait poll limit
    cw.gpart_n = (size_t)bcap * (c.ld / 128 + 2) * (2 * c.np + 1);
    r |= dalloc_n(&cw.gpart, cw.gpart_n);
    r |= dalloc_n(&cw.grad, (size_t)c.npt * bcap);
    if (!r) {
        if (cudaMallocHost((void**)&cw.st_h, sizeof(int) * (3 * (size_t)ccap + 1)) != cudaSuccess ||
            cudaMallocHost((void**)&cw.nd_h, sizeof(double) * 5 * (size_t)ccap) != cudaSuccess ||
            cudaMallocHost((void**)&cw.bstart_h, sizeof(int) * ((size_t)maxpanels + 1)) != cudaSuccess) {
            cudaGetLastError();
            r = -3;
        }
    }
    if (r) {
        cand_free(cw);
        return -3;
    }
    cw.bcap = bcap;
    cw.ccap = ccap;
    // zero the column blocks once: padded and spare columns stay finite
    void* zc[] = {cw.Mcol, cw.Scol, cw.Acol, cw.Lcol, cw.V, cw.W, cw.Y, cw.Z, cw.X, cw.X2};
    for (void* p : zc)
        if (cudaMemsetAsync(p, 0, col * sizeof(cd), c.stream) != cudaSuccess) return -2;
    if (cudaMemsetAsync(cw.brd, 0, 4 * (size_t)ccap * sizeof(cd), c.stream) != cudaSuccess) return -2;
    if (cudaMemcpyAsync(cw.abort_word + 1, &c.wait_limit, sizeof(int), cudaMemcpyHostToDevice, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return -2;
    return 0;
}

int solve_grid(Ctx& c)
{
    CandWork& cw = c.cand;
    if (cw.solve_grid) return cw.solve_grid;
    int coop = 0, nsm = 0, a = 0, b = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
    cudaFuncSetAttribute(k_cand_solve<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS_SMEM);
    cudaFuncSetAttribute(k_cand_solve<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TS_SMEM);
    cudaFuncSetAttribute(k_zgemm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G_SMEM);
    cudaFuncSetAttribute(k_zgemm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G_SMEM);
    cudaFuncSetAttribute(k_cand_gmat, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(G_STAGE * sizeof(double2)));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_cand_solve<true>, 256, TS_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cand_solve<false>, 256, TS_SMEM);
    cudaGetLastError();
    cw.solve_grid = (coop && std::min(a, b) > 0) ? nsm * std::min(a, b) : -1;
    return cw.solve_grid;
}

// One cooperative triangular solve over ncols columns (through cmap when
// it is not null).
int launch_solve(Ctx& c, bool fwd, int nb, int ncols, const cd* Win, cd* Yout, cd* Zout, const int* cmap)
{
    CandWork& cw = c.cand;
    const int ncb = ncols / CAND_NC;
    const int items = nb * ncb;
    if (items <= 0) return 0;
    if (cudaMemsetAsync(cw.flags, 0, sizeof(unsigned) * (size_t)items, c.stream) != cudaSuccess) return -2;
    if (cudaMemsetAsync(cw.abort_word, 0, sizeof(int), c.stream) != cudaSuccess) return -2;
    const int grid = std::min(items, solve_grid(c));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = TS_SMEM;
    cfg.stream = c.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cd* xk = cw.brd + BR_X * cw.ccap;
    cudaError_t e;
    if (fwd)
        e = cudaLaunchKernelEx(&cfg, k_cand_solve<true>, (const cd*)cw.Gm, c.ld, (const int*)cw.bstart, nb,
                               (const cd*)c.linv, (const cd*)c.invD, Win, Yout, Zout, (const cd*)cw.Lcol, xk, cw.ldv,
                               ncb, cmap, cw.flags, c.status, cw.abort_word);
    else
        e = cudaLaunchKernelEx(&cfg, k_cand_solve<false>, (const cd*)cw.Gm, c.ld, (const int*)cw.bstart, nb,
                               (const cd*)c.linv, (const cd*)c.invD, Win, Yout, Zout, (const cd*)cw.Lcol, xk, cw.ldv,
                               ncb, cmap, cw.flags, c.status, cw.abort_word);
    c.launches++;
    return e == cudaSuccess ? 0 : -2;
}

int launch_gemm(Ctx& c, int amode, const cd* A, int M, int ncols, const cd* B, cd* C, const cd* E1, const cd* e2,
                const int* cmap)
{
    CandWork& cw = c.cand;
    if (M <= 0) return 0;
    const int mt = (M + GM - 1) / GM, nt = ncols / GN;
    // few output tiles (the late iterations run on one or two 64-column
    // slots): split the inner dimension so that the GPU stays busy
    int nz = 1;
    if (ncols <= 2 * CAND_PAD) nz = std::max(1, std::min(CAND_KSPLIT, 148 / std::max(1, mt * nt)));
    dim3 g(mt, nt, nz);
    const size_t pstride = (size_t)cw.ldv * 2 * CAND_PAD;
    if (amode == 0)
        k_zgemm<0><<<g, 256, G_SMEM, c.stream>>>(A, c.ld, M, M, B, cw.ldv, C, cw.ldv, E1, e2, cmap, cw.Pk, pstride);
    else
        k_zgemm<1><<<g, 256, G_SMEM, c.stream>>>(A, c.ld, M, M, B, cw.ldv, C, cw.ldv, E1, e2, cmap, cw.Pk, pstride);
    c.launches++;
    if (nz > 1) {
        const long long cnt = (long long)M * ncols;
        k_zsum<<<(unsigned)((cnt + 255) / 256), 256, 0, c.stream>>>(cw.Pk, nz, pstride, M, ncols, cw.ldv, C, E1, e2,
                                                                    cmap);
        c.launches++;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// One inverse iteration for the active candidates (see the file header):
// ncols slots of the column map, a multiple of CAND_PAD.
int enqueue_iteration(Ctx& c, int nbase, int count, int ncols, int nb, double tol)
{
    CandWork& cw = c.cand;
    const int cc = cw.ccap;
    int r;
    if ((r = launch_gemm(c, 0, c.S, nbase, ncols, cw.V, cw.W, cw.Scol, cw.brd + BR_V * cc, cw.cmap))) return r;
    k_cand_wk<<<ncols, 256, 0, c.stream>>>(cw.Scol, cw.V, nbase, cw.ldv, cc, cw.brd, cw.cmap, count);
    c.launches++;
    if ((r = launch_solve(c, true, nb, ncols, cw.W, cw.Y, cw.Z, cw.cmap))) return r;
    k_cand_mid<<<ncols, 256, 0, c.stream>>>(cw.Lcol, cw.Y, nbase, cw.ldv, cc, cw.brd, cw.cmap, count);
    c.launches++;
    if ((r = launch_solve(c, false, nb, ncols, cw.Z, cw.X, nullptr, cw.cmap))) return r;
    k_cand_norm<<<ncols, 256, 0, c.stream>>>(cw.X, cw.V, nbase, cw.ldv, cc, cw.brd, cw.nd, cw.st,
                                             sqrt(2.0 * (nbase + 1)), tol, cw.cmap, count);
    k_cand_compact<<<1, 32, 0, c.stream>>>(cw.cmap, cw.st, cc, count, ncols, 0);
    c.launches += 2;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// Replay (capturing on first use) the iteration graph for this shape.
int run_iteration(Ctx& c, int nbase, int count, int ncols, int nb, double tol)
{
    CandWork& cw = c.cand;
    long long tl;
    memcpy(&tl, &tol, sizeof(tl));
    std::vector<int> key = {nbase, count, ncols, nb, (int)(tl & 0xffffffff), (int)(tl >> 32)};
    CandWork::IterGraph* g = nullptr;
    for (auto& e : cw.graphs)
        if (e.key == key) g = &e;
    if (!g) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        long long nl = 0;
        if (ok) {
            const long long l0 = c.launches;
            const int r = enqueue_iteration(c, nbase, count, ncols, nb, tol);
            nl = c.launches - l0;
            c.launches = l0;
            ok = cudaStreamEndCapture(c.stream, &graph) == cudaSuccess && graph && r == 0 &&
                 cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        }
        if (graph) cudaGraphDestroy(graph);
        if (!ok) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            return enqueue_iteration(c, nbase, count, ncols, nb, tol);  // capture unavailable: launch directly
        }
        if (cw.graphs.size() >= 16) {
            cudaGraphExecDestroy(cw.graphs.front().exec);
            cw.graphs.erase(cw.graphs.begin());
        }
        cw.graphs.push_back({key, exec, nl});
        g = &cw.graphs.back();
    }
    if (cudaGraphLaunch(g->exec, c.stream) != cudaSuccess) return -2;
    c.launches += g->launches;
    return 0;
}

// Pick the k_cand_row tile shape by timing every shape once on this
// workload (first call per system shape); the outputs of all shapes are
// identical, so the last run's stand.
int tune_rows(Ctx& c, int nbase, int count, double approx_e)
{
    CandWork& cw = c.cand;
    if (cw.row_variant >= 0 && cw.tuned_n == c.n && cw.tuned_T == c.T) return 0;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -2;
    float best = 1e30f;
    int bv = 0;
    for (int v = 0; v < CAND_ROW_SHAPES; v++) {
        cudaEventRecord(e0, c.stream);
        const int r = launch_cand_rows(c, cw, nbase, count, approx_e, v);
        cudaEventRecord(e1, c.stream);
        if (r) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return r;
        }
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            bv = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cw.row_variant = bv;
    cw.tuned_n = c.n;
    cw.tuned_T = c.T;
    return 0;
}

}  // namespace

void cand_free(CandWork& cw)
{
    drop_graphs(cw);
    void* ptrs[] = {cw.par, cw.bra, cw.ket, cw.det, cw.dS, cw.mu, cw.Mcol, cw.Scol, cw.Acol, cw.Lcol, cw.V, cw.W,
                    cw.Y, cw.Z, cw.X, cw.X2, cw.brd, cw.nd, cw.st, cw.cmap, cw.Gm, cw.Pk, cw.flags, cw.bstart,
                    cw.abort_word, cw.gpart, cw.grad};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (cw.st_h) cudaFreeHost(cw.st_h);
    if (cw.nd_h) cudaFreeHost(cw.nd_h);
    if (cw.bstart_h) cudaFreeHost(cw.bstart_h);
    const int rv = cw.row_variant, tn = cw.tuned_n, tT = cw.tuned_T, sg = cw.solve_grid;
    cw = CandWork();
    cw.row_variant = rv;
    cw.tuned_n = tn;
    cw.tuned_T = tT;
    cw.solve_grid = sg;
}

// See ecg_eval_candidates / ecg_eval_candidates_grad in ecg_abi.h.  Returns
// 0 or a negative status; per-candidate ErrorCodes go to errcodes.  With
// grad (host, npt x count), every candidate's energy gradient with respect
// to its own parameters too (requires nbase >= 1).
int eval_candidates(Ctx& c, int nbase, int count, const double* cand_host, double approx_e, double tol,
                    int max_iter, double* energies, int* errcodes, int* num_iter, double* rel_acc, double* grad)
{
    if (c.method != 'I') return ECG_EARG;
    if (nbase < 0 || count < 1 || nbase + 1 > c.ld || max_iter < 1 || !cand_host || !energies) return ECG_EARG;
    if (grad && nbase < 1) return ECG_EARG;
    if (ensure_work(c, count)) return ECG_ENOMEM;
    CandWork& cw = c.cand;
    const int cc = cw.ccap;
    const int ncols = ((count + CAND_PAD - 1) / CAND_PAD) * CAND_PAD;
    auto CKc = [](cudaError_t e) { return e == cudaSuccess ? 0 : (cudaGetLastError(), ECG_ECUDA); };
    int r;
    if ((r = CKc(cudaMemcpyAsync(cw.par, cand_host, sizeof(double) * c.npt * count, cudaMemcpyHostToDevice,
                                 c.stream))))
        return r;
    c.bytes_h2d += (long long)sizeof(double) * c.npt * count;
    if ((r = CKc(cudaMemsetAsync(c.status, 0, ST_COUNT * sizeof(int), c.stream)))) return r;
    if ((r = CKc(cudaMemsetAsync(cw.st, 0, sizeof(int) * (3 * (size_t)cc + 1), c.stream)))) return r;
    // the base factor must cover rows 1..nbase
    if (nbase > 0 && c.fact_n < nbase) {
        if (ldlh_factor(c, c.fact_n, nbase)) return ECG_ECUDA;
        if ((r = CKc(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost,
                                     c.stream))))
            return r;
        if ((r = CKc(cudaStreamSynchronize(c.stream)))) return r;
        if (c.status_h[ST_SOLVE_TIMEOUT]) {
            c.fact_n = 0;
            c.blk_start.clear();
            return ECG_ECUDA;
        }
        if (c.status_h[ST_ZERO_PIVOT] != 0) {
            c.fact_n = 0;
            c.blk_start.clear();
            return ECG_ESINGULAR;
        }
    }
    if (nbase > 0 && launch_prep(c, nbase)) return ECG_ECUDA;
    if (nbase > 0) {
        if (tune_rows(c, nbase, count, approx_e)) return ECG_ECUDA;
    }
    if (launch_cand_rows(c, cw, nbase, count, approx_e, cw.row_variant < 0 ? 0 : cw.row_variant)) return ECG_ECUDA;
    if (nbase == 0) {
        // one function: EnergyIA's Nmax == 1 branch, E = Re H(1,1) + lambda~
        if ((r = CKc(cudaMemcpyAsync(cw.nd_h, cw.mu, sizeof(double) * count, cudaMemcpyDeviceToHost, c.stream))))
            return r;
        if ((r = CKc(cudaStreamSynchronize(c.stream)))) return r;
        for (int j = 0; j < count; j++) {
            energies[j] = cw.nd_h[j] + approx_e;
            if (errcodes) errcodes[j] = 0;
            if (num_iter) num_iter[j] = 1;
            if (rel_acc) rel_acc[j] = 0.0;
        }
        return ECG_OK;
    }
    // panels of the base factor, the one holding row nbase truncated
    int nb = 0;
    for (int s : c.blk_start)
        if (s < nbase) cw.bstart_h[nb++] = s;
    cw.bstart_h[nb] = nbase;
    if ((r = CKc(cudaMemcpyAsync(cw.bstart, cw.bstart_h, sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, c.stream))))
        return r;
    if (solve_grid(c) <= 0) return ECG_ECUDA;
    // off-diagonal blocks premultiplied by the inverse diagonal blocks
    if (nb > 1) {
        k_cand_gmat<<<dim3(nb, nb), 256, G_STAGE * sizeof(double2), c.stream>>>(c.F, c.ld, cw.bstart, nb, c.linv,
                                                                                 cw.Gm);
        c.launches++;
    }
    // bordered factor row: Acol = L0^-1 Mcol, Lcol = invD o Acol, then d_K
    if (launch_solve(c, true, nb, ncols, cw.Mcol, cw.Acol, cw.Lcol, nullptr)) return ECG_ECUDA;
    k_cand_border<<<count, 256, 0, c.stream>>>(cw.Acol, cw.Lcol, cw.mu, nbase, cw.ldv, cc, cw.brd, cw.st,
                                               c.pivot_mode);
    {
        dim3 g((nbase + 255) / 256, ncols);
        if (g.x > 16) g.x = 16;
        k_cand_init<<<g, 256, 0, c.stream>>>(c.x, nbase, count, cw.ldv, cc, cw.V, cw.brd, cw.nd, cw.st);
    }
    k_cand_compact<<<1, 32, 0, c.stream>>>(cw.cmap, cw.st, cc, count, 0, 1);
    c.launches += 3;
    int nact = count;
    for (int it = 0; it < max_iter; it++) {
        if ((r = CKc(cudaMemcpyAsync(cw.st_h + 3 * cc, cw.st + 3 * cc, sizeof(int), cudaMemcpyDeviceToHost,
                                     c.stream))))
            return r;
        if ((r = CKc(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost,
                                     c.stream))))
            return r;
        if ((r = CKc(cudaStreamSynchronize(c.stream)))) return r;
        if (c.status_h[ST_SOLVE_TIMEOUT]) return ECG_ECUDA;
        nact = cw.st_h[3 * cc];
        if (nact == 0) break;
        const int nslots = ((nact + CAND_PAD - 1) / CAND_PAD) * CAND_PAD;
        if (run_iteration(c, nbase, count, nslots, nb, tol)) return ECG_ECUDA;
    }
    // Rayleigh quotients of the final iterates (all candidates)
    if (launch_gemm(c, 0, c.S, nbase, ncols, cw.V, cw.X, nullptr, nullptr, nullptr)) return ECG_ECUDA;
    if (launch_gemm(c, 1, c.F, nbase, ncols, cw.V, cw.X2, nullptr, nullptr, nullptr)) return ECG_ECUDA;
    k_cand_rayleigh<<<count, 256, 0, c.stream>>>(cw.X, cw.X2, cw.V, cw.Scol, cw.Mcol, cw.mu, nbase, cw.ldv, cc,
                                                 cw.brd, cw.nd, cw.st, approx_e);
    c.launches++;
    if (grad) {
        // EnergyIB's gradient for each candidate as function nbase+1, by the
        // fused adjoint pass over its row
        if (launch_cand_adjoint(c, cw, nbase, count, cw.brd + (size_t)BR_V * cc, cw.nd + (size_t)ND_T1 * cc,
                                cw.nd + (size_t)ND_E * cc, cw.st + (size_t)ST_ERR * cc, cw.grad))
            return ECG_ECUDA;
        if ((r = CKc(cudaMemcpyAsync(grad, cw.grad, sizeof(double) * c.npt * count, cudaMemcpyDeviceToHost,
                                     c.stream))))
            return r;
        c.bytes_d2h += (long long)sizeof(double) * c.npt * count;
    }
    if ((r = CKc(cudaMemcpyAsync(cw.st_h, cw.st, sizeof(int) * (3 * (size_t)cc + 1), cudaMemcpyDeviceToHost,
                                 c.stream))))
        return r;
    if ((r = CKc(cudaMemcpyAsync(cw.nd_h, cw.nd, sizeof(double) * 5 * (size_t)cc, cudaMemcpyDeviceToHost,
                                 c.stream))))
        return r;
    if ((r = CKc(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c.stream))))
        return r;
    if ((r = CKc(cudaStreamSynchronize(c.stream)))) return r;
    if (c.status_h[ST_SOLVE_TIMEOUT]) return ECG_ECUDA;
    c.bytes_d2h += (long long)(sizeof(int) * 3 + sizeof(double) * 5) * cc;
    for (int j = 0; j < count; j++) {
        int err = cw.st_h[ST_ERR * cc + j];
        if (err == 0 && cw.st_h[ST_ACTIVE * cc + j]) err = 2;  // not converged within MaxIter
        energies[j] = cw.nd_h[ND_E * cc + j];
        if (errcodes) errcodes[j] = err;
        if (num_iter) num_iter[j] = (err == 1) ? 0 : cw.st_h[ST_ITERS * cc + j];
        if (rel_acc) rel_acc[j] = (err == 1) ? DBL_MAX : cw.nd_h[ND_ND * cc + j];
    }
    return ECG_OK;
}

}  // namespace ecg
