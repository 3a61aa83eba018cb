// ldlh.cu -- bordered, blocked LDL^H factorisation of M = H - lambda~ S
// without pivoting, the drop-in for LDLHF (src/linalg.f90:316-455).
//
// Storage contract (identical to the reference): M's lower triangle,
// diagonal included, is left untouched; the strict upper triangle receives
// L^H (unit diagonal implied); invD receives 1/d_i.  Rows 0..m0-1 are an
// existing factorisation (the bordered update of the reference's m > 1).
//
// The factorisation is right-looking over 64-row panels and runs entirely
// in the upper triangle, which holds the working Schur complement W(r,c),
// r < c; the working diagonal lives in dw.  Per panel p = [p0,p1):
//   k_ldl_diag    eliminate the 64 x 64 diagonal block in shared memory,
//                 producing U (= L^H) and invD;
//   k_ldl_trsm    Wun(p, c) by substitution with U_pp, U(p, c) = invD Wun;
//   k_ldl_bulk    W(r, c) -= sum_q conj(U(q,r)) Wun(q,c), r <= c beyond p
//                 (the Hermitian trailing update, a complex GEMM);
//   k_ldl_linv    after the last panel: (U_pp^H)^-1 of every new panel;
//   k_ldl_mn      then the neighbour products Linv_p U(p-1, p)^H and
//                 Linv_p^H U(p, p+1) the cooperative solves apply.
// The off-diagonal recurrence and the pivot d = conj(.) follow
// src/linalg.f90:359-391 term for term; only the summation order differs,
// and the pivots are kept real (the reference's complex arithmetic leaves a
// rounding-level imaginary part in them).
// A whole factorisation (m0 = 0) below LDL_PAIR_MIN rows runs instead as
// the persistent tile kernel of ldlp.cu; ldlh_factor captures either form
// into a CUDA graph.
#include "ecg_internal.h"
#include "zmma.cuh"

namespace ecg {

__device__ __forceinline__ cd ldg2(const cd* p)
{
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}

// Mirror the lower triangle of the new columns into the upper triangle:
// A(r,c) = conj(A(c,r)) for r < c, c in [m0,n); dw[c] = A(c,c).
__global__ void __launch_bounds__(256) k_ldl_mirror(cd* __restrict__ A, int ld, int m0, int n, cd* __restrict__ dw,
                                                     int ct0)
{
    __shared__ double2 t[32][33];
    const int Ct = ct0 + blockIdx.x;
    const int Rt = blockIdx.y;
    if (Rt > Ct) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // source: rows c in tile Ct (lanes), columns r in tile Rt
    for (int q = ty; q < 32; q += 8) {
        const int c = Ct * 32 + tx, r = Rt * 32 + q;
        double2 v = make_double2(0.0, 0.0);
        if (c < n && c >= m0 && r <= c) {
            const cd a = A[(size_t)c + (size_t)r * ld];
            v = make_double2(a.x, -a.y);
            if (r == c) dw[c] = a;
        }
        t[q][tx] = v;
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        const int r = Rt * 32 + tx, c = Ct * 32 + q;
        if (c < n && c >= m0 && r < c) {
            const double2 v = t[tx][q];
            A[(size_t)r + (size_t)c * ld] = cd{v.x, v.y};
        }
    }
}

// Diagonal block elimination, blocked by 8-row sub-panels.  The working
// 64 x 64 upper triangle W(r, c), r <= c (diagonal from dw), sits in shared
// memory.  Per sub-panel (rows s0..s0+7):
//   (a) one thread eliminates the 8 x 8 diagonal sub-block in its
//       registers;
//   (b) one thread per column c beyond the sub-block forms the unscaled
//       rows Wun(q, c) = W(q, c) - sum_{q' < q} conj(U(q', q)) Wun(q', c)
//       by substitution and U(q, c) = invD_q Wun(q, c);
//   (c) the eight warps apply the rank-8 update W(r, c) -= sum_q
//       conj(U(q, r)) Wun(q, c) to the rows and columns beyond the
//       sub-panel on the FP64 tensor cores.
// Two barriers per sub-panel: the elimination (a) of the next sub-panel
// runs beside the update (c) of this one.  The recurrence and the pivot follow
// src/linalg.f90:359-391: W(q, q) accumulated this way is the reference's
// pivot conj(x) (M(q, q) is real), zero test included.  CPLX = false
// (default): the pivot's imaginary part, rounding noise of the updates, is
// dropped (kept, it sets a floor of 1e-13..1e-12 under GHEPIIS's residual
// NormOfDiff); true: the complex pivot is kept as the reference keeps it.
// (A register-resident rank-one form with one barrier per pivot measured
// slower, 61 against 32 us per 64 x 64 block: 64 dependent pivot steps of
// FP64 FMA work on eight warps.)
// one m8n8k4 FP64 tensor-core product, D = A B + C (C = D in place)
__device__ __forceinline__ void mma_f64(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

constexpr int DG_LD = LDL_NB + 1;
constexpr int DG_SUB = 8;
constexpr size_t DG_SMEM = (size_t)(LDL_NB * DG_LD + DG_SUB * LDL_NB) * sizeof(double2);

template <bool CPLX>
__global__ void __launch_bounds__(256) k_ldl_diag(cd* __restrict__ A, int ld, int p0, int p1, cd* __restrict__ dw,
                                                   cd* __restrict__ invD, int* __restrict__ status)
{
    extern __shared__ double2 dsm[];
    double2* Ws = dsm;                   // Ws[r * DG_LD + c], r <= c
    double2* Wu = dsm + LDL_NB * DG_LD;  // Wu[q * LDL_NB + c]: unscaled rows of the sub-panel
    __shared__ double2 sid[DG_SUB];      // invD of the sub-panel rows
    const int b = p1 - p0;
    const int tid = threadIdx.x;
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int r = e & 63, c = e >> 6;
        double2 v = make_double2(0.0, 0.0);
        if (r < b && c < b) {
            if (r < c) {
                const cd a = A[(size_t)(p0 + r) + (size_t)(p0 + c) * ld];
                v = make_double2(a.x, a.y);
            } else if (r == c) {
                const cd a = dw[p0 + r];
                v = make_double2(a.x, a.y);
            }
        }
        Ws[r * DG_LD + c] = v;
    }
    __syncthreads();
    // (a) for sub-panel s0: the 8 x 8 diagonal sub-block, in the registers
    // of one thread (no shuffles, so a pivot step costs one reciprocal and
    // three dependent FP64 operations)
    auto eliminate = [&](int s0) {
        const int nq = min(DG_SUB, b - s0);
        cd a[DG_SUB][DG_SUB];
#pragma unroll
        for (int i = 0; i < DG_SUB; i++)
#pragma unroll
            for (int j = i; j < DG_SUB; j++) {
                const double2 v = (j < nq) ? Ws[(s0 + i) * DG_LD + s0 + j] : make_double2(0.0, 0.0);
                a[i][j] = cd{v.x, v.y};
            }
#pragma unroll
        for (int q = 0; q < DG_SUB; q++) {
            if (q < nq) {
                // pivot d = W(q, q) (the reference's conj(x), M(q, q) real);
                // real: its rounding-level imaginary part dropped
                const double dr = a[q][q].x, di = CPLX ? a[q][q].y : 0.0;
                const bool zero = (dr == 0.0 && di == 0.0);
                double id, idi = 0.0;  // 1 / d
                if (CPLX) {
                    const double m = zero ? 0.0 : __drcp_rn(fma(dr, dr, di * di));
                    id = dr * m;
                    idi = -di * m;
                } else {
                    id = zero ? 0.0 : __drcp_rn(dr);
                }
                sid[q] = make_double2(id, idi);
                invD[p0 + s0 + q] = cd{id, idi};
                if (zero) atomicCAS(status + ST_ZERO_PIVOT, 0, p0 + s0 + q + 1);
                cd u[DG_SUB];
#pragma unroll
                for (int j = q + 1; j < DG_SUB; j++)
                    u[j] = CPLX ? cmul(a[q][j], cd{id, idi}) : cd{a[q][j].x * id, a[q][j].y * id};  // U(q, j)
#pragma unroll
                for (int i = q + 1; i < DG_SUB; i++)
#pragma unroll
                    for (int j = i; j < DG_SUB; j++) a[i][j] = cfms(conj(u[i]), a[q][j], a[i][j]);
#pragma unroll
                for (int j = q + 1; j < DG_SUB; j++) a[q][j] = u[j];
            }
        }
#pragma unroll
        for (int i = 0; i < DG_SUB; i++)
#pragma unroll
            for (int j = i + 1; j < DG_SUB; j++)
                if (j < nq) Ws[(s0 + i) * DG_LD + s0 + j] = make_double2(a[i][j].x, a[i][j].y);
    };
    if (tid == 0) eliminate(0);
    __syncthreads();
    const int lane = tid & 31, wp = tid >> 5;
    for (int s0 = 0; s0 < b; s0 += DG_SUB) {
        const int nq = min(DG_SUB, b - s0);
        // (b) sub-panel rows beyond the sub-block, one thread per column
        const int t0 = s0 + DG_SUB;
        if (t0 < b && tid < b - t0) {
            const int c = t0 + tid;
            cd wun[DG_SUB];
#pragma unroll
            for (int q = 0; q < DG_SUB; q++) {
                if (q < nq) {
                    const double2 w = Ws[(s0 + q) * DG_LD + c];
                    cd v = cd{w.x, w.y};
#pragma unroll
                    for (int q2 = 0; q2 < q; q2++) {
                        const double2 u = Ws[(s0 + q2) * DG_LD + s0 + q];  // U(q2, q)
                        v = cfms(cd{u.x, -u.y}, wun[q2], v);
                    }
                    wun[q] = v;
                    Wu[q * LDL_NB + c] = make_double2(v.x, v.y);
                    const double2 id = sid[q];
                    const cd uq = CPLX ? cmul(v, cd{id.x, id.y}) : cd{v.x * id.x, v.y * id.x};
                    Ws[(s0 + q) * DG_LD + c] = make_double2(uq.x, uq.y);
                } else {
                    wun[q] = cd{0.0, 0.0};
                }
            }
        }
        __syncthreads();
        // (c) rank-8 update of the rows and columns beyond the sub-panel on
        // the FP64 tensor cores: 8 x 8 output tiles of the upper triangle
        // (tile row <= tile column); per tile and k-step of 4, four m8n8k4
        // products with the conjugate and the minus sign folded into the U
        // fragment, accumulated onto W.  Warp 0 updates the next diagonal
        // sub-block (tile 0) and its lane 0 eliminates that sub-block at
        // once ((a) of the next sub-panel), while warps 1..7 update the
        // other tiles: the serial elimination overlaps the update.
        if (t0 < b) {
            const int g = lane >> 2, t4 = lane & 3;
            const int T = (b - t0 + 7) >> 3;
            const int ntiles = T * (T + 1) / 2;
            for (int tile = (wp == 0) ? 0 : wp; tile < ntiles; tile += (wp == 0) ? ntiles : 7) {
                int R = 0, rem = tile;
                while (rem >= T - R) {
                    rem -= T - R;
                    R++;
                }
                const int Cc = R + rem;
                const int r = t0 + 8 * R + g;         // fragment row (C and U)
                const int cg = t0 + 8 * Cc + g;       // fragment column of Wun
                const int ca = t0 + 8 * Cc + 2 * t4;  // C columns ca, ca + 1
                double accr[2], acci[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int c = ca + e;
                    double2 w = make_double2(0.0, 0.0);
                    if (r < b && c < b && r <= c) w = Ws[r * DG_LD + c];
                    accr[e] = w.x;
                    acci[e] = w.y;
                }
#pragma unroll
                for (int k0 = 0; k0 < DG_SUB; k0 += 4) {
                    const int q = k0 + t4;
                    double2 u = make_double2(0.0, 0.0), v = make_double2(0.0, 0.0);
                    if (q < nq && r < b) u = Ws[(s0 + q) * DG_LD + r];  // U(q, r)
                    if (q < nq && cg < b) v = Wu[q * LDL_NB + cg];      // Wun(q, c)
                    // W -= conj(U) Wun: Re -= Ur Vr + Ui Vi, Im -= Ur Vi - Ui Vr
                    mma_f64(accr[0], accr[1], -u.x, v.x);
                    mma_f64(accr[0], accr[1], -u.y, v.y);
                    mma_f64(acci[0], acci[1], -u.x, v.y);
                    mma_f64(acci[0], acci[1], u.y, v.x);
                }
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int c = ca + e;
                    if (r < b && c < b && r <= c) Ws[r * DG_LD + c] = make_double2(accr[e], acci[e]);
                }
            }
            if (wp == 0) {
                __syncwarp();
                if (lane == 0) eliminate(t0);
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int r = e & 63, c = e >> 6;
        if (r < c && c < b) {
            const double2 v = Ws[r * DG_LD + c];
            A[(size_t)(p0 + r) + (size_t)(p0 + c) * ld] = cd{v.x, v.y};
        }
    }
}
// Inverse of the unit lower diagonal block L_pp = U_pp^H of every panel in
// [first, nb) (one CTA per panel, all independent): Gaussian elimination of
// L applied to the identity, X(r,s) -= L(r,q) X(q,s).  Row r of X lands in
// linv[(p0 + r) * 64 + s]; the triangular solves of the inverse iteration
// apply these blocks instead of substituting row by row.
__global__ void __launch_bounds__(256) k_ldl_linv(const cd* __restrict__ A, int ld, const int* __restrict__ bstart,
                                                   int first, cd* __restrict__ linv)
{
    extern __shared__ double2 sm[];
    double2* U = sm;                   // U[q*DG_LD + r] = U(q, r), q < r
    double2* X = sm + LDL_NB * DG_LD;  // X[r*DG_LD + s]
    const int blk = first + blockIdx.x;
    const int p0 = bstart[blk], p1 = bstart[blk + 1], b = p1 - p0;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int q = e & 63, r = e >> 6;
        double2 v = make_double2(0.0, 0.0);
        if (q < r && r < b) {
            const cd a = A[(size_t)(p0 + q) + (size_t)(p0 + r) * ld];
            v = make_double2(a.x, a.y);
        }
        U[q * DG_LD + r] = v;
        X[q * DG_LD + r] = make_double2((q == r) ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int q = 0; q + 1 < b; q++) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = ty + 16 * i;
            if (r <= q || r >= b) continue;
            const double2 ur = U[q * DG_LD + r];  // L(r,q) = conj(U(q,r))
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int sc = tx + 16 * j;
                if (sc > q) continue;
                const double2 xq = X[q * DG_LD + sc];
                double2 a = X[r * DG_LD + sc];
                a.x -= ur.x * xq.x + ur.y * xq.y;
                a.y -= ur.x * xq.y - ur.y * xq.x;
                X[r * DG_LD + sc] = a;
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < b * LDL_NB; e += blockDim.x) {
        const int r = e >> 6, s2 = e & 63;
        const double2 v = X[r * DG_LD + s2];
        linv[(size_t)(p0 + r) * LDL_NB + s2] = cd{v.x, v.y};
    }
}

// Neighbour products of the cooperative triangular solves (invit.cu), for
// the panels j in [first, nb): M_j = Linv_j U(j-1, j)^H (blockIdx.y = 0,
// j >= 1) and N_j = Linv_j^H U(j, j+1) (blockIdx.y = 1, j + 1 < nb), each
// stored like linv, row r of panel j at [(p0 + r) * 64 + q].  With them a
// solve's panel j applies the neighbouring panel's solution as one 64 x 64
// product once that panel is published, everything else being done before.
__global__ void __launch_bounds__(256) k_ldl_mn(const cd* __restrict__ A, int ld, const int* __restrict__ bstart,
                                                 int nb, int first, const cd* __restrict__ linv, cd* __restrict__ lmf,
                                                 cd* __restrict__ lnb)
{
    extern __shared__ double2 sm[];
    double2* Ls = sm;                   // Ls[r * DG_LD + c] = Linv_j(r, c)
    double2* Us = sm + LDL_NB * DG_LD;  // Us[c * DG_LD + q]: conj(U(o0 + q, p0 + c)) or U(p0 + c, o0 + q)
    const int j = first + blockIdx.x;
    const bool fwd = blockIdx.y == 0;
    if (fwd ? j < 1 : j + 1 >= nb) return;
    const int p0 = bstart[j], b = bstart[j + 1] - p0;
    const int o0 = fwd ? bstart[j - 1] : bstart[j + 1];
    const int bo = fwd ? p0 - o0 : bstart[j + 2] - o0;
    const int tid = threadIdx.x;
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int c = e & 63, r = e >> 6;
        double2 v = make_double2(0.0, 0.0);
        if (r < b && c < b) {
            const cd x = linv[(size_t)(p0 + r) * LDL_NB + c];
            v = make_double2(x.x, x.y);
        }
        Ls[r * DG_LD + c] = v;
        // the neighbour block, read along its columns
        const int lo = e & 63, hi = e >> 6;
        double2 u = make_double2(0.0, 0.0);
        if (fwd) {
            if (hi < b && lo < bo) {
                const cd x = A[(size_t)(o0 + lo) + (size_t)(p0 + hi) * ld];
                u = make_double2(x.x, -x.y);
            }
            Us[hi * DG_LD + lo] = u;
        } else {
            if (lo < b && hi < bo) {
                const cd x = A[(size_t)(p0 + lo) + (size_t)(o0 + hi) * ld];
                u = make_double2(x.x, x.y);
            }
            Us[lo * DG_LD + hi] = u;
        }
    }
    __syncthreads();
    const int r = tid >> 2, q0 = tid & 3;
    double accr[16], acci[16];
#pragma unroll
    for (int i = 0; i < 16; i++) accr[i] = acci[i] = 0.0;
    const int c0 = fwd ? 0 : r, c1 = fwd ? r + 1 : LDL_NB;
    for (int c = c0; c < c1; c++) {
        double2 l = fwd ? Ls[r * DG_LD + c] : Ls[c * DG_LD + r];
        if (!fwd) l.y = -l.y;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const double2 u = Us[c * DG_LD + q0 + 4 * i];
            accr[i] = fma(l.x, u.x, fma(-l.y, u.y, accr[i]));
            acci[i] = fma(l.x, u.y, fma(l.y, u.x, acci[i]));
        }
    }
    if (r < b) {
        cd* out = (fwd ? lmf : lnb) + (size_t)(p0 + r) * LDL_NB;
#pragma unroll
        for (int i = 0; i < 16; i++) out[q0 + 4 * i] = cd{accr[i], acci[i]};
    }
}

// Panel rows beyond the diagonal block, by substitution:
//   Wun(q, c) = W(q, c) - sum_{q' < q} conj(U(q', q)) Wun(q', c)
//   U(q, c)   = invD_q Wun(q, c);  vbuf(q, c) = Wun(q, c)
// (the forward form of src/linalg.f90:384-389 for a whole panel).  One warp
// per column, lanes hold rows lane and lane + 32; U_pp comes from A through
// shared memory.  vbuf(q, c) sits at vbuf[c * vld + q].
constexpr int TRSM_COLS = 8;
__global__ void __launch_bounds__(256) k_ldl_trsm(cd* __restrict__ A, int ld, int p0, int p1, int c0, int n,
                                                   const cd* __restrict__ invD, cd* __restrict__ vbuf, int vld)
{
    extern __shared__ double2 sm[];
    double2* U = sm;  // U[q*DG_LD + r] = U(q, r), q < r
    const int b = p1 - p0;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int q = e & 63, r = e >> 6;
        if (q < r && r < b) {
            const cd a = A[(size_t)(p0 + q) + (size_t)(p0 + r) * ld];
            U[q * DG_LD + r] = make_double2(a.x, a.y);
        }
    }
    __syncthreads();
    const int r0 = lane, r1 = lane + 32;
    const cd d0 = (r0 < b) ? invD[p0 + r0] : cd{0.0, 0.0};
    const cd d1 = (r1 < b) ? invD[p0 + r1] : cd{0.0, 0.0};
    for (int m = 0; m < TRSM_COLS / 8; m++) {
        const int c = c0 + blockIdx.x * TRSM_COLS + wp * (TRSM_COLS / 8) + m;  // one column per warp
        if (c >= n) break;
        cd* col = A + (size_t)c * ld + p0;
        cd w0 = (r0 < b) ? col[r0] : cd{0.0, 0.0};
        cd w1 = (r1 < b) ? col[r1] : cd{0.0, 0.0};
        for (int q = 0; q < b; q++) {
            // broadcast the finished row q
            const cd src = (q < 32) ? w0 : w1;
            cd wq;
            wq.x = __shfl_sync(0xffffffffu, src.x, q & 31);
            wq.y = __shfl_sync(0xffffffffu, src.y, q & 31);
            if (r0 > q && r0 < b) {
                const double2 uq = U[q * DG_LD + r0];
                w0 = cfms(cd{uq.x, -uq.y}, wq, w0);
            }
            if (r1 > q && r1 < b) {
                const double2 uq = U[q * DG_LD + r1];
                w1 = cfms(cd{uq.x, -uq.y}, wq, w1);
            }
        }
        cd* v = vbuf + (size_t)c * vld;
        if (r0 < b) {
            v[r0] = w0;
            col[r0] = cmul(w0, d0);
        }
        if (r1 < b) {
            v[r1] = w1;
            col[r1] = cmul(w1, d1);
        }
    }
}

// Trailing update over 64 x TC output tiles on the FP64 tensor cores:
//   W(r, c) -= sum_q conj(U(q, r)) Wun(q, c),  r in [r0, rend), c in [max(r, c0), n)
// with mma.sync.m8n8k4.f64.  Eight warps as WR x WC, each a (64/WR) x
// (TC/WC) complex sub-tile of 8 x 8 tiles; per tile and k-step of 4 the real
// and imaginary accumulators take four mma: Re += Ur Vr + Ui Vi and
// Im += Ur Vi + (-Ui) Vr (the conjugate folded into a negated fragment).
// U and Wun are staged by cp.async in two buffers of 16 k rows each, so that
// the next chunk streams in while the current one is multiplied; complex
// values stay interleaved in shared memory with a pitch of 66 double2
// (= 2 mod 8 slots of 16 B), so the fragment loads of a warp are
// conflict-free.  The tile's old values are read after the products (kept
// out of registers during them).  <32, 4, 2>: the bulk (64 x 32 tiles, side
// stream; at 64 registers four CTAs fit on an SM, which measured faster
// than 64 x 64 tiles at three); <16, 8, 1>: the rows of the next panel
// (64 x 16 tiles, enough CTAs for one row of tiles, main stream).
constexpr int BLK_KC = 16;
constexpr int BLK_P = 66;
// pitch of the Wun buffer: TC + 2 double2 (also = 2 mod 8), 66 for TC = 64
template <int TC>
__host__ __device__ constexpr int blk_vp() { return TC == 64 ? BLK_P : TC + 2; }
template <int TC>
constexpr size_t blk_smem() { return (size_t)2 * BLK_KC * (BLK_P + blk_vp<TC>()) * sizeof(double2); }

template <int TC, int WR, int WC>
__global__ void __launch_bounds__(256, TC == 64 ? 3 : 4) k_ldl_bulk(cd* __restrict__ A, int ld, int p0, int p1, int r0, int rend,
                                                   int c0, int n, const cd* __restrict__ vbuf, int vld,
                                                   cd* __restrict__ dw)
{
    constexpr int MT = LDL_NB / WR / 8;  // 8 x 8 tiles per warp along rows
    constexpr int NT = TC / WC / 8;      // and along columns
    constexpr int VP = blk_vp<TC>();
    extern __shared__ double2 sb[];
    const int rb = r0 + blockIdx.y * LDL_NB;
    const int cb = c0 + blockIdx.x * TC;
    if (rb > cb + TC - 1) return;  // tile entirely below the diagonal
    const int b = p1 - p0;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    {
        // bring the tile's old values towards L2 now; they are read after
        // the products (64 rows x 16 B = eight 128-byte lines per column)
        const int cc = cb + (tid >> 3), rr = rb + 8 * (tid & 7);
        if (cc < n && (tid >> 3) < TC && rr < rend && rr <= cc)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(A + (size_t)rr + (size_t)cc * ld));
    }
    const int wr = wp / WC, wc = wp % WC;
    const int g = lane >> 2, t4 = lane & 3;
    double accr[MT][NT][2], acci[MT][NT][2];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) accr[mt][nt][e] = acci[mt][nt][e] = 0.0;
    auto stage = [&](int ch, int buf) {
        const int k0 = ch * BLK_KC;
        double2* Us = sb + buf * BLK_KC * (BLK_P + VP);
        double2* Vs = Us + BLK_KC * BLK_P;
        for (int e = tid; e < BLK_KC * LDL_NB; e += 256) {
            const int q = e % BLK_KC, mm = e / BLK_KC;
            const int r = rb + mm;
            const bool ku = (k0 + q < b) && (r < rend);
            cp_async16(Us + q * BLK_P + mm, ku ? (const void*)(A + (size_t)(p0 + k0 + q) + (size_t)r * ld) : (const void*)A,
                       ku ? 16 : 0);
        }
        for (int e = tid; e < BLK_KC * TC; e += 256) {
            const int q = e % BLK_KC, mm = e / BLK_KC;
            const int c = cb + mm;
            const bool kv = (k0 + q < b) && (c < n);
            cp_async16(Vs + q * VP + mm,
                       kv ? (const void*)(vbuf + (size_t)(k0 + q) + (size_t)c * vld) : (const void*)vbuf, kv ? 16 : 0);
        }
        cp_async_commit();
    };
    const int nch = (b + BLK_KC - 1) / BLK_KC;
    stage(0, 0);
    for (int ch = 0; ch < nch; ch++) {
        if (ch + 1 < nch) {
            stage(ch + 1, (ch + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double2* Us = sb + (ch & 1) * BLK_KC * (BLK_P + VP);
        const double2* Vs = Us + BLK_KC * BLK_P;
#pragma unroll
        for (int kk = 0; kk < BLK_KC; kk += 4) {
            const int kr = (kk + t4) * BLK_P;
            double2 a[MT], v[NT];
#pragma unroll
            for (int mt = 0; mt < MT; mt++) a[mt] = Us[kr + (wr * MT + mt) * 8 + g];
#pragma unroll
            for (int nt = 0; nt < NT; nt++) v[nt] = Vs[(kk + t4) * VP + (wc * NT + nt) * 8 + g];
#pragma unroll
            for (int mt = 0; mt < MT; mt++)
#pragma unroll
                for (int nt = 0; nt < NT; nt++) {
                    mma_f64(accr[mt][nt][0], accr[mt][nt][1], a[mt].x, v[nt].x);
                    mma_f64(accr[mt][nt][0], accr[mt][nt][1], a[mt].y, v[nt].y);
                    mma_f64(acci[mt][nt][0], acci[mt][nt][1], a[mt].x, v[nt].y);
                    mma_f64(acci[mt][nt][0], acci[mt][nt][1], -a[mt].y, v[nt].x);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int r = rb + (wr * MT + mt) * 8 + g;
                const int c = cb + (wc * NT + nt) * 8 + t4 * 2 + e;
                if (r >= rend || c >= n || c < r) continue;
                const double vr = accr[mt][nt][e], vi = acci[mt][nt][e];
                const double2 o = (c == r) ? *reinterpret_cast<const double2*>(dw + c)
                                           : *reinterpret_cast<const double2*>(A + (size_t)r + (size_t)c * ld);
                if (c == r)
                    *reinterpret_cast<double2*>(dw + c) = make_double2(o.x - vr, o.y + vi);
                else
                    *reinterpret_cast<double2*>(A + (size_t)r + (size_t)c * ld) = make_double2(o.x - vr, o.y - vi);
            }
}

static bool g_ldl_attr = false;

// Trailing update by panel [p0, p1) of rows [r0, rend), columns
// [max(r, c0), n).
// k rows [p0, p1) of U and of vb (vb(q, c) at vb[c * vld + q - p0]).
static void launch_update(Ctx& c, cudaStream_t st, const cd* vb, int vld, int p0, int p1, int r0, int rend, int c0,
                          int n)
{
    if (rend <= r0 || c0 >= n || p1 <= p0) return;
    const int nrb = (rend - r0 + LDL_NB - 1) / LDL_NB;
    if (nrb == 1) {
        // one panel of rows: narrow 64 x 16 tiles so that enough CTAs run
        dim3 g((n - c0 + 15) / 16, 1);
        k_ldl_bulk<16, 8, 1><<<g, 256, blk_smem<16>(), st>>>(c.F, c.ld, p0, p1, r0, rend, c0, n, vb, vld, c.dw);
    } else {
        dim3 g((n - c0 + 31) / 32, nrb);
        k_ldl_bulk<32, 4, 2><<<g, 256, blk_smem<32>(), st>>>(c.F, c.ld, p0, p1, r0, rend, c0, n, vb, vld, c.dw);
    }
    c.launches++;
}

// Enqueue the kernels of one factorisation (see ldlh_factor).
static void enqueue_factor(Ctx& c, int m0, int n, const std::vector<int>& starts, int nexist)
{
    const bool pairs = (n - m0) >= LDL_PAIR_MIN;
    const size_t sm1 = LDL_NB * DG_LD * sizeof(double2);
    const int nblk = (int)starts.size();
    auto blk_end = [&](int i) { return (i + 1 < nblk) ? starts[i + 1] : n; };
    auto trsm = [&](int p0, int p1, int cfrom, cd* vb) {
        if (cfrom >= n) return;
        k_ldl_trsm<<<(n - cfrom + TRSM_COLS - 1) / TRSM_COLS, 256, sm1, c.stream>>>(c.F, c.ld, p0, p1, cfrom, n,
                                                                                   c.invD, vb, LDL_VLD);
        c.launches++;
    };
    auto diag = [&](int p0, int p1) {
        if (c.pivot_mode)
            k_ldl_diag<true><<<1, 256, DG_SMEM, c.stream>>>(c.F, c.ld, p0, p1, c.dw, c.invD, c.status);
        else
            k_ldl_diag<false><<<1, 256, DG_SMEM, c.stream>>>(c.F, c.ld, p0, p1, c.dw, c.invD, c.status);
        c.launches++;
    };
    if (n > m0) {
        const int ct0 = m0 / 32, ct1 = (n + 31) / 32;
        dim3 g(ct1 - ct0, ct1);
        k_ldl_mirror<<<g, 256, 0, c.stream>>>(c.F, c.ld, m0, n, c.dw, ct0);
        c.launches++;
    }
    // existing panels (bordered update): apply them to the new columns in order
    for (int i = 0; i < nexist; i++) {
        const int p0 = starts[i], p1 = std::min(blk_end(i), m0);
        if (p1 <= p0 || m0 >= n) continue;
        trsm(p0, p1, m0, c.vbuf);
        launch_update(c, c.stream, c.vbuf, LDL_VLD, p0, p1, p1, n, m0, n);
    }
    // new panels, right-looking with a lookahead: the rows of the next panel
    // are updated first on the main stream, so that panel's factorisation
    // overlaps the trailing update running on the side stream.  The
    // trailing update of panel i is split: first the rows of panel i+2
    // (after which lev[1] is recorded; the lookahead update of panel i+1
    // needs only those), then the rest, which thus has two panel steps to
    // complete before the lookahead of panel i+2 touches its rows.  Three
    // panel buffers rotate, so a buffer is rewritten only after the update
    // that reads it has finished (stream order through lev[1]).
    bool bulk_recorded = false;  // lev[1] recorded by this sequence (never wait on an older record)
    for (int i = nexist; i < nblk && !pairs; i++) {
        const int p0 = starts[i], p1 = blk_end(i);
        const int p2 = (i + 1 < nblk) ? blk_end(i + 1) : n;
        const int p3 = (i + 2 < nblk) ? blk_end(i + 2) : n;
        cd* vb = c.vbuf + (size_t)((i - nexist) % 3) * LDL_VLD * c.ld;
        diag(p0, p1);
        if (p1 >= n) break;
        trsm(p0, p1, p1, vb);
        cudaEventRecord(c.lev[0], c.stream);
        // rows of the next panel wait for the previous trailing update's first part
        if (bulk_recorded) cudaStreamWaitEvent(c.stream, c.lev[1], 0);
        launch_update(c, c.stream, vb, LDL_VLD, p0, p1, p1, p2, p1, n);
        cudaStreamWaitEvent(c.side, c.lev[0], 0);
        launch_update(c, c.side, vb, LDL_VLD, p0, p1, p2, p3, p2, n);
        cudaEventRecord(c.lev[1], c.side);
        launch_update(c, c.side, vb, LDL_VLD, p0, p1, p3, n, p3, n);
        bulk_recorded = true;
    }
    // Large factorisations take the new panels in pairs (A = [a0, a1),
    // B = [a1, b1)): B's rows are updated by A (rank 64) before B is
    // eliminated, the rows of the next pair by both (rank 128) on the main
    // stream, and the rest of the matrix by both on the side stream (first
    // the rows of the pair after next, then everything beyond), which halves
    // the passes over the trailing triangle; it measured 57.5 against 63.8
    // ms at K = 10000 and 5.9 against 5.7 ms at K = 4000, where the longer
    // panel chain weighs more.
    int step = 0;
    for (int i = nexist; i < nblk && pairs; i += 2, step++) {
        const int a0 = starts[i], a1 = blk_end(i);
        const bool hasB = i + 1 < nblk;
        const int b1 = hasB ? blk_end(i + 1) : a1;
        const int n1 = (i + 3 < nblk) ? blk_end(i + 3) : n;  // end of the next pair
        const int n2 = (i + 5 < nblk) ? blk_end(i + 5) : n;  // end of the pair after next
        cd* vb = c.vbuf + (size_t)(step % 3) * LDL_VLD * c.ld;
        diag(a0, a1);
        if (a1 >= n) break;
        trsm(a0, a1, a1, vb);
        if (hasB) {
            launch_update(c, c.stream, vb, LDL_VLD, a0, a1, a1, b1, a1, n);
            diag(a1, b1);
            if (b1 >= n) break;
            trsm(a1, b1, b1, vb + LDL_NB);
        }
        cudaEventRecord(c.lev[0], c.stream);
        if (bulk_recorded) cudaStreamWaitEvent(c.stream, c.lev[1], 0);
        launch_update(c, c.stream, vb, LDL_VLD, a0, b1, b1, n1, b1, n);
        cudaStreamWaitEvent(c.side, c.lev[0], 0);
        launch_update(c, c.side, vb, LDL_VLD, a0, b1, n1, n2, n1, n);
        cudaEventRecord(c.lev[1], c.side);
        launch_update(c, c.side, vb, LDL_VLD, a0, b1, n2, n, n2, n);
        bulk_recorded = true;
    }
    if (bulk_recorded) {
        // join everything queued on the side stream
        cudaEventRecord(c.lev[0], c.side);
        cudaStreamWaitEvent(c.stream, c.lev[0], 0);
    }
    if (nblk > nexist) {
        k_ldl_linv<<<nblk - nexist, 256, 2 * sm1, c.stream>>>(c.F, c.ld, c.dblk, nexist, c.linv);
        // the last existing panel's N changes with the first new panel
        const int f = std::max(nexist - 1, 0);
        k_ldl_mn<<<dim3(nblk - f, 2), 256, 2 * sm1, c.stream>>>(c.F, c.ld, c.dblk, nblk, f, c.linv, c.lmf, c.lnb);
        c.launches += 2;
    }
}

// A whole factorisation (m0 = 0) as one persistent kernel (ldlp.cu): the
// working upper triangle and diagonal, the tile tasks, then the inverse
// diagonal blocks of the solves.
static void enqueue_persist(Ctx& c, int n, const unsigned* tasks, int ntasks, unsigned long long* trace = nullptr)
{
    const int ct1 = (n + 31) / 32;
    k_ldl_mirror<<<dim3(ct1, ct1), 256, 0, c.stream>>>(c.F, c.ld, 0, n, c.dw, 0);
    c.launches++;
    ldlp_enqueue(c, n, tasks, ntasks, trace);
    const int nblk = (n + LDL_NB - 1) / LDL_NB;
    k_ldl_linv<<<nblk, 256, 2 * LDL_NB * DG_LD * sizeof(double2), c.stream>>>(c.F, c.ld, c.dblk, 0, c.linv);
    k_ldl_mn<<<dim3(nblk, 2), 256, 2 * LDL_NB * DG_LD * sizeof(double2), c.stream>>>(c.F, c.ld, c.dblk, nblk, 0,
                                                                                    c.linv, c.lmf, c.lnb);
    c.launches += 2;
}

static void ldl_attrs()
{
    if (g_ldl_attr) return;
    const size_t sm1 = LDL_NB * DG_LD * sizeof(double2);
    cudaFuncSetAttribute(k_ldl_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    cudaFuncSetAttribute(k_ldl_diag<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DG_SMEM);
    cudaFuncSetAttribute(k_ldl_diag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DG_SMEM);
    cudaFuncSetAttribute(k_ldl_linv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * sm1));
    cudaFuncSetAttribute(k_ldl_mn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(2 * sm1));
    cudaFuncSetAttribute(k_ldl_bulk<32, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk_smem<32>());
    cudaFuncSetAttribute(k_ldl_bulk<16, 8, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk_smem<16>());
    g_ldl_attr = true;
}

// Factorise rows m0..n-1 of M = H - lambda~ S given the factor of rows
// 0..m0-1.  The launch sequence depends only on (m0, n) and the existing
// panel boundaries, so it is captured once into a CUDA graph (both streams)
// and replayed.  A whole factorisation (m0 = 0) runs as the persistent
// kernel of ldlp.cu unless ecg_set_factor_mode selected the launch-per-panel
// form.
int ldlh_factor(Ctx& c, int m0, int n)
{
    if (m0 < 0 || m0 > n || n > c.ld) return -1;
    if (m0 > c.fact_n) return -1;
    ldl_attrs();
    // block list: existing blocks truncated at m0, then new 64-row blocks
    std::vector<int> starts;
    for (int s : c.blk_start)
        if (s < m0) starts.push_back(s);
    const int nexist = (int)starts.size();
    for (int s = m0; s < n; s += LDL_NB) starts.push_back(s);
    // panel boundaries (starts..., n) for the inverse blocks and the solves
    const int nb = (int)starts.size();
    for (int i = 0; i < nb; i++) c.bounds_h[i] = starts[i];
    c.bounds_h[nb] = n;
    if (cudaMemcpyAsync(c.dblk, c.bounds_h, (nb + 1) * sizeof(int), cudaMemcpyHostToDevice, c.stream) !=
        cudaSuccess)
        return -2;
    // whole factorisations take the persistent kernel below LDL_PAIR_MIN
    // rows (at 10000 rows the panel pairs' rank-128 launches measured 57.2
    // against its 59.4 ms)
    const bool persist = (m0 == 0 && n > 0 && n < LDL_PAIR_MIN && c.factor_mode == 0 && ldlp_grid(c) > 0);
    std::vector<int> key = {m0, n, c.pivot_mode, persist ? 1 : 0};
    key.insert(key.end(), starts.begin(), starts.begin() + nexist);
    Ctx::LdlGraph* g = nullptr;
    for (auto& e : c.ldl_graphs)
        if (e.key == key) g = &e;
    if (!g) {
        unsigned* tasks = nullptr;
        int ntasks = 0;
        if (persist) {
            const int r = ldlp_reserve(c, nb);
            if (r) return r;
            const int t = ldlp_tasks(c, n, &tasks, &ntasks);
            if (t) return t;
        }
        auto enqueue = [&]() {
            if (persist)
                enqueue_persist(c, n, tasks, ntasks);
            else
                enqueue_factor(c, m0, n, starts, nexist);
        };
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            const long long l0 = c.launches;
            enqueue();
            c.graph_launches = c.launches - l0;
            c.launches = l0;
            ok = cudaStreamEndCapture(c.stream, &graph) == cudaSuccess && graph &&
                 cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        }
        if (graph) cudaGraphDestroy(graph);
        if (!ok) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            // capture unavailable: run the launches directly (a persistent
            // factorisation keeps its task list until the next one)
            if (persist) {
                if (c.lp_direct) {
                    cudaStreamSynchronize(c.stream);
                    cudaFree(c.lp_direct);
                }
                c.lp_direct = tasks;
                c.lp_direct_n = n;
                c.lp_direct_count = ntasks;
            }
            enqueue();
            if (cudaGetLastError() != cudaSuccess) return -2;
            c.blk_start = starts;
            c.fact_n = n;
            return 0;
        }
        if (c.ldl_graphs.size() >= 8) {
            cudaStreamSynchronize(c.stream);
            cudaGraphExecDestroy(c.ldl_graphs.front().exec);
            if (c.ldl_graphs.front().tasks) cudaFree(c.ldl_graphs.front().tasks);
            c.ldl_graphs.erase(c.ldl_graphs.begin());
        }
        c.ldl_graphs.push_back({key, exec});
        g = &c.ldl_graphs.back();
        g->launches = c.graph_launches;
        g->tasks = tasks;
        g->ntasks = ntasks;
    }
    if (cudaGraphLaunch(g->exec, c.stream) != cudaSuccess) return -2;
    c.launches += g->launches;
    c.blk_start = starts;
    c.fact_n = n;
    return 0;
}

// One persistent factorisation of rows 0..n-1 of the matrix in F's lower
// triangle, outside any graph, with a timing record per task: out receives
// 4 values per task (code | CTA << 32 | panels applied << 48, then the
// globaltimer in ns when the CTA began waiting for the task's tiles, when
// they were ready, when the task was published).  The factor is left as
// ldlh_factor(c, 0, n) leaves it.
int ldlh_factor_traced(Ctx& c, int n, unsigned long long* out, long long cap, long long* count)
{
    if (n < 1 || n > c.ld) return -1;
    if (ldlp_grid(c) <= 0) return -1;
    const int nb = (n + LDL_NB - 1) / LDL_NB;
    ldl_attrs();
    std::vector<int> starts;
    for (int s = 0; s < n; s += LDL_NB) starts.push_back(s);
    for (int i = 0; i < nb; i++) c.bounds_h[i] = starts[i];
    c.bounds_h[nb] = n;
    if (cudaMemcpyAsync(c.dblk, c.bounds_h, (nb + 1) * sizeof(int), cudaMemcpyHostToDevice, c.stream) !=
        cudaSuccess)
        return -2;
    if (ldlp_reserve(c, nb)) return -3;
    unsigned* tasks = nullptr;
    int ntasks = 0;
    if (ldlp_tasks(c, n, &tasks, &ntasks)) return -2;
    const long long total = ldlp_task_total(n);
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, (size_t)total * 4 * sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(tasks);
        return -3;
    }
    enqueue_persist(c, n, tasks, ntasks, d);
    unsigned recs = 0;
    const size_t ntile = (size_t)nb * (nb + 1) / 2;  // trace records at ctl[2], ctl = counters + 2 ntile
    int r = 0;
    if (cudaMemcpyAsync(&recs, c.lp_cnt + 2 * ntile + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        r = -2;
    if (!r) {
        *count = recs;
        if (out && cap >= (long long)recs * 4 &&
            cudaMemcpy(out, d, (size_t)recs * 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess)
            r = -2;
    }
    cudaFree(d);
    cudaFree(tasks);
    c.blk_start = starts;
    c.fact_n = n;
    return r;
}

}  // namespace ecg
