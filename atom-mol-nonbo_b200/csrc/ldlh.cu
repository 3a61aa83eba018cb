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
//                 producing U (= L^H), invD and Linv = (U_pp^H)^-1;
//   k_ldl_trsm    Wun(p, c) = Linv W(p, c), U(p, c) = invD Wun   (c beyond p);
//   k_ldl_update  W(r, c) -= sum_q conj(U(q,r)) Wun(q,c), r <= c beyond p
//                 (the Hermitian rank-64 trailing update, a complex GEMM).
// The off-diagonal recurrence and the pivot d = conj(.) follow
// src/linalg.f90:359-391 term for term; only the summation order differs.
#include "ecg_internal.h"

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

// Diagonal block elimination.  Shared memory: W (upper part used) and
// X = L_pp^-1 (unit lower), both 64 x 65 complex (padded rows).  Thread
// (ty, tx) of a 16 x 16 layout owns rows ty + 16i and columns tx + 16j of
// both matrices, so each elimination step is a masked 4 x 4 update per
// thread with no index arithmetic beyond shifts.
constexpr int DG_LD = LDL_NB + 1;
__global__ void __launch_bounds__(256) k_ldl_diag(cd* __restrict__ A, int ld, int p0, int p1, cd* __restrict__ dw,
                                                   cd* __restrict__ invD, cd* __restrict__ linv,
                                                   int* __restrict__ status)
{
    extern __shared__ double2 sm[];
    double2* W = sm;                   // W[r*DG_LD + c]
    double2* X = sm + LDL_NB * DG_LD;  // X[r*DG_LD + s]
    __shared__ double2 u[LDL_NB];
    __shared__ double2 dws[LDL_NB];
    const int b = p1 - p0;
    const int tid = threadIdx.x;
    const int ty = tid >> 4, tx = tid & 15;
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int r = e & 63, c = e >> 6;
        double2 v = make_double2(0.0, 0.0);
        if (r < c && c < b) {
            const cd a = A[(size_t)(p0 + r) + (size_t)(p0 + c) * ld];
            v = make_double2(a.x, a.y);
        }
        W[r * DG_LD + c] = v;
        X[r * DG_LD + c] = make_double2((r == c) ? 1.0 : 0.0, 0.0);
    }
    if (tid < LDL_NB) {
        const cd d = (tid < b) ? dw[p0 + tid] : cd{1.0, 0.0};
        dws[tid] = make_double2(d.x, d.y);
    }
    __syncthreads();
    for (int q = 0; q < b; q++) {
        // pivot d = conj(dw_q) (src/linalg.f90:375-383)
        const double2 dq = dws[q];
        const double dre = dq.x, dim = -dq.y;
        const double nrm = dre * dre + dim * dim;
        double2 iq = make_double2(0.0, 0.0);
        if (nrm != 0.0) iq = make_double2(dre / nrm, -dim / nrm);
        if (tid < LDL_NB) {
            const int c = tid;
            double2 uc = make_double2(0.0, 0.0);
            if (c > q && c < b) {
                const double2 wv = W[q * DG_LD + c];
                uc = make_double2(wv.x * iq.x - wv.y * iq.y, wv.x * iq.y + wv.y * iq.x);
            }
            u[c] = uc;
            if (tid == 0) {
                invD[p0 + q] = cd{iq.x, iq.y};
                if (nrm == 0.0) atomicCAS(status + ST_ZERO_PIVOT, 0, p0 + q + 1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = ty + 16 * i;
            if (r <= q || r >= b) continue;
            const double2 ur = u[r];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = tx + 16 * j;
                // W(r,c) -= conj(U(q,r)) W(q,c)   (r < c)
                if (c > r && c < b) {
                    const double2 wq = W[q * DG_LD + c];
                    double2 a = W[r * DG_LD + c];
                    a.x -= ur.x * wq.x + ur.y * wq.y;
                    a.y -= ur.x * wq.y - ur.y * wq.x;
                    W[r * DG_LD + c] = a;
                } else if (c == r) {
                    // dw -= conj(W(q,c)) U(q,c)
                    const double2 wq = W[q * DG_LD + c];
                    double2 a = dws[c];
                    a.x -= wq.x * ur.x + wq.y * ur.y;
                    a.y -= wq.x * ur.y - wq.y * ur.x;
                    dws[c] = a;
                }
                // X(r,s) -= L(r,q) X(q,s), L(r,q) = conj(U(q,r)), s <= q
                const int sc = c;
                if (sc <= q) {
                    const double2 xq = X[q * DG_LD + sc];
                    double2 a = X[r * DG_LD + sc];
                    a.x -= ur.x * xq.x + ur.y * xq.y;
                    a.y -= ur.x * xq.y - ur.y * xq.x;
                    X[r * DG_LD + sc] = a;
                }
            }
        }
        __syncthreads();
        if (tid < LDL_NB && tid > q && tid < b) W[q * DG_LD + tid] = u[tid];
        __syncthreads();
    }
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int r = e & 63, c = e >> 6;
        if (r < c && c < b) {
            const double2 v = W[r * DG_LD + c];
            A[(size_t)(p0 + r) + (size_t)(p0 + c) * ld] = cd{v.x, v.y};
        }
    }
    for (int e = tid; e < b * LDL_NB; e += blockDim.x) {
        const int r = e >> 6, s2 = e & 63;
        const double2 v = X[r * DG_LD + s2];
        linv[(size_t)(p0 + r) * LDL_NB + s2] = cd{v.x, v.y};
    }
}

// Panel rows: Wun(p, c) = Linv W(p, c); U(p, c) = invD Wun; vbuf(., c) = Wun.
// One CTA per 64 columns; 256 threads, each 4 rows x 4 columns.
__global__ void __launch_bounds__(256) k_ldl_trsm(cd* __restrict__ A, int ld, int p0, int p1, int c0, int n,
                                                   const cd* __restrict__ invD, const cd* __restrict__ linv,
                                                   cd* __restrict__ vbuf)
{
    extern __shared__ double2 sm[];
    double2* Ls = sm;                     // Ls[q*64 + r] = Linv(r, q)
    double2* Ws = sm + LDL_NB * LDL_NB;   // Ws[q*64 + c]
    const int b = p1 - p0;
    const int cbase = c0 + blockIdx.x * LDL_NB;
    const int tid = threadIdx.x;
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int s = e % LDL_NB, r = e / LDL_NB;
        double2 v = make_double2(0.0, 0.0);
        if (r < b && s < b) {
            const cd a = ldg2(linv + (size_t)(p0 + r) * LDL_NB + s);
            v = make_double2(a.x, a.y);
        }
        Ls[s * LDL_NB + r] = v;
    }
    for (int e = tid; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int q = e % LDL_NB, cc = e / LDL_NB;
        const int c = cbase + cc;
        double2 v = make_double2(0.0, 0.0);
        if (q < b && c < n) {
            const cd a = A[(size_t)(p0 + q) + (size_t)c * ld];
            v = make_double2(a.x, a.y);
        }
        Ws[q * LDL_NB + cc] = v;
    }
    __syncthreads();
    const int tr = tid % 16, tc = tid / 16;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0.0, 0.0);
    for (int q = 0; q < b; q++) {
        double2 a[4], w[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = Ls[q * LDL_NB + tr + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; j++) w[j] = Ws[q * LDL_NB + tc + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                acc[i][j].x = fma(a[i].x, w[j].x, fma(-a[i].y, w[j].y, acc[i][j].x));
                acc[i][j].y = fma(a[i].x, w[j].y, fma(a[i].y, w[j].x, acc[i][j].y));
            }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = tr + 16 * i;
        if (r >= b) continue;
        const cd id = invD[p0 + r];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = cbase + tc + 16 * j;
            if (c >= n) continue;
            const double2 v = acc[i][j];
            vbuf[(size_t)r + (size_t)c * LDL_NB] = cd{v.x, v.y};
            A[(size_t)(p0 + r) + (size_t)c * ld] = cd{v.x * id.x - v.y * id.y, v.x * id.y + v.y * id.x};
        }
    }
}

// Trailing update over 64 x 64 output tiles: rows r in [r0, n), columns
// c in [max(r, c0), n).  K-chunks of 32 panel rows through shared memory.
constexpr int UPD_KC = 32;
constexpr int UPD_LD = LDL_NB + 1;  // padded row of the shared tiles
__global__ void __launch_bounds__(256) k_ldl_update(cd* __restrict__ A, int ld, int p0, int p1, int r0, int c0,
                                                     int n, const cd* __restrict__ vbuf, cd* __restrict__ dw)
{
    extern __shared__ double2 sm[];
    double2(*Us)[UPD_LD] = reinterpret_cast<double2(*)[UPD_LD]>(sm);                   // U(q, r)
    double2(*Vs)[UPD_LD] = reinterpret_cast<double2(*)[UPD_LD]>(sm + UPD_KC * UPD_LD);  // Wun(q, c)
    const int rb = r0 + blockIdx.y * LDL_NB;
    const int cb = c0 + blockIdx.x * LDL_NB;
    if (rb > cb + LDL_NB - 1) return;  // tile entirely below the diagonal
    const int b = p1 - p0;
    const int tid = threadIdx.x;
    const int tr = tid % 16, tc = tid / 16;
    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = make_double2(0.0, 0.0);
    for (int k0 = 0; k0 < b; k0 += UPD_KC) {
        for (int e = tid; e < UPD_KC * LDL_NB; e += blockDim.x) {
            const int q = e % UPD_KC, rr = e / UPD_KC;
            const int r = rb + rr, c = cb + rr;
            double2 u = make_double2(0.0, 0.0), v = make_double2(0.0, 0.0);
            if (k0 + q < b) {
                if (r < n) {
                    const cd a = A[(size_t)(p0 + k0 + q) + (size_t)r * ld];
                    u = make_double2(a.x, a.y);
                }
                if (c < n) {
                    const cd a = ldg2(vbuf + (size_t)(k0 + q) + (size_t)c * LDL_NB);
                    v = make_double2(a.x, a.y);
                }
            }
            Us[q][rr] = u;
            Vs[q][rr] = v;
        }
        __syncthreads();
#pragma unroll 4
        for (int q = 0; q < UPD_KC; q++) {
            double2 a[4], w[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = Us[q][tr + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) w[j] = Vs[q][tc + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    // acc += conj(a) * w
                    acc[i][j].x = fma(a[i].x, w[j].x, fma(a[i].y, w[j].y, acc[i][j].x));
                    acc[i][j].y = fma(a[i].x, w[j].y, fma(-a[i].y, w[j].x, acc[i][j].y));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int r = rb + tr + 16 * i;
        if (r >= n) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = cb + tc + 16 * j;
            if (c >= n || c < r) continue;
            const double2 v = acc[i][j];
            if (c == r) {
                // dw -= conj(sum conj(U) Wun) = sum conj(Wun) U (src/linalg.f90:370-372)
                cd d = dw[c];
                d.x -= v.x;
                d.y += v.y;
                dw[c] = d;
            } else {
                cd& a = A[(size_t)r + (size_t)c * ld];
                a.x -= v.x;
                a.y -= v.y;
            }
        }
    }
}

static bool g_ldl_attr = false;

int ldlh_factor(Ctx& c, int m0, int n)
{
    if (m0 < 0 || m0 > n || n > c.ld) return -1;
    if (m0 > c.fact_n) return -1;
    if (!g_ldl_attr) {
        cudaFuncSetAttribute(k_ldl_diag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * LDL_NB * DG_LD * sizeof(double2)));
        cudaFuncSetAttribute(k_ldl_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * LDL_NB * LDL_NB * sizeof(double2)));
        cudaFuncSetAttribute(k_ldl_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(2 * UPD_KC * UPD_LD * sizeof(double2)));
        g_ldl_attr = true;
    }
    const size_t upd_sm = 2 * UPD_KC * UPD_LD * sizeof(double2);
    // block list: existing blocks truncated at m0, then new 64-row blocks
    std::vector<int> starts;
    for (int s : c.blk_start)
        if (s < m0) starts.push_back(s);
    const int nexist = (int)starts.size();
    for (int s = m0; s < n; s += LDL_NB) starts.push_back(s);
    const int nblk = (int)starts.size();
    auto blk_end = [&](int i) {
        if (i + 1 < nblk) return starts[i + 1];
        return n;
    };
    if (n > m0) {
        const int ct0 = m0 / 32, ct1 = (n + 31) / 32;
        dim3 g(ct1 - ct0, ct1);
        k_ldl_mirror<<<g, 256, 0, c.stream>>>(c.H, c.ld, m0, n, c.dw, ct0);
        c.launches++;
    }
    const size_t sm2 = 2 * LDL_NB * LDL_NB * sizeof(double2);
    for (int i = 0; i < nblk; i++) {
        const int p0 = starts[i];
        const int p1 = (i < nexist) ? std::min(blk_end(i), m0) : blk_end(i);
        if (p1 <= p0) continue;
        const bool existing = (i < nexist);
        if (!existing) {
            k_ldl_diag<<<1, 256, 2 * LDL_NB * DG_LD * sizeof(double2), c.stream>>>(c.H, c.ld, p0, p1, c.dw, c.invD,
                                                                                   c.linv, c.status);
            c.launches++;
        }
        const int clo = existing ? m0 : p1;
        if (clo >= n) continue;
        const int ncb = (n - clo + LDL_NB - 1) / LDL_NB;
        k_ldl_trsm<<<ncb, 256, sm2, c.stream>>>(c.H, c.ld, p0, p1, clo, n, c.invD, c.linv, c.vbuf);
        c.launches++;
        const int nrb = (n - p1 + LDL_NB - 1) / LDL_NB;
        dim3 g(ncb, nrb);
        k_ldl_update<<<g, 256, upd_sm, c.stream>>>(c.H, c.ld, p0, p1, p1, clo, n, c.vbuf, c.dw);
        c.launches++;
    }
    if (cudaGetLastError() != cudaSuccess) return -2;
    c.blk_start = starts;
    c.fact_n = n;
    // panel boundaries for the cooperative solves (starts..., n)
    std::vector<int> bounds(starts);
    bounds.push_back(n);
    if (cudaMemcpyAsync(c.dblk, bounds.data(), bounds.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream) !=
        cudaSuccess)
        return -2;
    return 0;
}

}  // namespace ecg
