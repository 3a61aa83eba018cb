// invit.cu -- one inverse-iteration step and the Rayleigh quotient of
// GHEPIIS (src/linalg.f90:1781-1926):
//   w = B^H v                  MHMV, ZGEMV('C')         (src/linalg.f90:1019-1107)
//   x = (L D L^H)^-1 w         LDLHS, 2 x ZTRSV + D^-1  (src/linalg.f90:618-775)
//   x /= max|Re x|,|Im x|      CMaxAbsReOrIm + CVScale
//   tc = x^H v / v^H v, NormOfDiff = sqrt(2n) ||x - tc v||
//   t1 = x^H B x, t2 = x^H M x VMMHMV on the lower triangles
//
// The triangular solves walk the panels of the LDL^H factor.  Each panel
// step is one launch whose CTAs share the dot products against the already
// solved part; the last CTA to finish (atomic ticket, no waiting) sums the
// partials in a fixed order and applies the panel's precomputed inverse
// block, so results are deterministic run to run.
#include <algorithm>
#include "ecg_internal.h"

namespace ecg {

constexpr int SOLVE_G_MAX = 64;

__device__ __forceinline__ cd ld2(const cd* p)
{
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}
__device__ __forceinline__ cd ldcg2(const cd* p)
{
    const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}
__device__ __forceinline__ cd warp_sum(cd s)
{
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    return s;
}

// w(i) = sum_j conj(B(j,i)) v(j); one warp per column, four accumulators.
__global__ void __launch_bounds__(256) k_hemv(const cd* __restrict__ B, int ld, int n, const cd* __restrict__ v,
                                              cd* __restrict__ w)
{
    const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (col >= n) return;
    const cd* b = B + (size_t)col * ld;
    cd s0 = mk(0.0, 0.0), s1 = s0, s2 = s0, s3 = s0;
    int j = lane;
    for (; j + 96 < n; j += 128) {
        const cd b0 = ld2(b + j), b1 = ld2(b + j + 32), b2 = ld2(b + j + 64), b3 = ld2(b + j + 96);
        s0 = cfma(conj(b0), ld2(v + j), s0);
        s1 = cfma(conj(b1), ld2(v + j + 32), s1);
        s2 = cfma(conj(b2), ld2(v + j + 64), s2);
        s3 = cfma(conj(b3), ld2(v + j + 96), s3);
    }
    for (; j < n; j += 32) s0 = cfma(conj(ld2(b + j)), ld2(v + j), s0);
    const cd s = warp_sum((s0 + s1) + (s2 + s3));
    if (lane == 0) w[col] = s;
}

// Forward solve of panel [j0, j1): y = Linv (w - U(0:j0, p)^H y(0:j0)),
// z = invD y.  CTA g covers rows [g*chunk, ...) of the solved part.
__global__ void __launch_bounds__(256) k_fwd(const cd* __restrict__ A, int ld, int j0, int j1, int chunk,
                                             const cd* __restrict__ w, cd* __restrict__ y, cd* __restrict__ z,
                                             const cd* __restrict__ invD, const cd* __restrict__ linv,
                                             cd* __restrict__ part, int* __restrict__ counter)
{
    __shared__ cd t[LDL_NB];
    __shared__ int last;
    const int b = j1 - j0;
    const int g = blockIdx.x, G = gridDim.x;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const int i0 = g * chunk, i1 = min(j0, i0 + chunk);
    for (int m = wp; m < b; m += 8) {
        const cd* col = A + (size_t)(j0 + m) * ld;
        cd s = mk(0.0, 0.0);
        for (int i = i0 + lane; i < i1; i += 32) s = cfma(conj(ld2(col + i)), ldcg2(y + i), s);
        s = warp_sum(s);
        if (lane == 0) part[g * LDL_NB + m] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1) == G - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < b) {
        cd s = mk(0.0, 0.0);
        for (int q = 0; q < G; q++) s = s + ldcg2(part + q * LDL_NB + threadIdx.x);
        t[threadIdx.x] = ld2(w + j0 + threadIdx.x) - s;
    }
    __syncthreads();
    if (threadIdx.x < b) {
        const int r = threadIdx.x;
        const cd* Lr = linv + (size_t)(j0 + r) * LDL_NB;
        cd s = mk(0.0, 0.0);
        for (int q = 0; q <= r; q++) s = cfma(ld2(Lr + q), t[q], s);
        y[j0 + r] = s;
        z[j0 + r] = cmul(s, ld2(invD + j0 + r));
    }
    if (threadIdx.x == 0) *counter = 0;
}

// Backward solve of panel [j0, j1): x = Linv^H (z - U(p, j1:n) x(j1:n)).
// CTA g covers columns [j1 + g*chunk, ...); 4 groups of 64 threads.
__global__ void __launch_bounds__(256) k_bwd(const cd* __restrict__ A, int ld, int j0, int j1, int n, int chunk,
                                             const cd* __restrict__ z, cd* __restrict__ x,
                                             const cd* __restrict__ linv, cd* __restrict__ part,
                                             int* __restrict__ counter)
{
    __shared__ cd sred[4][LDL_NB];
    __shared__ cd t[LDL_NB];
    __shared__ int last;
    const int b = j1 - j0;
    const int g = blockIdx.x, G = gridDim.x;
    const int r = threadIdx.x & 63, grp = threadIdx.x >> 6;
    const int c0 = j1 + g * chunk, c1 = min(n, c0 + chunk);
    cd s = mk(0.0, 0.0);
    if (r < b)
        for (int c = c0 + grp; c < c1; c += 4) s = cfma(ld2(A + (size_t)(j0 + r) + (size_t)c * ld), ldcg2(x + c), s);
    sred[grp][r] = s;
    __syncthreads();
    if (threadIdx.x < LDL_NB) {
        const cd v = (sred[0][r] + sred[1][r]) + (sred[2][r] + sred[3][r]);
        part[g * LDL_NB + r] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1) == G - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < b) {
        cd q = mk(0.0, 0.0);
        for (int k = 0; k < G; k++) q = q + ldcg2(part + k * LDL_NB + threadIdx.x);
        t[threadIdx.x] = ld2(z + j0 + threadIdx.x) - q;
    }
    __syncthreads();
    if (threadIdx.x < b) {
        const int rr = threadIdx.x;
        cd v = mk(0.0, 0.0);
        for (int q = rr; q < b; q++) v = cfma(conj(ld2(linv + (size_t)(j0 + q) * LDL_NB + rr)), t[q], v);
        x[j0 + rr] = v;
    }
    if (threadIdx.x == 0) *counter = 0;
}

// ---------------------------------------------------------------------------
// Cooperative triangular solves: one CTA per LDL^H panel, all CTAs
// co-resident (cooperative launch).  CTA j accumulates the contributions of
// the panels it depends on in panel order, each as soon as that panel's
// flag carries the current epoch (acquire / release), then applies its
// inverse diagonal block and publishes its own panel.  The neighbouring
// panel (j-1 forward, j+1 backward) is left out of that sum: its term is
// applied after the inverse block as one 64 x 64 product with the
// precomputed M_j = Linv_j U(j-1, j)^H or N_j = Linv_j^H U(j, j+1)
// (k_ldl_mn), so the step from one panel's flag to the next is that
// product alone.  Every wait is
// bounded: after SOLVE_SPIN_LIMIT polls, or as soon as any CTA has given
// up (the abort word), the CTA records ST_SOLVE_TIMEOUT and finishes
// without waiting; the host then reports the step as failed.
static_assert(SOLVE_SPIN_LIMIT == (1 << 22), "the default poll limit of the solves' waits");
constexpr int LS_LD = LDL_NB + 1;

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait (thread 0) for flags[a] == epoch; returns false if this CTA must stop.
// abort_word[1] holds the poll limit (SOLVE_SPIN_LIMIT unless a caller set
// another through ecg_set_wait_limit).
__device__ __forceinline__ bool wait_panel(const unsigned* flags, int a, unsigned epoch, int* status, int* abort_word,
                                           bool& ok)
{
    __shared__ int go;
    if (threadIdx.x == 0) {
        int g = 1;
        if (ok) {
            int spins = 0;
            const int limit = ((volatile int*)abort_word)[1];
            while (ld_acquire(flags + a) != epoch) {
                if (++spins > limit || *((volatile int*)abort_word) != 0) {
                    g = 0;
                    break;
                }
            }
            if (!g) {
                atomicExch(status + ST_SOLVE_TIMEOUT, 1);
                atomicExch(abort_word, 1);
            }
        } else {
            g = 0;
        }
        go = g;
    }
    __syncthreads();
    ok = ok && go;
    return ok;
}

// Rows [j0, j0 + b) of a per-panel 64-column block (linv, lmf, lnb) into
// Ls[r][q] for q < bq, zeros elsewhere.
__device__ __forceinline__ void load_linv(const cd* __restrict__ linv, int j0, int b, double2* Ls, int bq = -1)
{
    if (bq < 0) bq = b;
    for (int e = threadIdx.x; e < LDL_NB * LDL_NB; e += blockDim.x) {
        const int r = e / LDL_NB, q = e % LDL_NB;
        double2 v = make_double2(0.0, 0.0);
        if (r < b && q < bq) {
            const cd a = ld2(linv + (size_t)(j0 + r) * LDL_NB + q);
            v = make_double2(a.x, a.y);
        }
        Ls[r * LS_LD + q] = v;
    }
}

// Forward: y_j = Linv_j (w_j - sum_{a<j} U(a, j)^H y_a), z_j = invD_j y_j.
template <bool NEIGH>
__global__ void __launch_bounds__(256) k_fwd_coop(const cd* __restrict__ A, int ld, const int* __restrict__ bstart,
                                                  int nb, const cd* __restrict__ w, cd* __restrict__ y,
                                                  cd* __restrict__ z, const cd* __restrict__ invD,
                                                  const cd* __restrict__ linv, const cd* __restrict__ lmf,
                                                  unsigned* __restrict__ flags, unsigned epoch,
                                                  int* __restrict__ status, int* abort_word)
{
    extern __shared__ double2 sm[];
    double2* Ls = sm;                          // Linv_j, [r][q]
    double2* red = sm + LDL_NB * LS_LD;        // [8][64] warp partials, then [4][64]
    double2* Ms = red + 8 * LDL_NB;            // NEIGH: M_j, [r][q]
    __shared__ double2 t[LDL_NB];
    const int j = blockIdx.x;
    const int j0 = bstart[j], j1 = bstart[j + 1], b = j1 - j0;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    load_linv(linv, j0, b, Ls);
    if (NEIGH && j > 0) load_linv(lmf, j0, b, Ms, j0 - bstart[j - 1]);
    // this panel's right-hand side and pivots, read before the waits
    const cd wj = (threadIdx.x < b) ? ld2(w + j0 + threadIdx.x) : mk(0.0, 0.0);
    const cd dj = (threadIdx.x < b) ? ld2(invD + j0 + threadIdx.x) : mk(0.0, 0.0);
    // lane-partials for the 8 columns this warp owns
    cd acc[8];
#pragma unroll
    for (int m = 0; m < 8; m++) acc[m] = mk(0.0, 0.0);
    bool ok = true;
    // every panel but the previous one; that one comes in below through
    // M_j = Linv_j U(j-1, j)^H
    const int alast = NEIGH ? j - 1 : j;
    for (int a = 0; a < alast; a++) {
        const int a0 = bstart[a], a1 = bstart[a + 1];
        const int r0 = a0 + lane, r1 = a0 + lane + 32;
        // the factor block U(panel a, panel j) does not depend on panel a's
        // solution: load it before waiting for that panel's flag
        cd u0[8], u1[8];
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int c = wp * 8 + m;
            const cd* col = A + (size_t)(j0 + c) * ld;
            u0[m] = (c < b && r0 < a1) ? ld2(col + r0) : mk(0.0, 0.0);
            u1[m] = (c < b && r1 < a1) ? ld2(col + r1) : mk(0.0, 0.0);
        }
        if (!wait_panel(flags, a, epoch, status, abort_word, ok)) break;
        const cd y0 = (r0 < a1) ? ldcg2(y + r0) : mk(0.0, 0.0);
        const cd y1 = (r1 < a1) ? ldcg2(y + r1) : mk(0.0, 0.0);
#pragma unroll
        for (int m = 0; m < 8; m++) {
            acc[m] = cfma(conj(u0[m]), y0, acc[m]);
            acc[m] = cfma(conj(u1[m]), y1, acc[m]);
        }
    }
#pragma unroll
    for (int m = 0; m < 8; m++) acc[m] = warp_sum(acc[m]);
    if (lane == 0)
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int c = wp * 8 + m;
            if (c < b) t[c] = make_double2(0.0, 0.0), red[c] = make_double2(acc[m].x, acc[m].y);
        }
    __syncthreads();
    if (threadIdx.x < b) {
        const cd s = mk(red[threadIdx.x].x, red[threadIdx.x].y);
        const cd v = wj - s;
        t[threadIdx.x] = make_double2(v.x, v.y);
    }
    __syncthreads();
    // y = Ls t: row r = tid & 63, four interleaved partial sums over q
    {
        const int r = threadIdx.x & 63, g = threadIdx.x >> 6;
        cd s = mk(0.0, 0.0);
        if (r < b)
            for (int q = g; q <= r; q += 4) {
                const double2 l = Ls[r * LS_LD + q], tq = t[q];
                s = cfma(mk(l.x, l.y), mk(tq.x, tq.y), s);
            }
        red[g * LDL_NB + r] = make_double2(s.x, s.y);
    }
    __syncthreads();
    cd ys = mk(0.0, 0.0);
    if (threadIdx.x < b) {
        const int r = threadIdx.x;
#pragma unroll
        for (int g = 0; g < 4; g++) ys = ys + mk(red[g * LDL_NB + r].x, red[g * LDL_NB + r].y);
    }
    if (NEIGH && j > 0) {
        // y_j -= M_j y_{j-1}: row r = tid & 63, columns g, g + 4, ...
        const int a0 = bstart[j - 1], bp = j0 - a0;
        const int r = threadIdx.x & 63, g = threadIdx.x >> 6;
        // (the barrier inside also orders the reads of red above before the writes below)
        if (wait_panel(flags, j - 1, epoch, status, abort_word, ok)) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int q = g + 4 * i;
                if (q < bp) {
                    const double2 m = Ms[r * LS_LD + q];
                    s = cfma(mk(m.x, m.y), ldcg2(y + a0 + q), s);
                }
            }
            red[g * LDL_NB + r] = make_double2(s.x, s.y);
        }
        __syncthreads();
        if (ok && threadIdx.x < b) {
            const int rr = threadIdx.x;
#pragma unroll
            for (int g2 = 0; g2 < 4; g2++) ys = ys - mk(red[g2 * LDL_NB + rr].x, red[g2 * LDL_NB + rr].y);
        }
    }
    if (threadIdx.x < b) {
        y[j0 + threadIdx.x] = ys;
        z[j0 + threadIdx.x] = cmul(ys, dj);
    }
    // the release by thread 0 after the barrier publishes every thread's
    // stores above (cumulativity of the gpu-scope release)
    __syncthreads();
    if (threadIdx.x == 0) st_release(flags + j, epoch);
}

// Backward: x_j = Linv_j^H (z_j - sum_{c>j} U(j, c) x_c).
template <bool NEIGH>
__global__ void __launch_bounds__(256) k_bwd_coop(const cd* __restrict__ A, int ld, const int* __restrict__ bstart,
                                                  int nb, const cd* __restrict__ z, cd* __restrict__ x,
                                                  const cd* __restrict__ linv, const cd* __restrict__ lnb,
                                                  unsigned* __restrict__ flags, unsigned epoch,
                                                  int* __restrict__ status, int* abort_word)
{
    extern __shared__ double2 sm[];
    double2* Ls = sm;
    double2* red = sm + LDL_NB * LS_LD;  // [8][64]
    double2* Ns = red + 8 * LDL_NB;      // NEIGH: N_j, [r][q]
    __shared__ double2 t[LDL_NB];
    const int j = blockIdx.x;
    const int j0 = bstart[j], j1 = bstart[j + 1], b = j1 - j0;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    load_linv(linv, j0, b, Ls);
    if (NEIGH && j + 1 < nb) load_linv(lnb, j0, b, Ns, bstart[j + 2] - j1);
    const cd zj = (threadIdx.x < b) ? ld2(z + j0 + threadIdx.x) : mk(0.0, 0.0);  // read before the waits
    cd a0 = mk(0.0, 0.0), a1 = mk(0.0, 0.0);  // rows lane, lane + 32
    bool ok = true;
    // every later panel but the next one; that one comes in below through
    // N_j = Linv_j^H U(j, j+1)
    const int clast = NEIGH ? j + 1 : j;
    for (int c = nb - 1; c > clast; c--) {
        const int c0 = bstart[c], c1 = bstart[c + 1];
        // U(panel j, panel c) before the wait for panel c's solution
        cd u0[8], u1[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int col = c0 + wp + 8 * i;
            const cd* u = A + (size_t)col * ld + j0;
            u0[i] = (col < c1 && lane < b) ? ld2(u + lane) : mk(0.0, 0.0);
            u1[i] = (col < c1 && lane + 32 < b) ? ld2(u + lane + 32) : mk(0.0, 0.0);
        }
        if (!wait_panel(flags, c, epoch, status, abort_word, ok)) break;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int col = c0 + wp + 8 * i;
            const cd xc = (col < c1) ? ldcg2(x + col) : mk(0.0, 0.0);
            a0 = cfma(u0[i], xc, a0);
            a1 = cfma(u1[i], xc, a1);
        }
    }
    red[wp * LDL_NB + lane] = make_double2(a0.x, a0.y);
    red[wp * LDL_NB + lane + 32] = make_double2(a1.x, a1.y);
    __syncthreads();
    if (threadIdx.x < b) {
        const int r = threadIdx.x;
        cd s = mk(0.0, 0.0);
#pragma unroll
        for (int q = 0; q < 8; q++) s = s + mk(red[q * LDL_NB + r].x, red[q * LDL_NB + r].y);
        const cd v = zj - s;
        t[r] = make_double2(v.x, v.y);
    }
    __syncthreads();
    {
        const int r = threadIdx.x & 63, g = threadIdx.x >> 6;
        cd s = mk(0.0, 0.0);
        if (r < b)
            for (int q = r + g; q < b; q += 4) {
                const double2 l = Ls[q * LS_LD + r], tq = t[q];
                s = cfma(conj(mk(l.x, l.y)), mk(tq.x, tq.y), s);
            }
        red[g * LDL_NB + r] = make_double2(s.x, s.y);
    }
    __syncthreads();
    cd xs = mk(0.0, 0.0);
    if (threadIdx.x < b) {
        const int r = threadIdx.x;
#pragma unroll
        for (int g = 0; g < 4; g++) xs = xs + mk(red[g * LDL_NB + r].x, red[g * LDL_NB + r].y);
    }
    if (NEIGH && j + 1 < nb) {
        // x_j -= N_j x_{j+1}: row r = tid & 63, columns g, g + 4, ...
        const int c0 = bstart[j + 1], bn = bstart[j + 2] - c0;
        const int r = threadIdx.x & 63, g = threadIdx.x >> 6;
        if (wait_panel(flags, j + 1, epoch, status, abort_word, ok)) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int i = 0; i < 16; i++) {
                const int q = g + 4 * i;
                if (q < bn) {
                    const double2 m = Ns[r * LS_LD + q];
                    s = cfma(mk(m.x, m.y), ldcg2(x + c0 + q), s);
                }
            }
            red[g * LDL_NB + r] = make_double2(s.x, s.y);
        }
        __syncthreads();
        if (ok && threadIdx.x < b) {
            const int rr = threadIdx.x;
#pragma unroll
            for (int g2 = 0; g2 < 4; g2++) xs = xs - mk(red[g2 * LDL_NB + rr].x, red[g2 * LDL_NB + rr].y);
        }
    }
    if (threadIdx.x < b) x[j0 + threadIdx.x] = xs;
    __syncthreads();
    if (threadIdx.x == 0) st_release(flags + j, epoch);
}

// Block-wide deterministic sums (1024 threads).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh)
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
        for (int q = 0; q < 32; q++) s += sh[q * NV + k];
        v[k] = s;
    }
}

// Normalisation and convergence measure of one step; ends with v <- x.
__global__ void __launch_bounds__(1024) k_iter_norm(int n, cd* __restrict__ x, cd* __restrict__ v, double sqrtn,
                                                    double* __restrict__ red)
{
    __shared__ double sh[32 * 3];
    __shared__ double smax[32];
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    double m = 0.0;
    for (int j = tid; j < n; j += 1024) {
        const cd a = x[j];
        m = fmax(m, fmax(fabs(a.x), fabs(a.y)));
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) smax[wp] = m;
    __syncthreads();
    double t1 = 0.0;
    for (int q = 0; q < 32; q++) t1 = fmax(t1, smax[q]);
    const double ra = 1.0 / t1;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = tid; j < n; j += 1024) {
        cd a = x[j];
        a = cd{ra * a.x, ra * a.y};
        x[j] = a;
        const cd b = v[j];
        acc[0] = fma(a.x, b.x, fma(a.y, b.y, acc[0]));   // Re conj(x) v
        acc[1] = fma(a.x, b.y, fma(-a.y, b.x, acc[1]));  // Im conj(x) v
        acc[2] = fma(b.x, b.x, fma(b.y, b.y, acc[2]));
    }
    block_sum<3>(acc, sh);
    const cd tc = cd{acc[0] / acc[2], acc[1] / acc[2]};
    double d[1] = {0.0};
    for (int j = tid; j < n; j += 1024) {
        const cd a = x[j];
        const cd s = cfms(tc, v[j], a);
        d[0] = fma(s.x, s.x, fma(s.y, s.y, d[0]));
    }
    __syncthreads();
    block_sum<1>(d, sh);
    if (tid == 0) red[RD_NORMDIFF] = sqrtn * sqrt(d[0]);
    __syncthreads();
    for (int j = tid; j < n; j += 1024) v[j] = x[j];
}

// Per-column terms of x^H A x over the lower triangle (VMMHMV,
// src/linalg.f90:1195-1206) for A = B (blockIdx.y = 0) and A = M (1).
__global__ void __launch_bounds__(256) k_vmm_cols(const cd* __restrict__ B, const cd* __restrict__ M, int ld, int n,
                                                  const cd* __restrict__ x, double* __restrict__ colval)
{
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= n) return;
    const cd* A = (blockIdx.y == 0) ? B : M;
    const cd* col = A + (size_t)k * ld;
    double sr = 0.0, si = 0.0;
    for (int j = k + 1 + lane; j < n; j += 32) {
        const cd a = ld2(col + j), xj = ld2(x + j);
        sr = fma(xj.x, a.x, fma(xj.y, a.y, sr));
        si = fma(xj.y, a.x, fma(-xj.x, a.y, si));
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        const cd xk = ld2(x + k);
        const double dk = ld2(col + k).x;
        colval[(size_t)blockIdx.y * n + k] = fma(xk.x * xk.x + xk.y * xk.y, dk, 2.0 * (xk.x * sr + xk.y * si));
    }
}

__global__ void __launch_bounds__(1024) k_vmm_reduce(int n, const double* __restrict__ colval,
                                                     const cd* __restrict__ x, double* __restrict__ red)
{
    __shared__ double sh[32 * 3];
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = threadIdx.x; j < n; j += 1024) {
        acc[0] += colval[j];
        acc[1] += colval[n + j];
        const cd a = x[j];
        acc[2] = fma(a.x, a.x, fma(a.y, a.y, acc[2]));
    }
    block_sum<3>(acc, sh);
    if (threadIdx.x == 0) {
        red[RD_T1] = acc[0];
        red[RD_T2] = acc[1];
        red[RD_XX] = acc[2];
    }
}

__global__ void k_vec_scale(cd* __restrict__ v, int n, double s)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        const cd a = v[j];
        v[j] = cd{s * a.x, s * a.y};
    }
}

// ---------------------------------------------------------------------------
// Shared memory of the cooperative solves: the inverse diagonal block, the
// partial sums and, with NEIGH, the neighbour product M_j / N_j.
static size_t coop_smem(bool neigh)
{
    return (size_t)(LDL_NB * LS_LD + 8 * LDL_NB + (neigh ? LDL_NB * LS_LD : 0)) * sizeof(double2);
}

template <bool NEIGH>
static int coop_blocks(int dev)
{
    const int sm = (int)coop_smem(NEIGH);
    cudaFuncSetAttribute(k_fwd_coop<NEIGH>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_bwd_coop<NEIGH>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    int coop = 0, nsm = 0, per1 = 0, per2 = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, k_fwd_coop<NEIGH>, 256, sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_bwd_coop<NEIGH>, 256, sm);
    cudaGetLastError();
    return coop ? nsm * std::min(per1, per2) : -1;
}

// Largest grid the cooperative solves may use on this device (-1: none),
// without and with the neighbour products.
static int coop_capacity(Ctx& c, bool neigh)
{
    if (!c.coop_max_blocks) {
        c.coop_max_blocks = coop_blocks<false>(c.dev);
        c.coop_max_neigh = coop_blocks<true>(c.dev);
    }
    return neigh ? c.coop_max_neigh : c.coop_max_blocks;
}

static int solve_multi_launch(Ctx& c, int n)
{
    const int nb = (int)c.blk_start.size();
    for (int i = 0; i < nb; i++) {
        const int j0 = c.blk_start[i], j1 = (i + 1 < nb) ? c.blk_start[i + 1] : n;
        int G = (j0 + 127) / 128;
        G = G < 1 ? 1 : (G > SOLVE_G_MAX ? SOLVE_G_MAX : G);
        const int chunk = (j0 + G - 1) / G;
        k_fwd<<<G, 256, 0, c.stream>>>(c.F, c.ld, j0, j1, chunk > 0 ? chunk : 1, c.w, c.yv, c.zv, c.invD, c.linv,
                                      c.spart, c.counters);
        c.launches++;
    }
    for (int i = nb - 1; i >= 0; i--) {
        const int j0 = c.blk_start[i], j1 = (i + 1 < nb) ? c.blk_start[i + 1] : n;
        const int rest = n - j1;
        int G = (rest + 127) / 128;
        G = G < 1 ? 1 : (G > SOLVE_G_MAX ? SOLVE_G_MAX : G);
        const int chunk = (rest + G - 1) / G;
        k_bwd<<<G, 256, 0, c.stream>>>(c.F, c.ld, j0, j1, n, chunk > 0 ? chunk : 1, c.zv, c.x, c.linv, c.spart,
                                      c.counters + 1);
        c.launches++;
    }
    return 0;
}

static int solve_cooperative(Ctx& c, int n, bool neigh)
{
    int nb = (int)c.blk_start.size();
    const size_t sm = coop_smem(neigh);
    int* abort_word = c.counters + 2;
    if (cudaMemsetAsync(abort_word, 0, sizeof(int), c.stream) != cudaSuccess) return -2;
    const int* bs = c.dblk;
    const cd* H = c.F;
    const cd* w = c.w;
    const cd* invD = c.invD;
    const cd* linv = c.linv;
    const cd* lmf = c.lmf;
    const cd* lnb = c.lnb;
    int ld = c.ld;
    const void* kf = neigh ? (const void*)k_fwd_coop<true> : (const void*)k_fwd_coop<false>;
    const void* kb = neigh ? (const void*)k_bwd_coop<true> : (const void*)k_bwd_coop<false>;
    unsigned e1 = ++c.epoch;
    void* a1[] = {(void*)&H, &ld, (void*)&bs, &nb, (void*)&w, &c.yv, &c.zv, (void*)&invD, (void*)&linv, (void*)&lmf,
                  &c.flags, &e1, &c.status, &abort_word};
    if (cudaLaunchCooperativeKernel(kf, nb, 256, a1, sm, c.stream) != cudaSuccess) return -2;
    unsigned e2 = ++c.epoch;
    const cd* zv = c.zv;
    void* a2[] = {(void*)&H, &ld, (void*)&bs, &nb, (void*)&zv, &c.x, (void*)&linv, (void*)&lnb, &c.flags, &e2,
                  &c.status, &abort_word};
    if (cudaLaunchCooperativeKernel(kb, nb, 256, a2, sm, c.stream) != cudaSuccess) return -2;
    c.launches += 2;
    return 0;
}

int invit_step(Ctx& c, int n, bool /*first*/)
{
    k_hemv<<<(n * 32 + 255) / 256, 256, 0, c.stream>>>(c.S, c.ld, n, c.c, c.w);
    c.launches++;
    const int nb = (int)c.blk_start.size();
    // the neighbour products take a second 64 x 64 block of shared memory
    // (one CTA per SM): used while every panel still has an SM of its own
    int r;
    if (nb <= coop_capacity(c, true))
        r = solve_cooperative(c, n, true);
    else if (nb <= coop_capacity(c, false))
        r = solve_cooperative(c, n, false);
    else
        r = solve_multi_launch(c, n);
    if (r) return r;
    k_iter_norm<<<1, 1024, 0, c.stream>>>(n, c.x, c.c, sqrt(2.0 * n), c.red);
    c.launches++;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int invit_rayleigh(Ctx& c, int n)
{
    dim3 g((n * 32 + 255) / 256, 2);
    k_vmm_cols<<<g, 256, 0, c.stream>>>(c.S, c.F, c.ld, n, c.x, c.colval);
    k_vmm_reduce<<<1, 1024, 0, c.stream>>>(n, c.colval, c.x, c.red);
    c.launches += 2;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int vec_scale(Ctx& c, cd* v, int n, double s)
{
    k_vec_scale<<<(n + 255) / 256, 256, 0, c.stream>>>(v, n, s);
    c.launches++;
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // namespace ecg
