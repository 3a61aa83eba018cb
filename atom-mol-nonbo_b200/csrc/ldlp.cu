// ldlp.cu -- LDL^H factorisation of a whole matrix (no existing rows) as one
// persistent cooperative kernel over 64 x 64 tiles, the drop-in for LDLHF
// with m = 1 (src/linalg.f90:316-455).
//
// Same storage contract and recurrence as ldlh.cu: M's lower triangle is left
// untouched, the strict upper triangle receives L^H, invD receives 1/d; the
// working Schur complement W(r, c), r < c, lives in the upper triangle and
// its diagonal in dw.  The factorisation is split into tasks on 64 x 64 tiles
// (R, C), R <= C, of panel index s:
//   D(s)        eliminate the diagonal tile (s, s): U_ss, invD, pivots d_s
//               (written to dw over the consumed working diagonal);
//   T(s, C)     panel rows of tile (s, C): U(s, C) = invD L_ss^-1 W(s, C);
//   B(s, R, C)  W(R, C) -= conj(U(s, R))^T diag(d_s) U(s, C), s < R <= C
//               (the unscaled rows of the reference's recurrence, d U, are
//               formed in registers from U and d instead of being stored).
// Every tile has a counter: the number of panels applied to it (D and T set
// it to s + 1 when the tile is final).  A task waits (bounded) until its
// tiles carry the counts it needs:
//   D(s): cnt(s,s) >= s;  T(s,C): cnt(s,s) >= s+1, cnt(s,C) >= s;
//   B(s,R,C): cnt(s,R) >= s+1, cnt(s,C) >= s+1, cnt(R,C) >= s.
// CTA 0, alone on its SM, runs the chain D(s) -> T(s, s+1) -> B(s, s+1,
// s+1) -> D(s+1) with the diagonal tile kept in shared memory.  The other
// CTAs (all co-resident: cooperative launch) take every other task from a
// list in a fixed order through one atomic counter; an update whose next
// panels are already final applies them too (rank up to 256).  The list is
// a topological order of the dependency graph, made on the host by list
// scheduling on as many simulated workers as the grid has CTAs, always
// starting the ready task with the longest remaining path (upward rank).
// Because every task's dependencies come earlier in that order (the chain's
// included) and every CTA is resident, the earliest unfinished task can
// always proceed: the kernel cannot deadlock.  Waits are still bounded (the
// poll limit of ecg_set_wait_limit); a CTA that gives up records
// ST_SOLVE_TIMEOUT and sets the abort word, after which every CTA stops
// taking tasks.  The kernel's code is kept compact (loops that are not
// unrolled where unrolling gained nothing): the chain's per-panel loop has
// to stay in the instruction cache, and a larger form measured D(s) at 42
// instead of 21 us.
#include <algorithm>
#include <queue>
#include <utility>
#include <vector>
#include "ecg_internal.h"
#include "zmma.cuh"

namespace ecg {

constexpr unsigned LP_D = 0, LP_T = 1, LP_B = 2;
constexpr unsigned LP_NONE = 0xffffffffu;
constexpr int LP_KC = 16;          // k rows per cp.async stage of an update
constexpr int LP_P = 66;           // pitch (double2) of the staged operands: 2 mod 8, conflict-free fragments
constexpr int LP_ST = 3;           // stages
constexpr int LP_LD = LDL_NB + 1;  // pitch of the 64 x 64 shared tiles of D and T
constexpr int LP_SUB = 8;          // sub-panel rows of the diagonal elimination
constexpr int LP_MERGE = 4;        // most panels one trailing update applies at once
constexpr size_t LP_SMEM_B = (size_t)(LP_ST * LP_KC * 2 * LP_P + LP_MERGE * LDL_NB) * sizeof(double2);

__host__ __device__ __forceinline__ unsigned lp_code(unsigned type, int s, int R, int C, unsigned half = 0)
{
    return type << 30 | half << 29 | (unsigned)s << 20 | (unsigned)R << 10 | (unsigned)C;
}
// The updates of the two tile rows after panel s (the band the diagonal
// chain waits on), except the chain's own B(s, s+1, s+1), run as two tasks
// on the column halves of the tile, so each takes half the time on its SM.
__host__ __device__ __forceinline__ bool lp_split(int s, int R, int C)
{
    return R <= s + 2 && !(R == s + 1 && C == s + 1);
}
// counter of tile (R, C), R <= C: column-wise packed triangle
__host__ __device__ __forceinline__ long long lp_tix(int R, int C) { return (long long)C * (C + 1) / 2 + R; }

// ---------------------------------------------------------------------------
// Host: the task list.
// ---------------------------------------------------------------------------
// Task weights (us) for the list scheduler: the time a CTA is held by a
// task on a B200 with two CTAs per SM, waits and merged updates included
// (globaltimer records of ecg_factor_trace); a split update counts half.
// Only the ratios matter: at K = 4000 this set measured 4.82 ms, the raw
// run times (21, 24, 24, 15) 5.0 ms, and a T weighted above B 5.1-5.2 ms.
struct LpCost {
    double d = 21.0, t = 40.0, b = 60.0, bd = 40.0;
};

// Tasks of a factorisation with np panels: the list the P CTAs other than
// the chain CTA take, and (if full is given) every task in the simulated
// start order, the chain's included.
static void lp_schedule(int np, int P, const LpCost& cost, std::vector<unsigned>& list,
                        std::vector<unsigned>* full = nullptr)
{
    std::vector<unsigned> code;
    std::vector<long long> idD(np);
    std::vector<long long> idT((size_t)np * np, -1);
    std::vector<long long> idB((size_t)np * np * np, -1);  // first node of B(s, R, C)
    auto bix = [&](int s, int R, int C) -> size_t { return ((size_t)s * np + R) * np + C; };
    for (int s = 0; s < np; s++) {
        idD[s] = (long long)code.size();
        code.push_back(lp_code(LP_D, s, s, s));
        for (int C = s + 1; C < np; C++) {
            idT[(size_t)s * np + C] = (long long)code.size();
            code.push_back(lp_code(LP_T, s, s, C));
        }
        for (int R = s + 1; R < np; R++)
            for (int C = R; C < np; C++) {
                idB[bix(s, R, C)] = (long long)code.size();
                code.push_back(lp_code(LP_B, s, R, C));
                if (lp_split(s, R, C)) code.push_back(lp_code(LP_B, s, R, C, 1));  // the second column half
            }
    }
    const long long N = (long long)code.size();
    // predecessors in creation order, which is topological: an update that
    // is split in two column halves counts as both halves
    constexpr int NPRED = 6;
    std::vector<long long> pred((size_t)N * NPRED, -1);
    std::vector<double> w((size_t)N);
    for (long long t = 0; t < N; t++) {
        const unsigned c = code[t];
        const int type = c >> 30, s = (c >> 20) & 511, R = (c >> 10) & 1023, C = c & 1023;
        long long* p = &pred[(size_t)t * NPRED];
        int k = 0;
        auto addB = [&](int s2, int R2, int C2) {
            const long long b = idB[bix(s2, R2, C2)];
            p[k++] = b;
            if (lp_split(s2, R2, C2)) p[k++] = b + 1;
        };
        if (type == LP_D) {
            if (s > 0) addB(s - 1, s, s);
            w[t] = cost.d;
        } else if (type == LP_T) {
            p[k++] = idD[s];
            if (s > 0) addB(s - 1, s, C);
            w[t] = cost.t;
        } else {
            p[k++] = idT[(size_t)s * np + R];
            if (C != R) p[k++] = idT[(size_t)s * np + C];
            if (s > 0) addB(s - 1, R, C);
            w[t] = ((R == C) ? cost.bd : cost.b) * (lp_split(s, R, C) ? 0.5 : 1.0);
        }
    }
    // successors (CSR)
    std::vector<long long> so((size_t)N + 1, 0), sl;
    for (long long t = 0; t < N; t++)
        for (int k = 0; k < NPRED; k++)
            if (pred[(size_t)t * NPRED + k] >= 0) so[(size_t)pred[(size_t)t * NPRED + k] + 1]++;
    for (long long t = 0; t < N; t++) so[(size_t)t + 1] += so[(size_t)t];
    sl.resize((size_t)so[(size_t)N]);
    {
        std::vector<long long> fill(so.begin(), so.end() - 1);
        for (long long t = 0; t < N; t++)
            for (int k = 0; k < NPRED; k++) {
                const long long p = pred[(size_t)t * NPRED + k];
                if (p >= 0) sl[(size_t)fill[(size_t)p]++] = t;
            }
    }
    // upward rank: own duration plus the longest path through the successors
    std::vector<double> rank((size_t)N);
    for (long long t = N - 1; t >= 0; t--) {
        double m = 0.0;
        for (long long e = so[(size_t)t]; e < so[(size_t)t + 1]; e++) m = std::max(m, rank[(size_t)sl[(size_t)e]]);
        rank[(size_t)t] = w[(size_t)t] + m;
    }
    // list scheduling: the chain worker runs D(s), T(s, s+1), B(s, s+1,
    // s+1) in that order, each as soon as it is ready; the P list workers
    // start the ready task of highest rank (earliest created among equals)
    // whenever one of them is free.  `full` receives every task in start
    // order.
    std::vector<char> pool((size_t)N, 1);  // 0 chain, 1 list
    std::vector<long long> cseq;
    for (int s = 0; s < np; s++) {
        pool[(size_t)idD[s]] = 0;
        cseq.push_back(idD[s]);
        if (s + 1 < np) {
            const long long t = idT[(size_t)s * np + s + 1], b = idB[bix(s, s + 1, s + 1)];
            pool[(size_t)t] = pool[(size_t)b] = 0;
            cseq.push_back(t);
            cseq.push_back(b);
        }
    }
    std::vector<int> npred((size_t)N, 0);
    for (long long t = 0; t < N; t++)
        for (int k = 0; k < NPRED; k++) npred[(size_t)t] += pred[(size_t)t * NPRED + k] >= 0;
    typedef std::pair<double, long long> Item;
    std::priority_queue<Item> ready;                                        // (rank, -id)
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> busy;  // (finish, id)
    for (long long t = 0; t < N; t++)
        if (npred[(size_t)t] == 0 && pool[(size_t)t]) ready.push({rank[(size_t)t], -t});
    list.clear();
    if (full) {
        full->clear();
        full->reserve((size_t)N);
    }
    int free_w[2] = {1, std::max(1, P)};
    size_t ci = 0;
    long long started = 0;
    double now = 0.0;
    while (started < N) {
        if (free_w[0] > 0 && ci < cseq.size() && npred[(size_t)cseq[ci]] == 0) {
            const long long t = cseq[ci];
            if (full) full->push_back(code[(size_t)t]);
            busy.push({now + w[(size_t)t], t});
            free_w[0]--;
            started++;
        }
        while (free_w[1] > 0 && !ready.empty()) {
            const long long t = -ready.top().second;
            ready.pop();
            list.push_back(code[(size_t)t]);
            if (full) full->push_back(code[(size_t)t]);
            busy.push({now + w[(size_t)t], t});
            free_w[1]--;
            started++;
        }
        if (busy.empty()) break;  // cannot happen for a valid graph
        const Item f = busy.top();
        busy.pop();
        now = f.first;
        const int fp = pool[(size_t)f.second];
        free_w[fp]++;
        if (fp == 0) ci++;
        for (long long e = so[(size_t)f.second]; e < so[(size_t)f.second + 1]; e++) {
            const long long q = sl[(size_t)e];
            if (--npred[(size_t)q] == 0 && pool[(size_t)q]) ready.push({rank[(size_t)q], -q});
        }
    }
}

// ---------------------------------------------------------------------------
// Device.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned lp_ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void lp_st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ double2 lp_ldcg(const cd* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ void lp_mma(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}
__device__ __forceinline__ cd lp_shfl(cd v, int src)
{
    return cd{__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src)};
}

// Thread 0: wait until *p >= v.  False when this CTA must stop (the poll
// limit ran out here or the abort word is set).
__device__ __forceinline__ bool lp_wait(const unsigned* p, unsigned v, unsigned* ctl, int* status, int limit)
{
    int spins = 0;
    while (lp_ld_acquire(p) < v) {
        if (++spins > limit || *((volatile unsigned*)(ctl + 1)) != 0u) {
            atomicExch(status + ST_SOLVE_TIMEOUT, 1);
            atomicExch(ctl + 1, 1u);
            return false;
        }
        __nanosleep(32);
    }
    return true;
}

// T(s, C): U(s, C) = invD L_ss^-1 W(s, C) for the 64 columns of tile
// (s, C), L_ss = U_ss^H unit lower, on the FP64 tensor cores by 8-row
// blocks: with X_b = L_bb^-1 (the inverse of the b-th 8 x 8 diagonal block
// of L) and the blocks L_ab below it,
//     Wun_b = X_b W_b,   W_a -= L_ab Wun_b  (a > b),   b = 0..7,
// which is the substitution of src/linalg.f90:384-389 for eight rows at a
// time.  Each warp owns eight columns and runs the whole recurrence on them
// (no barrier between the blocks); the eight X_b are formed first, one per
// warp, by substitution on the identity.
constexpr int LT_WP = 66;  // pitch (double2) of the working tile: fragment loads conflict-free
constexpr size_t LP_SMEM_T = (size_t)(LDL_NB * LT_WP + 2016 + 8 * 64 + LDL_NB) * sizeof(double2);

__device__ __forceinline__ int lt_li(int r, int q) { return r * (r - 1) / 2 + q; }  // packed strict lower, q < r

__device__ void lp_trsm(cd* __restrict__ A, int ld, int n, int s, int C, const cd* __restrict__ invD, double2* sm)
{
    double2* Wt = sm;                      // Wt[q * LT_WP + c]: the tile, then Wun
    double2* Lp = Wt + LDL_NB * LT_WP;     // L(r, q) = conj(U(q, r)), q < r, packed
    double2* Xb = Lp + 2016;               // X_b(i, j) at Xb[b * 64 + i * 8 + j]
    double2* ids = Xb + 8 * 64;            // invD of the panel
    const int p0 = s * LDL_NB, b = min(LDL_NB, n - p0);
    const int cb = C * LDL_NB, wd = min(LDL_NB, n - cb);
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int q = e & 63, c = e >> 6;
        const bool in = q < b && c < wd;
        cp_async16(Wt + q * LT_WP + c, in ? (const void*)(A + (size_t)(p0 + q) + (size_t)(cb + c) * ld) : (const void*)A,
                   in ? 16 : 0);
    }
    cp_async_commit();
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int q = e & 63, r = e >> 6;
        if (q < r) {
            double2 v = make_double2(0.0, 0.0);
            if (r < b) {
                v = lp_ldcg(A + (size_t)(p0 + q) + (size_t)(p0 + r) * ld);
                v.y = -v.y;
            }
            Lp[lt_li(r, q)] = v;
        }
    }
    if (tid < LDL_NB) ids[tid] = tid < b ? lp_ldcg(invD + p0 + tid) : make_double2(0.0, 0.0);
    __syncthreads();
    // X_wp = L_bb^-1 for block bb = wp: lane j < 8 holds column j
    {
        const int bb = wp, j = lane;
        cd x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = cd{(i == j) ? 1.0 : 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 8; q++)
#pragma unroll
            for (int r = q + 1; r < 8; r++) {
                const double2 l = Lp[lt_li(8 * bb + r, 8 * bb + q)];
                x[r] = cfms(cd{l.x, l.y}, x[q], x[r]);
            }
        if (j < 8)
#pragma unroll
            for (int i = 0; i < 8; i++) Xb[bb * 64 + i * 8 + j] = make_double2(x[i].x, x[i].y);
    }
    cp_async_wait<0>();
    __syncthreads();
    // the recurrence on this warp's eight columns
    const int c0 = 8 * wp;
#pragma unroll 1
    for (int bk = 0; bk < 8; bk++) {
        // Wun_b = X_b W_b
        double wr[2] = {0.0, 0.0}, wi[2] = {0.0, 0.0};
#pragma unroll
        for (int k0 = 0; k0 < 8; k0 += 4) {
            const double2 xa = Xb[bk * 64 + g * 8 + k0 + t4];         // X_b(g, k)
            const double2 wv = Wt[(8 * bk + k0 + t4) * LT_WP + c0 + g];  // W(k, c)
            lp_mma(wr[0], wr[1], xa.x, wv.x);
            lp_mma(wr[0], wr[1], -xa.y, wv.y);
            lp_mma(wi[0], wi[1], xa.x, wv.y);
            lp_mma(wi[0], wi[1], xa.y, wv.x);
        }
        __syncwarp();
#pragma unroll
        for (int e = 0; e < 2; e++) Wt[(8 * bk + g) * LT_WP + c0 + 2 * t4 + e] = make_double2(wr[e], wi[e]);
        __syncwarp();
        // W_a -= L_ab Wun_b for the blocks a below
        double2 un[2];
#pragma unroll
        for (int k0 = 0; k0 < 8; k0 += 4) un[k0 / 4] = Wt[(8 * bk + k0 + t4) * LT_WP + c0 + g];  // Wun(k, c)
#pragma unroll 1
        for (int a = bk + 1; a < 8; a++) {
            double ar[2], ai[2];
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const double2 o = Wt[(8 * a + g) * LT_WP + c0 + 2 * t4 + e];
                ar[e] = o.x;
                ai[e] = o.y;
            }
#pragma unroll
            for (int k0 = 0; k0 < 8; k0 += 4) {
                const double2 l = Lp[lt_li(8 * a + g, 8 * bk + k0 + t4)];  // L(r, k)
                const double2 u = un[k0 / 4];
                lp_mma(ar[0], ar[1], -l.x, u.x);
                lp_mma(ar[0], ar[1], l.y, u.y);
                lp_mma(ai[0], ai[1], -l.x, u.y);
                lp_mma(ai[0], ai[1], -l.y, u.x);
            }
#pragma unroll
            for (int e = 0; e < 2; e++) Wt[(8 * a + g) * LT_WP + c0 + 2 * t4 + e] = make_double2(ar[e], ai[e]);
        }
        __syncwarp();
    }
    // U = invD Wun
    for (int e = lane; e < LDL_NB * 8; e += 32) {
        const int q = e & 63, c = c0 + (e >> 6);
        if (q < b && c < wd) {
            const double2 v = Wt[q * LT_WP + c], d = ids[q];
            A[(size_t)(p0 + q) + (size_t)(cb + c) * ld] = cmul(cd{v.x, v.y}, cd{d.x, d.y});
        }
    }
}

// B(s, R, C): W(r, c) -= sum_q conj(U(q, r)) d_q U(q, c) over the 64 x 64
// tile, r <= c on a diagonal tile (its diagonal in dw).  Eight warps as
// 2 x 4, each a 32 x 16 complex sub-tile of 8 x 8 mma tiles; the tile's
// old values are the accumulators' initial values (the minus sign is folded
// into the operand -d U(q, c)), so a product is accumulated straight onto
// them; U(s, R) and U(s, C) stream through three cp.async stages of 16 k
// rows.  m consecutive panels s..s+m-1 (whose rows are contiguous) are
// applied in one pass when they are all ready: a rank-64m update, the
// tile read and written once.
// MT x NT mma tiles per warp, WR x WC warps: <4, 2, 2, 4> covers the whole
// 64 x 64 tile, <2, 2, 4, 2> the 64 x 32 column half `half` of it.
template <int MT, int NT, int WR, int WC>
__device__ void lp_update(cd* __restrict__ A, int ld, int n, int s, int m, int R, int C, int half,
                          cd* __restrict__ dw, double2* sm)
{
    static_assert(WR * WC == 8 && WR * MT * 8 == LDL_NB, "eight warps over the 64 tile rows");
    constexpr int CW = WC * NT * 8;  // columns covered
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int wr = wp / WC, wc = wp % WC;
    const int g = lane >> 2, t4 = lane & 3;
    const int p0 = s * LDL_NB, b = min(m * LDL_NB, n - p0);
    const int rb = R * LDL_NB, cb = C * LDL_NB + half * CW;
    const bool dtile = (R == C);
    double2* dp = sm + LP_ST * LP_KC * 2 * LP_P;  // pivots d_q of panels s..s+m-1
    for (int q = tid; q < m * LDL_NB; q += 256) dp[q] = q < b ? lp_ldcg(dw + p0 + q) : make_double2(0.0, 0.0);
    // a warp whose sub-tile lies wholly below the diagonal has nothing to do
    const bool wact = !dtile || (wr * MT * 8 <= half * CW + (wc + 1) * NT * 8 - 1);
    auto stage = [&](int ch, int buf) {
        const int k0 = ch * LP_KC;
        double2* Us = sm + buf * LP_KC * 2 * LP_P;
        double2* Vs = Us + LP_KC * LP_P;
#pragma unroll
        for (int e = tid; e < LP_KC * LDL_NB; e += 256) {
            const int q = e % LP_KC, mm = e / LP_KC;
            const bool kq = k0 + q < b;
            const int r = rb + mm;
            const bool ku = kq && r < n;
            cp_async16(Us + q * LP_P + mm, ku ? (const void*)(A + (size_t)(p0 + k0 + q) + (size_t)r * ld) : (const void*)A,
                       ku ? 16 : 0);
        }
#pragma unroll
        for (int e = tid; e < LP_KC * CW; e += 256) {
            const int q = e % LP_KC, mm = e / LP_KC;
            const int c = cb + mm;
            const bool kv = (k0 + q < b) && c < n;
            cp_async16(Vs + q * LP_P + mm, kv ? (const void*)(A + (size_t)(p0 + k0 + q) + (size_t)c * ld) : (const void*)A,
                       kv ? 16 : 0);
        }
        cp_async_commit();
    };
    const int nch = (b + LP_KC - 1) / LP_KC;
    stage(0, 0);
    if (nch > 1) stage(1, 1);
    double accr[MT][NT][2], acci[MT][NT][2];
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int r = rb + (wr * MT + mt) * 8 + g;
                const int c = cb + (wc * NT + nt) * 8 + 2 * t4 + e;
                double2 o = make_double2(0.0, 0.0);
                if (r < n && c < n && r <= c) {
                    if (r == c) {
                        o = lp_ldcg(dw + c);
                        o.y = -o.y;  // dw keeps the conjugate of the upper-triangle value
                    } else {
                        o = lp_ldcg(A + (size_t)r + (size_t)c * ld);
                    }
                }
                accr[mt][nt][e] = o.x;
                acci[mt][nt][e] = o.y;
            }
    for (int ch = 0; ch < nch; ch++) {
        if (ch + 2 < nch) {
            __syncthreads();  // buffer (ch + 2) % 3 was read in step ch - 1
            stage(ch + 2, (ch + 2) % LP_ST);
            cp_async_wait<2>();
        } else if (ch + 1 < nch) {
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (wact) {
            const double2* Us = sm + (ch % LP_ST) * LP_KC * 2 * LP_P;
            const double2* Vs = Us + LP_KC * LP_P;
#pragma unroll
            for (int kk = 0; kk < LP_KC; kk += 4) {
                const double2 d = dp[ch * LP_KC + kk + t4];
                double2 a[MT];
                double vr[NT], vi[NT];
#pragma unroll
                for (int mt = 0; mt < MT; mt++) a[mt] = Us[(kk + t4) * LP_P + (wr * MT + mt) * 8 + g];
#pragma unroll
                for (int nt = 0; nt < NT; nt++) {
                    const double2 v = Vs[(kk + t4) * LP_P + (wc * NT + nt) * 8 + g];
                    // -(d v): the unscaled row, negated
                    vr[nt] = -fma(v.x, d.x, -v.y * d.y);
                    vi[nt] = -fma(v.x, d.y, v.y * d.x);
                }
#pragma unroll
                for (int mt = 0; mt < MT; mt++)
#pragma unroll
                    for (int nt = 0; nt < NT; nt++) {
                        lp_mma(accr[mt][nt][0], accr[mt][nt][1], a[mt].x, vr[nt]);
                        lp_mma(accr[mt][nt][0], accr[mt][nt][1], a[mt].y, vi[nt]);
                        lp_mma(acci[mt][nt][0], acci[mt][nt][1], a[mt].x, vi[nt]);
                        lp_mma(acci[mt][nt][0], acci[mt][nt][1], -a[mt].y, vr[nt]);
                    }
            }
        }
    }
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int r = rb + (wr * MT + mt) * 8 + g;
                const int c = cb + (wc * NT + nt) * 8 + 2 * t4 + e;
                if (r >= n || c >= n || c < r) continue;
                if (c == r)
                    dw[c] = cd{accr[mt][nt][e], -acci[mt][nt][e]};
                else
                    A[(size_t)r + (size_t)c * ld] = cd{accr[mt][nt][e], acci[mt][nt][e]};
            }
}

struct LpArgs {
    cd* A;
    int ld, n, np;
    const unsigned* tasks;  // the list of the CTAs other than the chain CTA
    int ntasks;
    unsigned* cnt;          // tile counters
    unsigned* hc;           // per tile: column halves of band updates finished
    unsigned* ctl;          // [0] next list index, [1] abort word, [2] trace records, [3] chain CTA's SM + 1
    cd* dw;
    cd* invD;
    int* status;
    const int* limitp;      // poll limit of the bounded waits
    unsigned long long* trace;  // optional: per task (code | cta << 32 | panels << 48, start, ready, done)
};

__device__ __forceinline__ unsigned long long lp_clock()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The tile counts a list task waits for: cnt[ix[i]] >= need[i], i < the
// returned count.
__device__ __forceinline__ int lp_deps(unsigned task, long long (&ix)[3], unsigned (&need)[3])
{
    const unsigned type = task >> 30;
    const int s = (task >> 20) & 511, R = (task >> 10) & 1023, C = task & 1023;
    ix[1] = ix[2] = 0;
    need[1] = need[2] = 0u;
    if (type == LP_T) {
        ix[0] = lp_tix(s, s), need[0] = (unsigned)s + 1;
        ix[1] = lp_tix(s, C), need[1] = (unsigned)s;
        return 2;
    }
    ix[0] = lp_tix(R, C), need[0] = (unsigned)s;
    ix[1] = lp_tix(s, R), need[1] = (unsigned)s + 1;
    ix[2] = lp_tix(s, C), need[2] = (unsigned)s + 1;
    return (R == C) ? 2 : 3;
}

// Thread 0: wait until cnt[ix[i]] >= need[i] for the k (<= 3) conditions,
// polling them together.  False when this CTA must stop.
__device__ __forceinline__ bool lp_wait_all(const LpArgs& a, const long long (&ix)[3], const unsigned (&need)[3],
                                            int k, int limit)
{
    int spins = 0;
    for (;;) {
        unsigned v[3];
#pragma unroll
        for (int i = 0; i < 3; i++) v[i] = (i < k) ? lp_ld_acquire(a.cnt + ix[i]) : 0u;
        bool ok = true;
#pragma unroll
        for (int i = 0; i < 3; i++) ok = ok && (i >= k || v[i] >= need[i]);
        if (ok) return true;
        if (++spins > limit || *((volatile unsigned*)(a.ctl + 1)) != 0u) {
            atomicExch(a.status + ST_SOLVE_TIMEOUT, 1);
            atomicExch(a.ctl + 1, 1u);
            return false;
        }
        __nanosleep(32);
    }
}

__device__ __forceinline__ void lp_trace(const LpArgs& a, unsigned code, int m, unsigned long long t0,
                                         unsigned long long t1)
{
    if (!a.trace) return;
    const unsigned long long t2 = lp_clock();
    const unsigned i = atomicAdd(a.ctl + 2, 1u);
    unsigned long long* r = a.trace + 4 * (size_t)i;
    r[0] = (unsigned long long)code | (unsigned long long)blockIdx.x << 32 | (unsigned long long)m << 48;
    r[1] = t0;
    r[2] = t1;
    r[3] = t2;
}

// One task, all threads.  Thread 0 has checked the dependencies; on return
// the task's stores are done (a barrier follows).  m: panels of an update.
__device__ __forceinline__ void lp_exec(const LpArgs& a, unsigned type, int s, int m, int R, int C, int half,
                                        double2* sm)
{
    if (type == LP_T)
        lp_trsm(a.A, a.ld, a.n, s, C, a.invD, sm);
    else if (lp_split(s, R, C))
        lp_update<2, 2, 4, 2>(a.A, a.ld, a.n, s, 1, R, C, half, a.dw, sm);
    else
        lp_update<4, 2, 2, 4>(a.A, a.ld, a.n, s, m, R, C, 0, a.dw, sm);
}

// After the task's barrier: thread 0 publishes the tile's new count.  The
// barrier orders every thread's stores before the gpu-scope release.
__device__ __forceinline__ void lp_publish(const LpArgs& a, long long ix, unsigned v)
{
    if (threadIdx.x == 0) lp_st_release(a.cnt + ix, v);
}

// ---------------------------------------------------------------------------
// The chain CTA.  It keeps the working diagonal tile (s, s) in shared
// memory (its diagonal as dw holds it) and per panel s runs the three tasks
// the next diagonal tile waits for:
//   D(s)          elimination of the tile by 8-row sub-panels (8 x 8 blocks
//                 by the lanes of warp 0, the rows beyond them by
//                 substitution, rank-8 updates on the FP64 tensor cores,
//                 the next block's elimination beside the update);
//                 published at once, so the other panel rows start;
//   T(s, s+1)     the tile to its right, by the blocked recurrence of
//                 lp_trsm with L read from the tile in shared memory;
//   B(s, s+1, s+1) tile (s+1, s+1) loaded once the other CTAs have applied
//                 panels 0..s-1, then panel s applied from the panel rows
//                 still in shared memory; it stays there for step s+1.
// The tile (s+1, s+2) that T(s+1, s+2) needs comes from the other CTAs
// (T(s, s+2), then B(s, s+1, s+2)) while this CTA runs D(s+1).
constexpr int LC_NP = 2080;  // packed upper triangle of a 64 x 64 tile
__device__ __forceinline__ int lc_pu(int r, int c) { return r * 64 - r * (r - 1) / 2 + (c - r); }  // r <= c
constexpr size_t LP_SMEM_C = (size_t)(LC_NP + LDL_NB * LT_WP + 2 * LDL_NB + 8 * 64) * sizeof(double2);
constexpr size_t lp_max(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t LP_SMEM = lp_max(LP_SMEM_B, lp_max(LP_SMEM_C, LP_SMEM_T));

template <bool CPLX>
__device__ void lp_chain(const LpArgs& a, double2* sm, int limit)
{
    double2* P = sm;                      // packed tile: U_ss during T, tile (s+1, s+1) during B
    double2* Rt = sm + LC_NP;             // right tile, Rt[q * LT_WP + c] (during T and B)
    double2* Ws = Rt;                     // working diagonal tile, Ws[r * LP_LD + c] (during D)
    double2* dpv = Rt + LDL_NB * LT_WP;   // pivots d of the panel
    double2* sinv = dpv + LDL_NB;         // their inverses (invD)
    double2* Xb = sinv + LDL_NB;          // X_b = L_bb^-1, Xb[b * 64 + i * 8 + j]
    __shared__ double2 sid[LP_SUB];
    __shared__ int s_go, s_v;
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int n = a.n, ld = a.ld;
    cd* A = a.A;
    // tile (0, 0) from global memory (upper triangle and dw)
    for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
        const int r = e & 63, c = e >> 6;
        double2 v = make_double2(0.0, 0.0);
        if (r <= c && c < min(LDL_NB, n)) v = (r < c) ? lp_ldcg(A + (size_t)r + (size_t)c * ld) : lp_ldcg(a.dw + r);
        Ws[r * LP_LD + c] = v;
    }
    __syncthreads();
    for (int s = 0; s < a.np; s++) {
        const int p0 = s * LDL_NB, b = min(LDL_NB, n - p0);
        const bool right = s + 1 < a.np;
        const int cb = p0 + LDL_NB, wd = right ? min(LDL_NB, n - cb) : 0;
        unsigned long long t0 = 0;
        if (tid == 0 && a.trace) t0 = lp_clock();
        // ================= D(s)
        auto eliminate = [&](int s0) {  // warp 0: the 8 x 8 sub-block at s0
            const int nq = min(LP_SUB, b - s0);
            const int j = lane;
            const bool col = j < nq;
            cd x[LP_SUB];
#pragma unroll
            for (int i = 0; i < LP_SUB; i++) {
                double2 v = make_double2(0.0, 0.0);
                if (col && i <= j) v = Ws[(s0 + i) * LP_LD + s0 + j];
                x[i] = cd{v.x, v.y};
            }
#pragma unroll
            for (int q = 0; q < LP_SUB; q++) {
                if (q < nq) {
                    const cd dq = lp_shfl(x[q], q);
                    const double dr = dq.x, di = CPLX ? dq.y : 0.0;
                    const bool zero = (dr == 0.0 && di == 0.0);
                    double id, idi = 0.0;
                    if (CPLX) {
                        const double m = zero ? 0.0 : __drcp_rn(fma(dr, dr, di * di));
                        id = dr * m;
                        idi = -di * m;
                    } else {
                        id = zero ? 0.0 : __drcp_rn(dr);
                    }
                    if (lane == 0) {
                        sid[q] = make_double2(id, idi);
                        dpv[s0 + q] = make_double2(dr, di);
                        sinv[s0 + q] = make_double2(id, idi);
                        a.invD[p0 + s0 + q] = cd{id, idi};
                        a.dw[p0 + s0 + q] = cd{dr, di};
                        if (zero) atomicCAS(a.status + ST_ZERO_PIVOT, 0, p0 + s0 + q + 1);
                    }
                    cd u = cd{0.0, 0.0};
                    if (col && j > q) u = CPLX ? cmul(x[q], cd{id, idi}) : cd{x[q].x * id, x[q].y * id};
#pragma unroll
                    for (int i = q + 1; i < LP_SUB; i++) {
                        const cd ui = lp_shfl(u, i);
                        if (col && j >= i) x[i] = cfms(conj(ui), x[q], x[i]);
                    }
                    if (col && j > q) x[q] = u;
                }
            }
#pragma unroll
            for (int i = 0; i < LP_SUB; i++)
                if (col && i < j) Ws[(s0 + i) * LP_LD + s0 + j] = make_double2(x[i].x, x[i].y);
        };
        // s0 = -8: the first sub-block's elimination alone; then per
        // sub-panel (b), (c) and the next elimination (one call site keeps
        // the code small)
        for (int s0 = -LP_SUB; s0 < b; s0 += LP_SUB) {
            if (s0 < 0) {
                if (wp == 0) eliminate(0);
                __syncthreads();
                continue;
            }
            const int nq = min(LP_SUB, b - s0);
            const int t0c = s0 + LP_SUB;
            if (t0c >= b) break;
            // (b) sub-panel rows beyond the sub-block, one thread per column
            if (tid < b - t0c) {
                const int c = t0c + tid;
                cd wun[LP_SUB];
#pragma unroll
                for (int q = 0; q < LP_SUB; q++) {
                    if (q < nq) {
                        double2* wq = Ws + (s0 + q) * LP_LD + c;
                        const double2 w = *wq;
                        cd v = cd{w.x, w.y};
#pragma unroll
                        for (int q2 = 0; q2 < q; q2++) {
                            const double2 u = Ws[(s0 + q2) * LP_LD + s0 + q];  // U(q2, q)
                            v = cfms(cd{u.x, -u.y}, wun[q2], v);
                        }
                        wun[q] = v;
                        const double2 id = sid[q];
                        const cd uq = CPLX ? cmul(v, cd{id.x, id.y}) : cd{v.x * id.x, v.y * id.x};
                        *wq = make_double2(uq.x, uq.y);
                    } else {
                        wun[q] = cd{0.0, 0.0};
                    }
                }
            }
            __syncthreads();
            // (c) rank-8 update of rows and columns [t0c, b), B operand
            // d_q U(q, c); warp 0 takes the next diagonal sub-block and
            // eliminates it at once
            {
                const int T = (b - t0c + 7) >> 3;
                const int ntiles = T * (T + 1) / 2;
                for (int tile = (wp == 0) ? 0 : wp; tile < ntiles; tile += (wp == 0) ? ntiles : 7) {
                    int Rr = 0, rem = tile;
                    while (rem >= T - Rr) {
                        rem -= T - Rr;
                        Rr++;
                    }
                    const int Cc = Rr + rem;
                    const int r = t0c + 8 * Rr + g, cgc = t0c + 8 * Cc + g, ca = t0c + 8 * Cc + 2 * t4;
                    double accr[2], acci[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int c = ca + e;
                        double2 w = make_double2(0.0, 0.0);
                        if (r < b && c < b && r <= c) w = Ws[(r) * LP_LD + c];
                        accr[e] = w.x;
                        acci[e] = w.y;
                    }
#pragma unroll
                    for (int k0 = 0; k0 < LP_SUB; k0 += 4) {
                        const int q = k0 + t4;
                        double2 u = make_double2(0.0, 0.0), v = make_double2(0.0, 0.0);
                        if (q < nq && r < b) u = Ws[(s0 + q) * LP_LD + r];  // U(q, r)
                        if (q < nq && cgc < b) {
                            const double2 uc = Ws[(s0 + q) * LP_LD + cgc];  // U(q, c)
                            const double2 d = dpv[s0 + q];
                            v = make_double2(fma(uc.x, d.x, -uc.y * d.y), fma(uc.x, d.y, uc.y * d.x));
                        }
                        lp_mma(accr[0], accr[1], -u.x, v.x);
                        lp_mma(accr[0], accr[1], -u.y, v.y);
                        lp_mma(acci[0], acci[1], -u.x, v.y);
                        lp_mma(acci[0], acci[1], u.y, v.x);
                    }
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int c = ca + e;
                        if (r < b && c < b && r <= c) Ws[(r) * LP_LD + c] = make_double2(accr[e], acci[e]);
                    }
                }
                if (wp == 0) {
                    __syncwarp();
                    eliminate(t0c);
                }
            }
            __syncthreads();
        }
        // U_ss out, and packed for T (the right tile overwrites Ws)
        for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
            const int r = e & 63, c = e >> 6;
            if (r < c) {
                const double2 v = Ws[r * LP_LD + c];
                P[lc_pu(r, c)] = v;
                if (c < b) A[(size_t)(p0 + r) + (size_t)(p0 + c) * ld] = cd{v.x, v.y};
            }
        }
        __syncthreads();
        lp_publish(a, lp_tix(s, s), (unsigned)s + 1);
        if (tid == 0) lp_trace(a, lp_code(LP_D, s, s, s), 1, t0, t0);
        if (!right) break;
        // ================= T(s, s+1)
        if (tid == 0) {
            if (a.trace) t0 = lp_clock();
            long long ix[3] = {lp_tix(s, s + 1), 0, 0};
            unsigned need[3] = {(unsigned)s, 0u, 0u};
            s_go = lp_wait_all(a, ix, need, 1, limit) ? 1 : 0;
        }
        __syncthreads();
        if (!s_go) return;
        unsigned long long t1 = 0;
        if (tid == 0 && a.trace) t1 = lp_clock();
        for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
            const int q = e & 63, c = e >> 6;
            const bool in = c < wd;
            cp_async16(Rt + q * LT_WP + c, in ? (const void*)(A + (size_t)(p0 + q) + (size_t)(cb + c) * ld) : (const void*)A,
                       in ? 16 : 0);
        }
        cp_async_commit();
        {
            // X_wp = L_bb^-1 of block bb = wp, L(r, q) = conj(U(q, r)); lane j < 8 holds column j
            const int bb = wp, j = lane;
            cd x[8];
#pragma unroll
            for (int i = 0; i < 8; i++) x[i] = cd{(i == j) ? 1.0 : 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < 8; q++)
#pragma unroll
                for (int r = q + 1; r < 8; r++) {
                    const double2 u = P[lc_pu(8 * bb + q, 8 * bb + r)];
                    x[r] = cfms(cd{u.x, -u.y}, x[q], x[r]);
                }
            if (j < 8)
#pragma unroll
                for (int i = 0; i < 8; i++) Xb[bb * 64 + i * 8 + j] = make_double2(x[i].x, x[i].y);
        }
        cp_async_wait<0>();
        __syncthreads();
        {
            const int c0 = 8 * wp;
#pragma unroll 1
            for (int bk = 0; bk < 8; bk++) {
                double wr[2] = {0.0, 0.0}, wi[2] = {0.0, 0.0};
#pragma unroll
                for (int k0 = 0; k0 < 8; k0 += 4) {
                    const double2 xa = Xb[bk * 64 + g * 8 + k0 + t4];
                    const double2 wv = Rt[(8 * bk + k0 + t4) * LT_WP + c0 + g];
                    lp_mma(wr[0], wr[1], xa.x, wv.x);
                    lp_mma(wr[0], wr[1], -xa.y, wv.y);
                    lp_mma(wi[0], wi[1], xa.x, wv.y);
                    lp_mma(wi[0], wi[1], xa.y, wv.x);
                }
                __syncwarp();
#pragma unroll
                for (int e = 0; e < 2; e++) Rt[(8 * bk + g) * LT_WP + c0 + 2 * t4 + e] = make_double2(wr[e], wi[e]);
                __syncwarp();
                double2 un[2];
#pragma unroll
                for (int k0 = 0; k0 < 8; k0 += 4) un[k0 / 4] = Rt[(8 * bk + k0 + t4) * LT_WP + c0 + g];
#pragma unroll 1
                for (int a2 = bk + 1; a2 < 8; a2++) {
                    double ar[2], ai[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const double2 o = Rt[(8 * a2 + g) * LT_WP + c0 + 2 * t4 + e];
                        ar[e] = o.x;
                        ai[e] = o.y;
                    }
#pragma unroll
                    for (int k0 = 0; k0 < 8; k0 += 4) {
                        const double2 uu = P[lc_pu(8 * bk + k0 + t4, 8 * a2 + g)];  // U(k, r): L(r, k) = conj
                        const double2 u = un[k0 / 4];
                        lp_mma(ar[0], ar[1], -uu.x, u.x);
                        lp_mma(ar[0], ar[1], -uu.y, u.y);
                        lp_mma(ai[0], ai[1], -uu.x, u.y);
                        lp_mma(ai[0], ai[1], uu.y, u.x);
                    }
#pragma unroll
                    for (int e = 0; e < 2; e++) Rt[(8 * a2 + g) * LT_WP + c0 + 2 * t4 + e] = make_double2(ar[e], ai[e]);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // U(s, s+1) = invD Wun: kept in shared memory and written out
        for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
            const int q = e & 63, c = e >> 6;
            const double2 v = Rt[q * LT_WP + c], d = sinv[q];
            const cd u = cmul(cd{v.x, v.y}, cd{d.x, d.y});
            Rt[q * LT_WP + c] = make_double2(u.x, u.y);
            if (c < wd) A[(size_t)(p0 + q) + (size_t)(cb + c) * ld] = u;
        }
        __syncthreads();
        lp_publish(a, lp_tix(s, s + 1), (unsigned)s + 1);
        if (tid == 0) lp_trace(a, lp_code(LP_T, s, s, s + 1), 1, t0, t1);
        // ================= B(s, s+1, s+1)
        if (tid == 0) {
            if (a.trace) t0 = lp_clock();
            long long ix[3] = {lp_tix(s + 1, s + 1), 0, 0};
            unsigned need[3] = {(unsigned)s, 0u, 0u};
            const int go = lp_wait_all(a, ix, need, 1, limit) ? 1 : 0;
            s_go = go;
            s_v = go ? (int)lp_ld_acquire(a.cnt + ix[0]) : 0;
            if (a.trace) t1 = lp_clock();
        }
        __syncthreads();
        if (!s_go) return;
        const int applied = s_v;  // panels already applied to tile (s+1, s+1)
        const int q0 = p0 + LDL_NB, bn = min(LDL_NB, n - q0);
        for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
            const int r = e & 63, c = e >> 6;
            if (r > c) continue;
            double2 v = make_double2(0.0, 0.0);
            if (c < bn) v = (r < c) ? lp_ldcg(A + (size_t)(q0 + r) + (size_t)(q0 + c) * ld) : lp_ldcg(a.dw + q0 + r);
            P[lc_pu(r, c)] = v;
        }
        __syncthreads();
        if (applied == s) {
            // 8 x 8 tiles of the upper triangle; A = conj(U(q, r)), B = -(d_q U(q, c))
            for (int tile = wp; tile < 36; tile += 8) {
                int Rr = 0, rem = tile;
                while (rem >= 8 - Rr) {
                    rem -= 8 - Rr;
                    Rr++;
                }
                const int Cc = Rr + rem;
                const int r = 8 * Rr + g, cgc = 8 * Cc + g, ca = 8 * Cc + 2 * t4;
                double accr[2], acci[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int c = ca + e;
                    double2 w = make_double2(0.0, 0.0);
                    if (r <= c && c < bn) {
                        w = P[lc_pu(r, c)];
                        if (r == c) w.y = -w.y;  // dw keeps the conjugate of the upper-triangle value
                    }
                    accr[e] = w.x;
                    acci[e] = w.y;
                }
#pragma unroll 2
                for (int k0 = 0; k0 < LDL_NB; k0 += 4) {
                    const int q = k0 + t4;
                    const double2 u = Rt[q * LT_WP + r];
                    const double2 uc = Rt[q * LT_WP + cgc];
                    const double2 d = dpv[q];
                    const double vr = -fma(uc.x, d.x, -uc.y * d.y), vi = -fma(uc.x, d.y, uc.y * d.x);
                    lp_mma(accr[0], accr[1], u.x, vr);
                    lp_mma(accr[0], accr[1], u.y, vi);
                    lp_mma(acci[0], acci[1], u.x, vi);
                    lp_mma(acci[0], acci[1], -u.y, vr);
                }
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int c = ca + e;
                    if (r <= c && c < bn) P[lc_pu(r, c)] = (r == c) ? make_double2(accr[e], -acci[e]) : make_double2(accr[e], acci[e]);
                }
            }
        }
        __syncthreads();
        // the next diagonal tile into Ws (the right tile is no longer needed)
        for (int e = tid; e < LDL_NB * LDL_NB; e += 256) {
            const int r = e & 63, c = e >> 6;
            Ws[r * LP_LD + c] = (r <= c) ? P[lc_pu(r, c)] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (tid == 0) lp_trace(a, lp_code(LP_B, s, s + 1, s + 1), applied == s ? 1 : 0, t0, t1);
    }
}

// CTA 0 runs the critical chain, per panel s: D(s), then T(s, s+1) and
// B(s, s+1, s+1), which D(s+1) needs; D(s) is published before the other
// two so that the panel rows of the other tiles start at once.  The other
// CTAs take every remaining task from the list, each when it is free.  An update B(s, R, C)
// whose tile already carries more than s panels (applied by an earlier
// merged update) does nothing; otherwise it also applies the following
// panels s+1.. (up to LP_MERGE in all, below R) whose panel rows of R and
// C are already final.
template <bool CPLX>
__global__ void __launch_bounds__(256, 2) k_ldl_persist(LpArgs a)
{
    extern __shared__ double2 lsm[];
    __shared__ unsigned s_next;
    __shared__ int s_go, s_m;
    const int tid = threadIdx.x;
    const int limit = *((const volatile int*)a.limitp);
    // the chain CTA has its SM to itself: it publishes its SM, and the CTA
    // sharing that SM takes no tasks
    if (tid == 0) {
        unsigned smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        int go = 1;
        if (blockIdx.x == 0) {
            lp_st_release(a.ctl + 3, smid + 1);
        } else {
            int spins = 0;
            unsigned v;
            while ((v = lp_ld_acquire(a.ctl + 3)) == 0u) {
                if (++spins > limit || *((volatile unsigned*)(a.ctl + 1)) != 0u) {
                    atomicExch(a.status + ST_SOLVE_TIMEOUT, 1);
                    atomicExch(a.ctl + 1, 1u);
                    break;
                }
                __nanosleep(32);
            }
            go = (v != 0u && v != smid + 1);
        }
        s_go = go;
    }
    __syncthreads();
    if (!s_go) return;
    if (blockIdx.x == 0) {
        lp_chain<CPLX>(a, lsm, limit);
        return;
    }
    for (;;) {
        unsigned long long t0 = 0, t1 = 0;
        if (tid == 0) {
            if (a.trace) t0 = lp_clock();
            // the next task in list order, taken when this CTA is free (a
            // task fetched earlier could wait behind a long update)
            unsigned task = LP_NONE;
            if (*((volatile unsigned*)(a.ctl + 1)) == 0u) {
                const unsigned i = atomicAdd(a.ctl, 1u);
                if (i < (unsigned)a.ntasks) task = __ldg(a.tasks + i);
            }
            int go = 0, m = 1;
            if (task != LP_NONE) {
                const unsigned type = task >> 30;
                const int s = (task >> 20) & 511, R = (task >> 10) & 1023, C = task & 1023;
                long long ix[3] = {0, 0, 0};
                unsigned need[3] = {0u, 0u, 0u};
                const int k = lp_deps(task, ix, need);
                go = lp_wait_all(a, ix, need, k, limit) ? 1 : 0;
                if (go && type == LP_B) {
                    if (lp_ld_acquire(a.cnt + ix[0]) > (unsigned)s) {
                        go = 2;  // applied already by a merged update
                    } else if (!lp_split(s, R, C)) {
                        // following panels whose rows of R and C are final
                        unsigned fr[LP_MERGE - 1], fc[LP_MERGE - 1];
#pragma unroll
                        for (int j = 1; j < LP_MERGE; j++) {
                            const bool in = s + j < R;
                            fr[j - 1] = in ? lp_ld_acquire(a.cnt + lp_tix(s + j, R)) : 0u;
                            fc[j - 1] = (in && R != C) ? lp_ld_acquire(a.cnt + lp_tix(s + j, C)) : 0u;
                        }
#pragma unroll
                        for (int j = 1; j < LP_MERGE; j++) {
                            const unsigned want = (unsigned)(s + j) + 1;
                            // the panels of the band next to row R (split in column
                            // halves) and the chain's own update keep their own short
                            // tasks: a long merged update would hold up the panel rows
                            // the chain waits for
                            const bool own = lp_split(s + j, R, C) || (s + j == R - 1);
                            if (m == j && !own && s + j < R && fr[j - 1] >= want && (R == C || fc[j - 1] >= want))
                                m = j + 1;
                        }
                    }
                }
                if (!go) task = LP_NONE;
            }
            s_next = task;
            s_go = go;
            s_m = m;
            if (a.trace) t1 = lp_clock();
        }
        __syncthreads();
        const unsigned task = s_next;
        const int go = s_go, m = s_m;
        if (task == LP_NONE) return;
        const unsigned type = task >> 30;
        const int s = (task >> 20) & 511, R = (task >> 10) & 1023, C = task & 1023;
        const int half = (task >> 29) & 1;
        if (go == 1) {
            lp_exec(a, type, s, m, R, C, half, lsm);
            __syncthreads();
            const long long tt = (type == LP_B) ? lp_tix(R, C) : lp_tix(s, (type == LP_D) ? s : C);
            if (type == LP_B && lp_split(s, R, C)) {
                // a column half: the second of the two to finish publishes the tile
                if (tid == 0) {
                    unsigned old;
                    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(a.hc + tt) : "memory");
                    if (old & 1u) lp_st_release(a.cnt + tt, (unsigned)s + 1);
                }
            } else {
                lp_publish(a, tt, (unsigned)(s + m));
            }
        }
        if (tid == 0) lp_trace(a, task, go == 1 ? m : 0, t0, t1);
        __syncthreads();  // s_next, s_go, s_m are rewritten by the next task
    }
}

static bool g_lp_attr = false;

// Grid of the persistent kernel (co-resident CTAs), 0 if unavailable.
int ldlp_grid(Ctx& c)
{
    if (!g_lp_attr) {
        if (cudaFuncSetAttribute(k_ldl_persist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LP_SMEM) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_ldl_persist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LP_SMEM) !=
                cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        g_lp_attr = true;
    }
    if (c.lp_grid > 0) return c.lp_grid;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ldl_persist<false>, 256, LP_SMEM) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.dev);
    if (!coop || per_sm < 1) return 0;
    c.lp_grid = per_sm * sms;
    c.lp_sms = sms;
    return c.lp_grid;
}

// The task list of an n-row factorisation in device memory (owned by the
// caller, freed with cudaFree; at least one entry); *count receives its
// length (0 when the chain CTA does everything).
int ldlp_tasks(Ctx& c, int n, unsigned** tasks, int* count)
{
    const int grid = ldlp_grid(c);
    if (grid <= 0) return -1;
    const int np = (n + LDL_NB - 1) / LDL_NB;
    if (np > 200) return -1;
    const int per_sm = std::max(1, c.lp_grid / std::max(1, c.lp_sms));
    std::vector<unsigned> list;
    lp_schedule(np, std::max(1, grid - per_sm), LpCost(), list);
    unsigned* d = nullptr;
    if (cudaMalloc(&d, std::max<size_t>(1, list.size()) * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        return -3;
    }
    if (!list.empty() &&
        cudaMemcpy(d, list.data(), list.size() * sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return -2;
    }
    *tasks = d;
    *count = (int)list.size();
    return 0;
}

// Number of tasks of an n-row factorisation, the chain's included.
long long ldlp_task_total(int n)
{
    const long long np = (n + LDL_NB - 1) / LDL_NB;
    long long split = 0;  // the second column halves of the band updates
    for (long long s = 0; s + 2 < np; s++) split += 2 * (np - s - 2);
    return np + np * (np - 1) / 2 + (np - 1) * np * (np + 1) / 6 + split;
}

// Tile counters and the control words (next task, abort word, trace
// records, the chain CTA's SM) for np panels.
int ldlp_reserve(Ctx& c, int np)
{
    const size_t need = (size_t)np * (np + 1) + 4;
    if (c.lp_cap >= need) return 0;
    if (c.lp_cnt) cudaFree(c.lp_cnt);
    c.lp_cnt = nullptr;
    c.lp_cap = 0;
    if (cudaMalloc(&c.lp_cnt, need * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        return -3;
    }
    c.lp_cap = need;
    return 0;
}

// Queue one persistent factorisation of rows 0..n-1 (the working upper
// triangle and dw already initialised by k_ldl_mirror); trace (device,
// 4 x ldlp_task_total(n) values) may be null.
void ldlp_enqueue(Ctx& c, int n, const unsigned* tasks, int ntasks, unsigned long long* trace)
{
    const int np = (n + LDL_NB - 1) / LDL_NB;
    const size_t ntile = (size_t)np * (np + 1) / 2;
    cudaMemsetAsync(c.lp_cnt, 0, (2 * ntile + 4) * sizeof(unsigned), c.stream);
    LpArgs a;
    a.A = c.F;
    a.ld = c.ld;
    a.n = n;
    a.np = np;
    a.tasks = tasks;
    a.ntasks = ntasks;
    a.cnt = c.lp_cnt;
    a.hc = c.lp_cnt + ntile;
    a.ctl = c.lp_cnt + 2 * ntile;
    a.dw = c.dw;
    a.invD = c.invD;
    a.status = c.status;
    a.limitp = c.counters + 3;
    a.trace = trace;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(std::min(c.lp_grid, 1 + ntasks));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = LP_SMEM;
    cfg.stream = c.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (c.pivot_mode)
        cudaLaunchKernelEx(&cfg, k_ldl_persist<true>, a);
    else
        cudaLaunchKernelEx(&cfg, k_ldl_persist<false>, a);
    c.launches++;
}

}  // namespace ecg

// Host-only diagnostic: every task of the persistent factorisation of n
// rows for a grid of `workers` CTAs in the scheduler's start order (the
// chain CTA's tasks included; the kernel's list is this order without
// them).  No GPU needed.
extern "C" int ecg_ldl_schedule(int n, int workers, unsigned* out, long long cap, long long* count)
{
    using namespace ecg;
    if (n < 1 || workers < 1 || !count) return -1;
    const int np = (n + LDL_NB - 1) / LDL_NB;
    if (np > 200) return -1;
    std::vector<unsigned> full, list;
    lp_schedule(np, workers, LpCost(), list, &full);
    *count = (long long)full.size();
    if (out && cap >= (long long)full.size()) std::copy(full.begin(), full.end(), out);
    return 0;
}
