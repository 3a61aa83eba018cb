// ecg_internal.h -- device-side state of one ECG context and the kernel
// launchers shared by the translation units of libecgb200.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>
#include "ecg_math.cuh"

namespace ecg {

// Pair tiles are 32 x 32 blocks of the lower triangle of the pair matrix.
constexpr int TILE = 32;
// Default poll limit of the bounded device waits of the triangular solves
// (each poll sleeps about 64 ns): a wait that runs out records
// ST_SOLVE_TIMEOUT and the call reports ECG_ECUDA.
constexpr int SOLVE_SPIN_LIMIT = 1 << 22;

// LDL^H block size (rows of one panel).
constexpr int LDL_NB = 64;
// Factorisations of at least this many new rows take the panels in pairs
// with rank-128 trailing updates (ldlh.cu); the buffers of unscaled panel
// rows hold a pair's rows per column.
constexpr int LDL_PAIR_MIN = 6000;
constexpr int LDL_VLD = 2 * LDL_NB;

// Number of 32 x 32 tiles with row-tile index in [Rlo, Rhi) and column-tile
// index 0..R (lower triangle including diagonal tiles).
inline long long tile_count(int Rlo, int Rhi)
{
    auto tri = [](long long r) { return r * (r + 1) / 2; };
    return tri(Rhi) - tri(Rlo);
}

// Number of k_cand_row tile shapes the autotuner chooses from.
constexpr int CAND_ROW_SHAPES = 5;
// k_pair_energy shapes (warps per 32 x 32 tile x minimum CTAs per SM) and
// k_adjoint shapes (minimum CTAs per SM) the autotuner chooses from.
constexpr int PAIR_SHAPES = 4;
constexpr int ADJ_SHAPES = 2;
// Columns (candidates) per work item of the batched triangular solves and
// the padding unit of the candidate column blocks.
constexpr int CAND_NC = 16;
constexpr int CAND_PAD = 64;
// Largest split of the inner dimension of the candidates' GEMM.
constexpr int CAND_KSPLIT = 4;

// Workspace of the batched candidate evaluation (allocated on first use).
// Column blocks are ldv x ccap, column j = candidate j, rows = base
// functions, then CAND_PAD spare columns that pad the active set; the
// border (row nbase+1) entries are separate vectors.  Per-column arrays use
// the stride ccap.
struct CandWork {
    int bcap = 0;            // candidate capacity (multiple of CAND_PAD)
    int ccap = 0;            // physical columns: bcap + CAND_PAD spare columns (stride of the per-column arrays)
    int ldv = 0;             // rows of the column blocks (ld rounded up to 64)
    int* cmap = nullptr;     // slot -> physical column of the active candidates (ccap)
    cd* Gm = nullptr;        // ld x ld: off-diagonal factor blocks premultiplied by Linv (solves)
    cd* Pk = nullptr;        // CAND_KSPLIT x ldv x 2 CAND_PAD: split-K partial sums of the GEMM
    double* par = nullptr;   // npt x bcap candidate parameters
    cd* bra = nullptr;       // bcap x NP
    cd* ket = nullptr;       // bcap x T x NP
    double* det = nullptr;   // bcap
    double* dS = nullptr;    // diagS of the candidate (its Re S_KK)
    double* mu = nullptr;    // M(K, K) = Re H_KK / diagS - lambda~
    cd* Mcol = nullptr;      // M(q, K), the bordered column of H - lambda~ S
    cd* Scol = nullptr;      // S(q, K)
    cd* Acol = nullptr;      // L0^-1 Mcol (unscaled new row of the factor)
    cd* Lcol = nullptr;      // U(q, K) = invD o Acol (column K of L^H)
    cd* V = nullptr;         // iterate v (rows < nbase)
    cd* W = nullptr;         // B v
    cd* Y = nullptr;         // forward solve
    cd* Z = nullptr;         // invD o Y
    cd* X = nullptr;         // backward solve (new x); Rayleigh products
    cd* X2 = nullptr;        // second Rayleigh product
    cd* brd = nullptr;       // border entries: [0] vK [1] wK [2] invDK [3] xK
    double* nd = nullptr;    // NormOfDiff, NormOfDiffPrev, t1, t2, E
    int* st = nullptr;       // active, iterations, ErrorCode, then the active count
    int* st_h = nullptr;     // pinned host mirror of st
    double* nd_h = nullptr;  // pinned host mirror of nd
    unsigned* flags = nullptr;  // work-item flags of the cooperative solves
    int nflags = 0;
    int* bstart = nullptr;   // device panel boundaries of the base factor
    int* bstart_h = nullptr; // pinned staging
    int* abort_word = nullptr;
    double* gpart = nullptr;  // candidate gradients: per (candidate, 128-row chunk) adjoint sums
    size_t gpart_n = 0;
    double* grad = nullptr;   // npt x bcap candidate gradients
    int solve_grid = 0;      // co-resident CTAs of the solve kernel
    int row_variant = -1;    // autotuned k_cand_row shape
    int tuned_n = 0, tuned_T = 0;
    struct IterGraph {
        std::vector<int> key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;
    };
    std::vector<IterGraph> graphs;
};

struct Ctx {
    int dev = 0;
    int n = 0, np = 0, npt = 0, T = 0;
    int ld = 0;          // leading dimension and capacity (max basis size)
    int max_nfo = 0;     // capacity of the plain derivative array Glob_D
    char method = 'I';   // 'I' (inverse iteration) or 'G' (generalised solver) storage
    SysParams sp{};
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // second stream of the LDL^H lookahead
    cudaEvent_t lev[3];            // LDL^H lookahead events (two in use)

    // Glob_* state, device resident
    double* params = nullptr;   // npt x ld, column-major (Glob_NonlinParam)
    cd* H = nullptr;            // ld x ld column-major (Glob_H)
    // The matrix the LDL^H factorisation and the inverse iterations work on:
    // Glob_H itself in 'I' contexts (H - lambda~ S in its lower triangle), a
    // separate ld x ld array in 'G' contexts, where it holds H - sigma S for
    // the shifts of the eigenvalue bisection and Glob_H keeps the 'G' layout.
    cd* F = nullptr;
    cd* S = nullptr;            // ld x ld column-major (Glob_S)
    double* diagS = nullptr;    // Glob_diagS
    double* diagH = nullptr;    // Glob_diagH
    cd* invD = nullptr;         // Glob_invD
    cd* c = nullptr;            // Glob_c (v of GHEPIIS, consumed)
    cd* x = nullptr;            // Glob_LastEigvector (x of GHEPIIS)
    cd* w = nullptr;            // GHEPIIS work vector
    cd* D = nullptr;            // Glob_D: 2npt x max_nfo x ld (plain gradient only)
    double* grad = nullptr;     // npt x ld gradient output

    // derived per-function data for the pair kernels
    double* Pd = nullptr;       // T x NMAX x NMAX permutation matrices (double, row-major)
    double* coef = nullptr;     // T coefficients (double)
    std::vector<int> yhy_h;     // host copy of Glob_YHYMatr (n x n x T column-major)
    std::vector<int> yhy_coef_h;  // host copy of Glob_YHYCoeff
    cd* bra = nullptr;          // ld x NP: Ck = A - iB packed (vech order)
    cd* ket = nullptr;          // ld x T x NP: P'AP + iP'BP packed
    double* detL = nullptr;     // ld

    // adjoint partial sums
    double* part = nullptr;
    size_t part_bytes = 0;

    // LDL^H workspace
    cd* dw = nullptr;           // working diagonal (ld)
    cd* linv = nullptr;         // ld x LDL_NB: inverse unit-lower diagonal blocks
    cd* lmf = nullptr;          // ld x LDL_NB: Linv_j U(j-1, j)^H per panel (forward solves)
    cd* lnb = nullptr;          // ld x LDL_NB: Linv_j^H U(j, j+1) per panel (backward solves)
    cd* vbuf = nullptr;         // 3 x LDL_VLD x ld: unscaled rows of a panel (pair) (rotating)
    int* status = nullptr;      // device status words (see ST_*)
    int* status_h = nullptr;    // pinned host mirror
    double* red = nullptr;      // reduction scratch for the solver (doubles)
    double* red_h = nullptr;    // pinned host mirror of the reduction results
    int* counters = nullptr;    // last-block counters [0,1], abort word [2], wait poll limit [3] of the solves
    int wait_limit = SOLVE_SPIN_LIMIT;
    int tune_pair = -1, tune_adj = -1;  // autotuned pair-kernel shapes (-1: not yet)
    float tune_pair_ms[PAIR_SHAPES] = {0}, tune_adj_ms[ADJ_SHAPES] = {0};
    int pivot_mode = 0;         // LDL^H pivots: 0 real (default), 1 complex as the reference keeps them
    cd* yv = nullptr;           // forward-solve result (ld)
    cd* zv = nullptr;           // D^-1 scaled forward result (ld)
    cd* spart = nullptr;        // per-CTA partial sums of the blocked solves
    double* colval = nullptr;   // per-column values of the quadratic forms (2 ld)
    int* dblk = nullptr;        // device copy of blk_start + end (ld + 2 ints)
    unsigned* flags = nullptr;  // per-panel ready flags of the cooperative solves (ld + 2)
    unsigned epoch = 0;         // value a panel flag takes when its panel is solved
    int coop_max_blocks = 0;    // co-resident CTAs of the cooperative solve kernels
    int coop_max_neigh = 0;     // the same with the neighbour products in shared memory
    std::vector<int> blk_start; // block starts of the current LDL^H factor
    // captured LDL^H factorisations, keyed by (m0, n, existing block starts)
    struct LdlGraph {
        std::vector<int> key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;  // kernel launches one replay performs
        unsigned* tasks = nullptr;  // task lists of a persistent factorisation (ldlp.cu), owned
        int ntasks = 0;
    };
    long long graph_launches = 0;
    std::vector<LdlGraph> ldl_graphs;
    int* bounds_h = nullptr;    // pinned staging of the panel boundaries (ld + 2)
    int fact_n = 0;             // rows covered by the current factor
    // persistent factorisation of whole matrices (ldlp.cu)
    int factor_mode = 0;        // 0: persistent kernel for m0 = 0, 1: one launch per panel step
    int lp_grid = 0;            // co-resident CTAs of the persistent kernel (0: not yet known)
    int lp_sms = 1;             // SMs of the device
    unsigned* lp_cnt = nullptr; // tile counters, then the next-task counter and the abort word
    size_t lp_cap = 0;          // capacity of lp_cnt (unsigned)
    unsigned* lp_direct = nullptr;  // task list of the uncaptured fallback, for lp_direct_n rows
    int lp_direct_n = 0, lp_direct_count = 0;

    // bookkeeping
    long long launches = 0;
    long long bytes_h2d = 0, bytes_d2h = 0;
    cudaEvent_t tev[2];
    bool timing = false;
    cudaEvent_t ev[16];
    double stage_ms[8] = {0};
    int last_numiter = 0;

    CandWork cand;           // batched candidate evaluation

    // 'G' path (ZHEGVX semantics by inertia bisection)
    int* gcnt = nullptr;     // device: [0] negative pivots, [1] first non-positive pivot (n = none)
    int* gcnt_h = nullptr;   // pinned host mirror
    double g_last_e = 0.0;   // last eigenvalue found, and its index
    int g_last_which = 0;
    int g_last_factorizations = 0;
};

enum StatusWord {
    ST_ZERO_PIVOT = 0,   // first zero pivot row + 1 (0 = none)
    ST_NONFINITE = 1,    // a non-finite pair element was produced
    ST_SOLVE_TIMEOUT = 2,  // a cooperative solve gave up waiting for a panel
    ST_COUNT = 8
};

// reduction slots in Ctx::red (doubles)
enum RedSlot {
    RD_NORMDIFF = 0,
    RD_T1 = 1,       // x^H B x
    RD_T2 = 2,       // x^H M x
    RD_XX = 3,       // x^H x
    RD_COUNT = 8
};

// ---- launchers (pair_kernels.cu) ----
int launch_prep(Ctx& c, int nfun);
int launch_pair_diag(Ctx& c, int r0, int r1, double approx_e, int deriv, int nfru);
int launch_pair_energy(Ctx& c, int r0, int r1, double approx_e);
int launch_pair_plain_grad(Ctx& c, int r0, int r1, int nfru, double approx_e);
int launch_adjoint(Ctx& c, int nfru, int nfa, double E);
int launch_plain_contract(Ctx& c, int nfo, int nfa, int nfru, double E);
int launch_term_batch(Ctx& c, int count, const double* pk, const double* pl, const int* term, int gradflag,
                      cd* hs, cd* dk, cd* dl);

int launch_cand_rows(Ctx& c, CandWork& cw, int nbase, int count, double approx_e, int variant);
// Pair tiles split over ranks: a range of the off-diagonal tile list of
// rows [r0, r1) (tile_count order), its packing, and the adjoint pass over
// a range with the gradient from all partials.
int launch_pair_energy_tiles(Ctx& c, int r0, int r1, double approx_e, long long t0, long long count);
int launch_tiles_copy(Ctx& c, int r0, int r1, long long t0, long long count, cd* buf, int dir);
int launch_adjoint_tiles(Ctx& c, int nfru, int nfa, double E, const cd* cvec, long long t0, long long count,
                         double* part);
int launch_adjoint_finish(Ctx& c, int nfru, int nfa, const double* part);
int adjoint_nv(int n);
// Gradients of the candidates' energies with respect to their own
// parameters from their final eigenpairs (border entry vK, x^H S x = t1).
int launch_cand_adjoint(Ctx& c, CandWork& cw, int nbase, int count, const cd* vK, const double* t1,
                        const double* energy, const int* err, double* grad);
// overlap penalty: part receives one partial sum per function nfru..nfa-1;
// mode 0 value only, 1 adds the reference's gradient to c.grad, 2 the exact one
int launch_penalty(Ctx& c, int nfru, int nfa, double t2, double pc, int mode, double* part);

// ---- batched candidates (cand.cu) ----
int eval_candidates(Ctx& c, int nbase, int count, const double* cand_host, double approx_e, double tol,
                    int max_iter, double* energies, int* errcodes, int* num_iter, double* rel_acc,
                    double* grad = nullptr);
void cand_free(CandWork& cw);

// ---- expectation values (expc.cu) ----
// The accumulation loop of ExpectationValuesG over functions 1..nbasis for
// a term list (Pbra_t, Pket_t column-major n x n, weights coef1_t coef2_t).
int expectation_values(Ctx& c, int nbasis, const double* masses, int nterms, const int* pbra, const int* pket,
                       const double* coef1, const double* coef2, int err_mult, double energy, const cd* c_host,
                       int ncf, const double* cf_grid, int ndens, const double* dens_grid, double* values,
                       double* errors, double* cf, double* dens);

// ---- 'G' path (gpath.cu kernels; driver energy_ga in ecg_abi.cu) ----
int g_shift(Ctx& c, const cd* A, const cd* B, const double* dA, const double* dB, int n, double sigma);
int g_mirror_s(Ctx& c, int n);
int g_inertia(Ctx& c, int n);

// ---- launchers (ldlh.cu) ----
int ldlh_factor(Ctx& c, int m0, int n);

// ---- persistent factorisation (ldlp.cu) ----
int ldlp_grid(Ctx& c);
int ldlp_tasks(Ctx& c, int n, unsigned** tasks, int* count);
long long ldlp_task_total(int n);
int ldlp_reserve(Ctx& c, int np);
void ldlp_enqueue(Ctx& c, int n, const unsigned* tasks, int ntasks, unsigned long long* trace = nullptr);
// One persistent factorisation of rows 0..n-1 of the current matrix with a
// per-task timing record (4 values per task, see ecg_factor_trace).
int ldlh_factor_traced(Ctx& c, int n, unsigned long long* out, long long cap, long long* count);

// ---- launchers (invit.cu) ----
int invit_step(Ctx& c, int n, bool first);
int invit_rayleigh(Ctx& c, int n);
int vec_scale(Ctx& c, cd* v, int n, double s);

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? 0 : -2; }

}  // namespace ecg
