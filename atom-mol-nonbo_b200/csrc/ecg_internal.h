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
// LDL^H block size (rows of one panel).
constexpr int LDL_NB = 64;

// Number of 32 x 32 tiles with row-tile index in [Rlo, Rhi) and column-tile
// index 0..R (lower triangle including diagonal tiles).
inline long long tile_count(int Rlo, int Rhi)
{
    auto tri = [](long long r) { return r * (r + 1) / 2; };
    return tri(Rhi) - tri(Rlo);
}

struct Ctx {
    int dev = 0;
    int n = 0, np = 0, npt = 0, T = 0;
    int ld = 0;          // leading dimension and capacity (max basis size)
    int max_nfo = 0;     // capacity of the plain derivative array Glob_D
    char method = 'I';   // 'I' (inverse iteration) or 'G' (generalised solver) storage
    SysParams sp{};
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;   // second stream of the LDL^H lookahead
    cudaEvent_t lev[2];            // LDL^H lookahead events

    // Glob_* state, device resident
    double* params = nullptr;   // npt x ld, column-major (Glob_NonlinParam)
    cd* H = nullptr;            // ld x ld column-major (Glob_H)
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
    cd* bra = nullptr;          // ld x NP: Ck = A - iB packed (vech order)
    cd* ket = nullptr;          // ld x T x NP: P'AP + iP'BP packed
    double* detL = nullptr;     // ld

    // adjoint partial sums
    double* part = nullptr;
    size_t part_bytes = 0;

    // LDL^H workspace
    cd* dw = nullptr;           // working diagonal (ld)
    cd* linv = nullptr;         // ld x LDL_NB: inverse unit-lower diagonal blocks
    cd* vbuf = nullptr;         // 2 x LDL_NB x ld: unscaled panel rows (ping-pong)
    int* status = nullptr;      // device status words (see ST_*)
    int* status_h = nullptr;    // pinned host mirror
    double* red = nullptr;      // reduction scratch for the solver (doubles)
    double* red_h = nullptr;    // pinned host mirror of the reduction results
    int* counters = nullptr;    // last-block counters for the triangular solves
    cd* yv = nullptr;           // forward-solve result (ld)
    cd* zv = nullptr;           // D^-1 scaled forward result (ld)
    cd* spart = nullptr;        // per-CTA partial sums of the blocked solves
    double* colval = nullptr;   // per-column values of the quadratic forms (2 ld)
    int* dblk = nullptr;        // device copy of blk_start + end (ld + 2 ints)
    unsigned* flags = nullptr;  // per-panel ready flags of the cooperative solves (ld + 2)
    unsigned epoch = 0;         // value a panel flag takes when its panel is solved
    int coop_max_blocks = 0;    // co-resident CTAs of the cooperative solve kernels
    std::vector<int> blk_start; // block starts of the current LDL^H factor
    // captured LDL^H factorisations, keyed by (m0, n, existing block starts)
    struct LdlGraph {
        std::vector<int> key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;  // kernel launches one replay performs
    };
    long long graph_launches = 0;
    std::vector<LdlGraph> ldl_graphs;
    int* bounds_h = nullptr;    // pinned staging of the panel boundaries (ld + 2)
    int fact_n = 0;             // rows covered by the current factor

    // bookkeeping
    long long launches = 0;
    long long bytes_h2d = 0, bytes_d2h = 0;
    cudaEvent_t tev[2];
    bool timing = false;
    cudaEvent_t ev[16];
    double stage_ms[8] = {0};
    int last_numiter = 0;
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

// ---- launchers (ldlh.cu) ----
int ldlh_factor(Ctx& c, int m0, int n);

// ---- launchers (invit.cu) ----
int invit_step(Ctx& c, int n, bool first);
int invit_rayleigh(Ctx& c, int n);
int vec_scale(Ctx& c, cd* v, int n, double s);

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? 0 : -2; }

}  // namespace ecg
