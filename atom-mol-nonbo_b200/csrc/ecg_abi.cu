// ecg_abi.cu -- host side of libecgb200.so: context lifetime, the GHEPIIS
// driver and the EnergyIA / EnergyIB glue behind the C ABI in ecg_abi.h.
#include <float.h>
#include <stdio.h>
#include <stdlib.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <new>
#include "../../include/ecg_abi.h"
#include "ecg_internal.h"

using namespace ecg;

struct ecg_ctx {
    Ctx c;
};

#define CK(call)                                  \
    do {                                          \
        if ((call) != cudaSuccess) {              \
            cudaGetLastError();                   \
            return ECG_ECUDA;                     \
        }                                         \
    } while (0)
#define CKR(expr)                                 \
    do {                                          \
        const int _r = (expr);                    \
        if (_r != 0) return _r == -3 ? ECG_ENOMEM : (_r == -1 ? ECG_EARG : ECG_ECUDA); \
    } while (0)

namespace {

constexpr int SOLVE_G_MAX = 64;

// ECG_TRACE=1 in the environment prints the residual of every inverse
// iteration to stderr (the reference's only convergence log is the
// eigenvalue-tolerance bookkeeping of src/workproc.f90:1994-1995).
bool trace_on()
{
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("ECG_TRACE");
        on = (e && e[0] == '1') ? 1 : 0;
    }
    return on == 1;
}

template <typename T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) return 0;
    if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return ECG_ENOMEM;
    }
    return 0;
}

void free_ctx(Ctx& c)
{
    if (c.F && c.F != c.H) cudaFree(c.F);
    if (c.gcnt_h) cudaFreeHost(c.gcnt_h);
    void* ptrs[] = {c.gcnt, c.params, c.H, c.S, c.diagS, c.diagH, c.invD, c.c, c.x, c.w, c.D, c.grad, c.Pd, c.coef,
                    c.bra, c.ket, c.detL, c.part, c.dw, c.linv, c.lmf, c.lnb, c.vbuf, c.status, c.red, c.counters, c.yv,
                    c.zv, c.spart, c.colval, c.dblk, c.flags};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto& g : c.ldl_graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.tasks) cudaFree(g.tasks);
    }
    c.ldl_graphs.clear();
    if (c.lp_cnt) cudaFree(c.lp_cnt);
    if (c.lp_direct) cudaFree(c.lp_direct);
    cand_free(c.cand);
    if (c.bounds_h) cudaFreeHost(c.bounds_h);
    if (c.status_h) cudaFreeHost(c.status_h);
    if (c.red_h) cudaFreeHost(c.red_h);
    if (c.stream) {
        for (int i = 0; i < 16; i++) cudaEventDestroy(c.ev[i]);
        for (int i = 0; i < 2; i++) cudaEventDestroy(c.tev[i]);
        for (int i = 0; i < 3; i++) cudaEventDestroy(c.lev[i]);
        if (c.side) cudaStreamDestroy(c.side);
        cudaStreamDestroy(c.stream);
    }
}

void mark(Ctx& c, int i)
{
    if (c.timing) cudaEventRecord(c.ev[i], c.stream);
}

double elapsed(Ctx& c, int a, int b)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev[a], c.ev[b]) != cudaSuccess) {
        cudaGetLastError();
        return 0.0;
    }
    return ms;
}

int read_red(Ctx& c)
{
    CK(cudaMemcpyAsync(c.red_h, c.red, RD_COUNT * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.bytes_d2h += RD_COUNT * sizeof(double) + ST_COUNT * sizeof(int);
    CK(cudaStreamSynchronize(c.stream));
    // a cooperative solve that gave up waiting leaves an unusable step
    if (c.status_h[ST_SOLVE_TIMEOUT]) return ECG_ECUDA;
    return 0;
}

int compute_hs(Ctx& c, int nmin, int nmax, double approx_e)
{
    if (nmin < 1 || nmax < nmin || nmax > c.ld) return ECG_EARG;
    CKR(launch_prep(c, nmax));
    CKR(launch_pair_diag(c, nmin - 1, nmax, approx_e, 0, 0));
    CKR(launch_pair_energy(c, nmin - 1, nmax, approx_e));
    return 0;
}

int compute_hsd(Ctx& c, int nmin, int nmax, int nfru, double approx_e)
{
    if (nmin < 1 || nmax < nmin || nmax > c.ld || nfru < 0 || nfru >= nmin) return ECG_EARG;
    if (nmax - nfru > c.max_nfo) return ECG_EARG;
    if (!c.D) {
        const size_t cnt = (size_t)2 * c.npt * c.max_nfo * c.ld;
        if (dalloc(&c.D, cnt)) return ECG_ENOMEM;
    }
    CKR(launch_prep(c, nmax));
    CKR(launch_pair_diag(c, nmin - 1, nmax, approx_e, 1, nfru));
    CKR(launch_pair_plain_grad(c, nmin - 1, nmax, nfru, approx_e));
    return 0;
}

// GHEPIIS, src/linalg.f90:1781-1926, on the factor matrix F (Glob_H in 'I'
// contexts).
int ghepiis_core(Ctx& c, int k, int n, double apprlambda, double tol, int max_iter, int specif_norm,
                 double* lambda, double* rel_acc, int* num_iter)
{
    if (k < 1 || n < k || n > c.ld || max_iter < 0) return ECG_EARG;
    *rel_acc = DBL_MAX;
    *num_iter = 0;
    CK(cudaMemsetAsync(c.status, 0, ST_COUNT * sizeof(int), c.stream));
    CKR(ldlh_factor(c, k - 1, n));
    CK(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.bytes_d2h += ST_COUNT * sizeof(int);
    CK(cudaStreamSynchronize(c.stream));
    mark(c, 2);
    if (c.status_h[ST_SOLVE_TIMEOUT]) {
        // a bounded wait of the factorisation ran out: no factor
        c.fact_n = 0;
        c.blk_start.clear();
        return ECG_ECUDA;
    }
    if (c.status_h[ST_ZERO_PIVOT] != 0) {
        // LDLHF returned ErrorCode = 1 (src/linalg.f90:377-380); the factor
        // is incomplete, so no row of it may be reused.
        c.fact_n = 0;
        c.blk_start.clear();
        mark(c, 3);
        return ECG_ESINGULAR;
    }
    bool notconverged = true;
    double nd = 0.0, prev = DBL_MAX;
    int it = 0;
    while (notconverged && it < max_iter) {
        CKR(invit_step(c, n, it == 0));
        CKR(read_red(c));
        nd = c.red_h[RD_NORMDIFF];
        if (trace_on()) fprintf(stderr, "ecg: GHEPIIS(%d,%d) iteration %d NormOfDiff %.3e\n", k, n, it + 1, nd);
        if (tol > 0.0) {
            if (nd <= tol) notconverged = false;
        } else {
            if (nd > prev && nd <= fabs(tol)) notconverged = false;
            prev = nd;
        }
        it++;
    }
    mark(c, 3);
    *rel_acc = nd;
    *num_iter = it;
    c.last_numiter = it;
    CKR(invit_rayleigh(c, n));
    CKR(read_red(c));
    const double t1 = c.red_h[RD_T1], t2 = c.red_h[RD_T2];
    *lambda = t2 / t1 + apprlambda;
    if (specif_norm == 0) {
        CKR(vec_scale(c, c.x, n, 1.0 / sqrt(t1)));
    } else if (specif_norm == 1) {
        CKR(vec_scale(c, c.x, n, 1.0 / sqrt(c.red_h[RD_XX])));
    }
    return notconverged ? ECG_ENOCONV : ECG_OK;
}

int ghepiis(Ctx& c, int k, int n, double apprlambda, double tol, int max_iter, int specif_norm, double* lambda,
            double* rel_acc, int* num_iter)
{
    if (c.method != 'I') return ECG_EARG;
    return ghepiis_core(c, k, n, apprlambda, tol, max_iter, specif_norm, lambda, rel_acc, num_iter);
}

// ---------------------------------------------------------------------------
// 'G' path: EnergyGA / EnergyGAM (src/workproc.f90:1697-1838).  The reference
// mirrors H and S into full Hermitian matrices and calls ZHEGVX(ITYPE=1,
// JOBZ, RANGE='I', IL=IU=which) (src/workproc.f90:1750): Cholesky of S (INFO
// = n + i when its leading minor of order i is not positive definite), then
// the which-th eigenvalue.  Here: the LDL^H pivots of S give the same test;
// nu(sigma) = number of negative pivots of LDL^H(H - sigma S) = number of
// eigenvalues below sigma (Sylvester's law of inertia) brackets the which-th
// eigenvalue, bisection isolates it (nu(lo) = which - 1, nu(hi) = which),
// and GHEPIIS at the bracket's centre converges to it, since every other
// eigenvalue lies outside the bracket and so farther from its centre.
// ---------------------------------------------------------------------------
constexpr int G_MAX_FACT = 400;   // bound on the factorisations of one call
constexpr int G_EXTRA_BISECT = 10;  // halvings after isolation: faster inverse iteration

// nu(sigma) into *nu; *zero = 1 when a pivot was exactly zero
int g_count(Ctx& c, int n, double sigma, int* nu, int* zero)
{
    CKR(g_shift(c, c.H, c.S, c.diagH, nullptr, n, sigma));
    CK(cudaMemsetAsync(c.status, 0, ST_COUNT * sizeof(int), c.stream));
    CKR(ldlh_factor(c, 0, n));
    CKR(g_inertia(c, n));
    CK(cudaMemcpyAsync(c.gcnt_h, c.gcnt, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.g_last_factorizations++;
    if (c.status_h[ST_SOLVE_TIMEOUT]) return ECG_ECUDA;
    *nu = c.gcnt_h[0];
    *zero = c.status_h[ST_ZERO_PIVOT] != 0;
    return 0;
}

int energy_ga(Ctx& c, int nmin, int nmax, int needed, int which, int want_vector, double* energy)
{
    if (c.method != 'G') return ECG_EARG;
    if (nmin < 1 || nmax < nmin || nmax > c.ld || which < 1 || which > nmax) return ECG_EARG;
    c.g_last_factorizations = 0;
    if (needed) CKR(compute_hs(c, nmin, nmax, 0.0));
    const int n = nmax;
    if (n == 1) {  // EnergyGA's one-function branch: E = Glob_diagH(1)
        double h;
        CK(cudaMemcpyAsync(&h, c.diagH, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        const cd one{1.0, 0.0};
        if (want_vector) CK(cudaMemcpyAsync(c.c, &one, sizeof(cd), cudaMemcpyHostToDevice, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        *energy = h;
        return ECG_OK;
    }
    CKR(g_mirror_s(c, n));
    // S positive definite?  (ZPOTRF inside ZHEGVX: INFO = n + i)
    CKR(g_shift(c, c.S, nullptr, nullptr, nullptr, n, 0.0));
    CK(cudaMemsetAsync(c.status, 0, ST_COUNT * sizeof(int), c.stream));
    CKR(ldlh_factor(c, 0, n));
    CKR(g_inertia(c, n));
    CK(cudaMemcpyAsync(c.gcnt_h, c.gcnt, 2 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(c.status_h, c.status, ST_COUNT * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.g_last_factorizations++;
    if (c.status_h[ST_SOLVE_TIMEOUT]) return ECG_ECUDA;
    if (c.gcnt_h[1] < n) return n + c.gcnt_h[1] + 1;
    // initial bracket around the previous eigenvalue, or below min diag(H)
    // (the lowest eigenvalue is at most every diagonal Rayleigh quotient)
    double center, delta;
    if (c.g_last_which == which) {
        center = c.g_last_e;
        delta = 1e-6 * std::max(1.0, fabs(center));
    } else {
        std::vector<double> dh(n);
        CK(cudaMemcpyAsync(dh.data(), c.diagH, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        center = *std::min_element(dh.begin(), dh.end());
        delta = 1e-3 * std::max(1.0, fabs(center));
    }
    int nu = 0, zero = 0;
    double lo = center - delta, hi = center + delta;
    int nlo, nhi;
    auto count = [&](double& s, int* v) -> int {
        // an exactly zero pivot leaves the count undefined: move sigma by a few ulps
        for (int tries = 0; tries < 8; tries++) {
            const int r = g_count(c, n, s, v, &zero);
            if (r) return r;
            if (!zero) return 0;
            s = s + (fabs(s) + 1e-300) * 1e-14 * (tries + 1);
        }
        return ECG_ENOCONV;
    };
    int r;
    if ((r = count(lo, &nlo))) return r;
    for (double d = delta; nlo >= which; ) {
        d *= 4.0;
        lo = center - d;
        if ((r = count(lo, &nlo))) return r;
        if (c.g_last_factorizations > G_MAX_FACT) return ECG_ENOCONV;
    }
    if ((r = count(hi, &nhi))) return r;
    for (double d = delta; nhi < which; ) {
        d *= 4.0;
        hi = center + d;
        if ((r = count(hi, &nhi))) return r;
        if (c.g_last_factorizations > G_MAX_FACT) return ECG_ENOCONV;
    }
    // bisect until the bracket holds the which-th eigenvalue alone, then a
    // few halvings more
    int extra = 0;
    for (;;) {
        const bool isolated = (nlo == which - 1) && (nhi == which);
        if (isolated && extra >= G_EXTRA_BISECT) break;
        if (hi - lo <= 4.0 * DBL_EPSILON * std::max(fabs(lo), fabs(hi))) break;
        if (c.g_last_factorizations > G_MAX_FACT) return ECG_ENOCONV;
        double mid = 0.5 * (lo + hi);
        if ((r = count(mid, &nu))) return r;
        if (nu >= which) {
            hi = mid;
            nhi = nu;
        } else {
            lo = mid;
            nlo = nu;
        }
        if (isolated) extra++;
    }
    // inverse iteration at the centre of the isolating bracket
    double sigma = 0.5 * (lo + hi);
    CKR(g_shift(c, c.H, c.S, c.diagH, nullptr, n, sigma));
    if (c.g_last_which > 0) {
        CK(cudaMemcpyAsync(c.c, c.x, (size_t)n * sizeof(cd), cudaMemcpyDeviceToDevice, c.stream));
    } else {
        std::vector<cd> ones(n, cd{1.0, 0.0});
        CK(cudaMemcpyAsync(c.c, ones.data(), (size_t)n * sizeof(cd), cudaMemcpyHostToDevice, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    }
    double lam = 0.0, ra = 0.0;
    int it = 0;
    const int e = ghepiis_core(c, 1, n, sigma, 1e-12, 20, want_vector ? 0 : -1, &lam, &ra, &it);
    c.g_last_factorizations++;
    if (e < 0) return e;
    if (e == ECG_ESINGULAR) return ECG_ENOCONV;
    // the converged eigenvalue is the bracket's; otherwise the bisection's own estimate
    *energy = (lam >= lo && lam <= hi) ? lam : sigma;
    c.last_numiter = it;
    if (want_vector) CK(cudaMemcpyAsync(c.c, c.x, (size_t)n * sizeof(cd), cudaMemcpyDeviceToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.g_last_e = *energy;
    c.g_last_which = which;
    return ECG_OK;
}

int single_function_energy(Ctx& c, double approx_e, double* energy)
{
    cd h11;
    CK(cudaMemcpyAsync(&h11, c.H, sizeof(cd), cudaMemcpyDeviceToHost, c.stream));
    c.bytes_d2h += sizeof(cd);
    CK(cudaStreamSynchronize(c.stream));
    *energy = h11.x + approx_e;
    const cd one{1.0, 0.0};
    CK(cudaMemcpyAsync(c.c, &one, sizeof(cd), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return 0;
}

void finish_timing(Ctx& c, bool grad)
{
    if (!c.timing) return;
    cudaStreamSynchronize(c.stream);
    c.stage_ms[0] = elapsed(c, 0, 1);
    c.stage_ms[1] = elapsed(c, 1, 2);
    c.stage_ms[2] = elapsed(c, 2, 3);
    c.stage_ms[3] = grad ? elapsed(c, 3, 4) : 0.0;
}

int energy_ib_common(Ctx& c, int nfru, int nfa, int needed, double approx_e, double tol, int max_iter,
                     double* energy, double* grad_host, int* num_iter, bool adjoint)
{
    if (c.method != 'I') return ECG_EARG;
    if (nfru < 0 || nfa <= nfru || nfa > c.ld) return ECG_EARG;
    const int nfo = nfa - nfru;
    mark(c, 0);
    if (needed) {
        const int r = adjoint ? compute_hs(c, nfru + 1, nfa, approx_e) : compute_hsd(c, nfru + 1, nfa, nfru, approx_e);
        if (r) return r;
    } else if (!adjoint && !c.D) {
        return ECG_EARG;
    }
    mark(c, 1);
    int err = 0;
    if (nfa == 1) {
        mark(c, 2);
        const int r = single_function_energy(c, approx_e, energy);
        if (r) return r;
        *num_iter = 1;
        mark(c, 3);
    } else {
        CK(cudaMemcpyAsync(c.c, c.x, (size_t)nfa * sizeof(cd), cudaMemcpyDeviceToDevice, c.stream));
        double lam = 0.0, ra = 0.0;
        int it = 0;
        err = ghepiis(c, nfru + 1, nfa, approx_e, tol, max_iter, 0, &lam, &ra, &it);
        if (err < 0) return err;
        if (err == ECG_ESINGULAR) {
            *num_iter = 0;
            return err;
        }
        *energy = lam;
        *num_iter = it;
        // Glob_c(1:nfa) = Glob_LastEigvector(1:nfa), src/workproc.f90:2114
        CK(cudaMemcpyAsync(c.c, c.x, (size_t)nfa * sizeof(cd), cudaMemcpyDeviceToDevice, c.stream));
    }
    if (adjoint) {
        CKR(launch_adjoint(c, nfru, nfa, *energy));
    } else {
        CKR(launch_plain_contract(c, nfo, nfa, nfru, *energy));
    }
    mark(c, 4);
    if (grad_host) {
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
        c.bytes_d2h += (long long)nfo * c.npt * sizeof(double);
    }
    CK(cudaStreamSynchronize(c.stream));
    finish_timing(c, true);
    return err;
}

}  // namespace

extern "C" {

int ecg_ctx_create(int n, const double* mass_matrix_host, const double* charges_host, int nterms,
                   const int* yhy_mats_host, const int* yhy_coeffs_host, int ld, int max_nfo, char method,
                   int device, ecg_ctx** out)
{
    if (!out) return ECG_EARG;
    *out = nullptr;
    if (n < 2 || n > NMAX || nterms < 1 || nterms > TMAX || ld < 1 || max_nfo < 0 || max_nfo > ld) return ECG_EARG;
    if (method != 'I' && method != 'G') return ECG_EARG;
    if (!mass_matrix_host || !charges_host || !yhy_mats_host || !yhy_coeffs_host) return ECG_EARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return ECG_ENODEV;
    }
    if (device < 0 || device >= ndev) return ECG_EARG;
    CK(cudaSetDevice(device));
    ecg_ctx* h = new (std::nothrow) ecg_ctx();
    if (!h) return ECG_ENOMEM;
    Ctx& c = h->c;
    c.dev = device;
    c.n = n;
    c.np = n * (n + 1) / 2;
    c.npt = 2 * c.np;
    c.T = nterms;
    c.ld = ld;
    c.max_nfo = max_nfo;
    c.method = method;
    memset(&c.sp, 0, sizeof(c.sp));
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) c.sp.M[i * NMAX + j] = mass_matrix_host[i + j * n];
    c.sp.q0 = charges_host[0];
    for (int i = 0; i < n; i++) c.sp.q[i] = charges_host[1 + i];
    c.sp.two_r3n2 = pow(2.0, (3 * n) / 2.0);
    c.sp.n = n;
    c.sp.T = nterms;
    std::vector<double> P((size_t)nterms * NMAX * NMAX, 0.0), cf(nterms);
    for (int t = 0; t < nterms; t++) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) P[((size_t)t * NMAX + i) * NMAX + j] = yhy_mats_host[(size_t)t * n * n + i + j * n];
        cf[t] = yhy_coeffs_host[t];
    }
    c.yhy_h.assign(yhy_mats_host, yhy_mats_host + (size_t)nterms * n * n);
    c.yhy_coef_h.assign(yhy_coeffs_host, yhy_coeffs_host + nterms);
    int r = 0;
    // the context's stream carries the LDL^H panel chain; its higher
    // priority lets the chain's CTAs take SMs ahead of the bulk trailing
    // updates queued on the side stream
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c.stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return ECG_ECUDA;
    }
    for (int i = 0; i < 16; i++) cudaEventCreate(&c.ev[i]);
    for (int i = 0; i < 2; i++) cudaEventCreate(&c.tev[i]);
    for (int i = 0; i < 3; i++) cudaEventCreateWithFlags(&c.lev[i], cudaEventDisableTiming);
    if (cudaStreamCreateWithPriority(&c.side, cudaStreamNonBlocking, prio_lo) != cudaSuccess) {
        cudaGetLastError();
        free_ctx(c);
        delete h;
        return ECG_ECUDA;
    }
    const size_t L = (size_t)ld;
    r |= dalloc(&c.params, (size_t)c.npt * L);
    r |= dalloc(&c.H, L * L);
    r |= dalloc(&c.S, L * L);
    if (method == 'G')
        r |= dalloc(&c.F, L * L);
    else
        c.F = c.H;
    r |= dalloc(&c.gcnt, (size_t)4);
    r |= dalloc(&c.diagS, L);
    r |= dalloc(&c.diagH, L);
    r |= dalloc(&c.invD, L);
    r |= dalloc(&c.c, L);
    r |= dalloc(&c.x, L);
    r |= dalloc(&c.w, L);
    r |= dalloc(&c.yv, L);
    r |= dalloc(&c.zv, L);
    r |= dalloc(&c.grad, (size_t)c.npt * L);
    r |= dalloc(&c.Pd, P.size());
    r |= dalloc(&c.coef, (size_t)nterms);
    r |= dalloc(&c.bra, L * c.np);
    r |= dalloc(&c.ket, L * nterms * c.np);
    r |= dalloc(&c.detL, L);
    r |= dalloc(&c.dw, L);
    r |= dalloc(&c.linv, L * LDL_NB);
    r |= dalloc(&c.lmf, L * LDL_NB);
    r |= dalloc(&c.lnb, L * LDL_NB);
    r |= dalloc(&c.vbuf, 3 * L * LDL_VLD);
    r |= dalloc(&c.status, (size_t)ST_COUNT);
    r |= dalloc(&c.red, (size_t)RD_COUNT);
    r |= dalloc(&c.counters, (size_t)4);
    r |= dalloc(&c.spart, (size_t)SOLVE_G_MAX * LDL_NB);
    r |= dalloc(&c.colval, 2 * L);
    r |= dalloc(&c.dblk, L + 2);
    r |= dalloc(&c.flags, L + 2);
    if (!r) {
        if (cudaMallocHost((void**)&c.status_h, ST_COUNT * sizeof(int)) != cudaSuccess ||
            cudaMallocHost((void**)&c.bounds_h, (L + 2) * sizeof(int)) != cudaSuccess ||
            cudaMallocHost((void**)&c.red_h, RD_COUNT * sizeof(double)) != cudaSuccess ||
            cudaMallocHost((void**)&c.gcnt_h, 4 * sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            r = ECG_ENOMEM;
        }
    }
    if (r) {
        free_ctx(c);
        delete h;
        return ECG_ENOMEM;
    }
    bool ok = cudaMemcpy(c.Pd, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemcpy(c.coef, cf.data(), cf.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(c.H, 0, L * L * sizeof(cd)) == cudaSuccess &&
              cudaMemset(c.S, 0, L * L * sizeof(cd)) == cudaSuccess &&
              cudaMemset(c.counters, 0, 4 * sizeof(int)) == cudaSuccess &&
              cudaMemcpy(c.counters + 3, &c.wait_limit, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMemset(c.flags, 0, (L + 2) * sizeof(unsigned)) == cudaSuccess &&
              cudaMemset(c.status, 0, ST_COUNT * sizeof(int)) == cudaSuccess &&
              cudaMemset(c.c, 0, L * sizeof(cd)) == cudaSuccess && cudaMemset(c.x, 0, L * sizeof(cd)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        free_ctx(c);
        delete h;
        return ECG_ECUDA;
    }
    *out = h;
    return ECG_OK;
}

int ecg_ctx_destroy(ecg_ctx* ctx)
{
    if (!ctx) return ECG_EARG;
    cudaSetDevice(ctx->c.dev);
    cudaStreamSynchronize(ctx->c.stream);
    free_ctx(ctx->c);
    delete ctx;
    return ECG_OK;
}

int ecg_set_params(ecg_ctx* ctx, const double* params_host, int first, int count)
{
    if (!ctx || !params_host || first < 1 || count < 0 || first - 1 + count > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    CK(cudaMemcpyAsync(c.params + (size_t)(first - 1) * c.npt, params_host, (size_t)count * c.npt * sizeof(double),
                       cudaMemcpyHostToDevice, c.stream));
    c.bytes_h2d += (long long)count * c.npt * sizeof(double);
    return ECG_OK;
}

int ecg_set_params_device(ecg_ctx* ctx, const double* params_dev, int first, int count)
{
    if (!ctx || !params_dev || first < 1 || count < 0 || first - 1 + count > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    CK(cudaMemcpyAsync(c.params + (size_t)(first - 1) * c.npt, params_dev, (size_t)count * c.npt * sizeof(double),
                       cudaMemcpyDeviceToDevice, c.stream));
    return ECG_OK;
}

int ecg_pair_tiles(ecg_ctx* ctx, int nmin, int nmax, long long* ntiles)
{
    if (!ctx || !ntiles || nmin < 1 || nmax < nmin || nmax > ctx->c.ld) return ECG_EARG;
    *ntiles = tile_count((nmin - 1) / TILE, (nmax + TILE - 1) / TILE);
    return ECG_OK;
}

static bool tile_range_ok(Ctx& c, int nmin, int nmax, long long first, long long count)
{
    if (nmin < 1 || nmax < nmin || nmax > c.ld || first < 0 || count < 0) return false;
    return first + count <= tile_count((nmin - 1) / TILE, (nmax + TILE - 1) / TILE) && count < (1LL << 31);
}

int ecg_compute_mat_elem_tiles(ecg_ctx* ctx, int nmin, int nmax, double approx_energy, long long first,
                               long long count)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    if (!tile_range_ok(c, nmin, nmax, first, count)) return ECG_EARG;
    CKR(launch_prep(c, nmax));
    CKR(launch_pair_diag(c, nmin - 1, nmax, approx_energy, 0, 0));
    CKR(launch_pair_energy_tiles(c, nmin - 1, nmax, approx_energy, first, count));
    return ECG_OK;
}

int ecg_pack_tiles(ecg_ctx* ctx, int nmin, int nmax, long long first, long long count, void* packed_dev)
{
    if (!ctx || (!packed_dev && count > 0)) return ECG_EARG;
    Ctx& c = ctx->c;
    if (!tile_range_ok(c, nmin, nmax, first, count)) return ECG_EARG;
    CKR(launch_tiles_copy(c, nmin - 1, nmax, first, count, static_cast<cd*>(packed_dev), 0));
    return ECG_OK;
}

int ecg_unpack_tiles(ecg_ctx* ctx, int nmin, int nmax, long long first, long long count, const void* packed_dev)
{
    if (!ctx || (!packed_dev && count > 0)) return ECG_EARG;
    Ctx& c = ctx->c;
    if (!tile_range_ok(c, nmin, nmax, first, count)) return ECG_EARG;
    CKR(launch_tiles_copy(c, nmin - 1, nmax, first, count, static_cast<cd*>(const_cast<void*>(packed_dev)), 1));
    return ECG_OK;
}

int ecg_adjoint_part_doubles(ecg_ctx* ctx, long long* per_tile)
{
    if (!ctx || !per_tile) return ECG_EARG;
    *per_tile = 2LL * TILE * adjoint_nv(ctx->c.n);
    return ECG_OK;
}

int ecg_adjoint_tiles(ecg_ctx* ctx, int nfru, int nfa, double energy, long long first, long long count,
                      void* part_dev)
{
    if (!ctx || (!part_dev && count > 0)) return ECG_EARG;
    Ctx& c = ctx->c;
    if (nfru < 0 || !tile_range_ok(c, nfru + 1, nfa, first, count)) return ECG_EARG;
    CKR(launch_adjoint_tiles(c, nfru, nfa, energy, c.x, first, count, static_cast<double*>(part_dev)));
    return ECG_OK;
}

int ecg_adjoint_finish(ecg_ctx* ctx, int nfru, int nfa, const void* part_dev, double* grad_host)
{
    if (!ctx || !part_dev) return ECG_EARG;
    Ctx& c = ctx->c;
    if (nfru < 0 || nfa <= nfru || nfa > c.ld) return ECG_EARG;
    CKR(launch_adjoint_finish(c, nfru, nfa, static_cast<const double*>(part_dev)));
    if (grad_host) {
        const int nfo = nfa - nfru;
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
        c.bytes_d2h += (long long)nfo * c.npt * sizeof(double);
    }
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_get_tuning(ecg_ctx* ctx, int* pair_shape, int* adjoint_shape, int* cand_row_shape, double* times_ms)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    if (pair_shape) *pair_shape = c.tune_pair;
    if (adjoint_shape) *adjoint_shape = c.tune_adj;
    if (cand_row_shape) *cand_row_shape = c.cand.row_variant;
    if (times_ms) {
        for (int v = 0; v < PAIR_SHAPES; v++) times_ms[v] = c.tune_pair_ms[v];
        for (int v = 0; v < ADJ_SHAPES; v++) times_ms[PAIR_SHAPES + v] = c.tune_adj_ms[v];
    }
    return ECG_OK;
}

int ecg_set_pivot_mode(ecg_ctx* ctx, int mode)
{
    if (!ctx || mode < 0 || mode > 1) return ECG_EARG;
    Ctx& c = ctx->c;
    if (c.pivot_mode != mode) {
        c.pivot_mode = mode;
        // a factor made with the other pivots is not reused
        c.fact_n = 0;
        c.blk_start.clear();
    }
    return ECG_OK;
}

int ecg_set_factor_mode(ecg_ctx* ctx, int mode)
{
    if (!ctx || mode < 0 || mode > 1) return ECG_EARG;
    ctx->c.factor_mode = mode;
    return ECG_OK;
}

int ecg_factor_trace(ecg_ctx* ctx, int n, unsigned long long* records, long long cap, long long* count)
{
    if (!ctx || !count || n < 1 || n > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    CK(cudaMemsetAsync(c.status, 0, ST_COUNT * sizeof(int), c.stream));
    const int r = ldlh_factor_traced(c, n, records, cap, count);
    if (r == -3) return ECG_ENOMEM;
    return r ? ECG_ECUDA : ECG_OK;
}

int ecg_set_wait_limit(ecg_ctx* ctx, int polls)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    c.wait_limit = polls < 0 ? SOLVE_SPIN_LIMIT : polls;
    CK(cudaMemcpyAsync(c.counters + 3, &c.wait_limit, sizeof(int), cudaMemcpyHostToDevice, c.stream));
    if (c.cand.abort_word)
        CK(cudaMemcpyAsync(c.cand.abort_word + 1, &c.wait_limit, sizeof(int), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_compute_mat_elem(ecg_ctx* ctx, int nmin, int nmax, double approx_energy)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    mark(c, 0);
    const int r = compute_hs(c, nmin, nmax, approx_energy);
    mark(c, 1);
    if (r) return r;
    if (c.timing) {
        cudaStreamSynchronize(c.stream);
        c.stage_ms[0] = elapsed(c, 0, 1);
    }
    return ECG_OK;
}

int ecg_compute_mat_elem_and_deriv(ecg_ctx* ctx, int nmin, int nmax, int nfru, double approx_energy)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    mark(c, 0);
    const int r = compute_hsd(c, nmin, nmax, nfru, approx_energy);
    mark(c, 1);
    if (r) return r;
    if (c.timing) {
        cudaStreamSynchronize(c.stream);
        c.stage_ms[0] = elapsed(c, 0, 1);
    }
    return ECG_OK;
}

int ecg_ghepiis(ecg_ctx* ctx, int k, int n, double apprlambda, double tol, int max_iter, int specif_norm,
                double* lambda, double* rel_acc, int* num_iter)
{
    if (!ctx || !lambda || !rel_acc || !num_iter) return ECG_EARG;
    Ctx& c = ctx->c;
    mark(c, 1);
    const int r = ghepiis(c, k, n, apprlambda, tol, max_iter, specif_norm, lambda, rel_acc, num_iter);
    cudaStreamSynchronize(c.stream);
    if (c.timing) {
        c.stage_ms[1] = elapsed(c, 1, 2);
        c.stage_ms[2] = elapsed(c, 2, 3);
    }
    return r;
}

int ecg_energy_ia(ecg_ctx* ctx, int nmin, int nmax, int mat_elem_needed, double approx_energy, double tol,
                  int max_iter, int specif_norm, double* energy, int* num_iter)
{
    if (!ctx || !energy || !num_iter) return ECG_EARG;
    Ctx& c = ctx->c;
    if (c.method != 'I') return ECG_EARG;
    if (nmin < 1 || nmax < nmin || nmax > c.ld) return ECG_EARG;
    mark(c, 0);
    if (mat_elem_needed) {
        const int r = compute_hs(c, nmin, nmax, approx_energy);
        if (r) return r;
    }
    mark(c, 1);
    if (nmax == 1) {
        mark(c, 2);
        const int r = single_function_energy(c, approx_energy, energy);
        mark(c, 3);
        *num_iter = 1;
        finish_timing(c, false);
        return r;
    }
    // Glob_c(1:Nmax) = Glob_LastEigvector(1:Nmax), src/workproc.f90:1989
    CK(cudaMemcpyAsync(c.c, c.x, (size_t)nmax * sizeof(cd), cudaMemcpyDeviceToDevice, c.stream));
    double lam = 0.0, ra = 0.0;
    int it = 0;
    const int r = ghepiis(c, nmin, nmax, approx_energy, tol, max_iter, specif_norm, &lam, &ra, &it);
    *num_iter = it;
    if (r >= 0 && r != ECG_ESINGULAR) *energy = lam;
    finish_timing(c, false);
    return r;
}

int ecg_energy_ib(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, double approx_energy, double tol,
                  int max_iter, double* energy, double* grad_host, int* num_iter)
{
    if (!ctx || !energy || !num_iter) return ECG_EARG;
    return energy_ib_common(ctx->c, nfru, nfa, mat_elem_needed, approx_energy, tol, max_iter, energy, grad_host,
                            num_iter, false);
}

int ecg_energy_ib_adjoint(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, double approx_energy, double tol,
                          int max_iter, double* energy, double* grad_host, int* num_iter)
{
    if (!ctx || !energy || !num_iter) return ECG_EARG;
    return energy_ib_common(ctx->c, nfru, nfa, mat_elem_needed, approx_energy, tol, max_iter, energy, grad_host,
                            num_iter, true);
}

int ecg_eval_candidates(ecg_ctx* ctx, int nbase, int count, const double* cand_host, double approx_energy,
                        double tol, int max_iter, double* energies_host, int* errcodes_host, int* num_iter_host,
                        double* rel_acc_host)
{
    if (!ctx) return ECG_EARG;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.dev) != cudaSuccess) return ECG_ECUDA;
    return eval_candidates(c, nbase, count, cand_host, approx_energy, tol, max_iter, energies_host, errcodes_host,
                           num_iter_host, rel_acc_host);
}

int ecg_eval_candidates_grad(ecg_ctx* ctx, int nbase, int count, const double* cand_host, double approx_energy,
                             double tol, int max_iter, double* energies_host, int* errcodes_host, int* num_iter_host,
                             double* rel_acc_host, double* grad_host)
{
    if (!ctx || !grad_host) return ECG_EARG;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.dev) != cudaSuccess) return ECG_ECUDA;
    return eval_candidates(c, nbase, count, cand_host, approx_energy, tol, max_iter, energies_host, errcodes_host,
                           num_iter_host, rel_acc_host, grad_host);
}

int ecg_energy_ga(ecg_ctx* ctx, int nmin, int nmax, int mat_elem_needed, int which, int want_vector, double* energy,
                  int* num_factorizations)
{
    if (!ctx || !energy) return ECG_EARG;
    Ctx& c = ctx->c;
    const int r = energy_ga(c, nmin, nmax, mat_elem_needed, which, want_vector, energy);
    if (num_factorizations) *num_factorizations = c.g_last_factorizations;
    return r;
}

int ecg_energy_gb(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, int which, double* energy, double* grad_host)
{
    if (!ctx || !energy) return ECG_EARG;
    Ctx& c = ctx->c;
    if (c.method != 'G' || nfru < 0 || nfa <= nfru || nfa > c.ld) return ECG_EARG;
    if (nfa - nfru > c.max_nfo) return ECG_EARG;
    if (!mat_elem_needed && !c.D) return ECG_EARG;  // Glob_D is formed by the first derivative pass
    if (cudaSetDevice(c.dev) != cudaSuccess) return ECG_ECUDA;
    if (mat_elem_needed) CKR(compute_hsd(c, nfru + 1, nfa, nfru, 0.0));
    const int r = energy_ga(c, nfru + 1, nfa, 0, which, 1, energy);
    if (r != ECG_OK) return r;
    const int nfo = nfa - nfru;
    CKR(launch_plain_contract(c, nfo, nfa, nfru, *energy));
    if (grad_host) {
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
        c.bytes_d2h += (long long)nfo * c.npt * sizeof(double);
    }
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_energy_gb_adjoint(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, int which, double* energy,
                          double* grad_host)
{
    if (!ctx || !energy) return ECG_EARG;
    Ctx& c = ctx->c;
    if (c.method != 'G' || nfru < 0 || nfa <= nfru || nfa > c.ld) return ECG_EARG;
    if (mat_elem_needed) CKR(compute_hs(c, nfru + 1, nfa, 0.0));
    const int r = energy_ga(c, nfru + 1, nfa, 0, which, 1, energy);
    if (r != ECG_OK) return r;
    CKR(launch_adjoint(c, nfru, nfa, *energy));
    const int nfo = nfa - nfru;
    if (grad_host) {
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
        c.bytes_d2h += (long long)nfo * c.npt * sizeof(double);
    }
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_overlap_penalty(ecg_ctx* ctx, int nfru, int nfa, double max_pair_overlap_penalty, double overlap_threshold2,
                        int mode, double* total_penalty, double* grad_host)
{
    if (!ctx || !total_penalty) return ECG_EARG;
    Ctx& c = ctx->c;
    if (nfru < 0 || nfa <= nfru || nfa > c.ld || mode < 0 || mode > 2) return ECG_EARG;
    if (cudaSetDevice(c.dev) != cudaSuccess) return ECG_ECUDA;
    const double pc = max_pair_overlap_penalty / (1.0 - overlap_threshold2);
    const int nfo = nfa - nfru;
    // one partial sum per function; the solver's per-column scratch (2 ld doubles) holds them
    double* part = c.colval;
    CKR(launch_penalty(c, nfru, nfa, overlap_threshold2, pc, mode, part));
    std::vector<double> h((size_t)nfo);
    CK(cudaMemcpyAsync(h.data(), part, (size_t)nfo * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (mode > 0 && grad_host) {
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
        c.bytes_d2h += (long long)nfo * c.npt * sizeof(double);
    }
    CK(cudaStreamSynchronize(c.stream));
    c.bytes_d2h += (long long)nfo * sizeof(double);
    double tp = 0.0;
    for (int r = 0; r < nfo; r++) tp += h[r];
    *total_penalty = tp;
    return ECG_OK;
}

int ecg_expectation_values(ecg_ctx* ctx, int nbasis, const double* masses_host, int symm_adapt_method, int ny,
                           const int* y_mats_host, const int* y_coeffs_host, double energy, const double* c_host,
                           int ncf, const double* cf_grid_host, int ndens, const double* dens_grid_host,
                           double* values_host, double* errors_host, double* cf_host, double* dens_host)
{
    if (!ctx || !masses_host) return ECG_EARG;
    Ctx& c = ctx->c;
    const int n = c.n;
    if (nbasis < 1 || nbasis > c.ld || ncf < 0 || ndens < 0) return ECG_EARG;
    if ((ncf > 0 && !cf_grid_host) || (ndens > 0 && !dens_grid_host)) return ECG_EARG;
    // term lists of src/workproc.f90:8175-8347
    std::vector<int> pb, pk;
    std::vector<double> c1, c2;
    int em;
    if (symm_adapt_method == 1) {
        std::vector<int> eye((size_t)n * n, 0);
        for (int i = 0; i < n; i++) eye[i + i * n] = 1;
        for (int t = 0; t < c.T; t++) {
            pb.insert(pb.end(), eye.begin(), eye.end());
            pk.insert(pk.end(), c.yhy_h.begin() + (size_t)t * n * n, c.yhy_h.begin() + (size_t)(t + 1) * n * n);
            c1.push_back(c.yhy_coef_h[t]);
            c2.push_back(1.0);
        }
        em = 2;
    } else if (symm_adapt_method == 2) {
        if (ny < 1 || ny > 64 || !y_mats_host || !y_coeffs_host) return ECG_EARG;
        for (int k = 0; k < ny; k++)
            for (int kk = 0; kk < ny; kk++) {
                pb.insert(pb.end(), y_mats_host + (size_t)k * n * n, y_mats_host + (size_t)(k + 1) * n * n);
                pk.insert(pk.end(), y_mats_host + (size_t)kk * n * n, y_mats_host + (size_t)(kk + 1) * n * n);
                c1.push_back(y_coeffs_host[k]);
                c2.push_back(y_coeffs_host[kk]);
            }
        em = 3;
    } else {
        return ECG_EARG;
    }
    if (cudaSetDevice(c.dev) != cudaSuccess) return ECG_ECUDA;
    const int r = expectation_values(c, nbasis, masses_host, (int)c1.size(), pb.data(), pk.data(), c1.data(),
                                     c2.data(), em, energy, reinterpret_cast<const cd*>(c_host), ncf, cf_grid_host,
                                     ndens, dens_grid_host, values_host, errors_host, cf_host, dens_host);
    return r == 0 ? ECG_OK : (r == -3 ? ECG_ENOMEM : (r == -1 ? ECG_EARG : ECG_ECUDA));
}

int ecg_get_matrices(ecg_ctx* ctx, int n, double* H_host, double* S_host, int ld_host, double* diagS_host,
                     double* diagH_host, double* invD_host)
{
    if (!ctx || n < 0 || n > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    if ((H_host || S_host) && ld_host < n) return ECG_EARG;
    const size_t w = (size_t)n * sizeof(cd);
    if (n > 0) {
        if (H_host)
            CK(cudaMemcpy2DAsync(H_host, (size_t)ld_host * sizeof(cd), c.H, (size_t)c.ld * sizeof(cd), w, n,
                                 cudaMemcpyDeviceToHost, c.stream));
        if (S_host)
            CK(cudaMemcpy2DAsync(S_host, (size_t)ld_host * sizeof(cd), c.S, (size_t)c.ld * sizeof(cd), w, n,
                                 cudaMemcpyDeviceToHost, c.stream));
        if (diagS_host)
            CK(cudaMemcpyAsync(diagS_host, c.diagS, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (diagH_host)
            CK(cudaMemcpyAsync(diagH_host, c.diagH, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        if (invD_host) CK(cudaMemcpyAsync(invD_host, c.invD, w, cudaMemcpyDeviceToHost, c.stream));
    }
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_set_matrices(ecg_ctx* ctx, int n, const double* H_host, const double* S_host, int ld_host,
                     const double* diagS_host, const double* diagH_host)
{
    if (!ctx || n < 0 || n > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    if ((H_host || S_host) && ld_host < n) return ECG_EARG;
    const size_t w = (size_t)n * sizeof(cd);
    if (n > 0) {
        if (H_host)
            CK(cudaMemcpy2DAsync(c.H, (size_t)c.ld * sizeof(cd), H_host, (size_t)ld_host * sizeof(cd), w, n,
                                 cudaMemcpyHostToDevice, c.stream));
        if (S_host)
            CK(cudaMemcpy2DAsync(c.S, (size_t)c.ld * sizeof(cd), S_host, (size_t)ld_host * sizeof(cd), w, n,
                                 cudaMemcpyHostToDevice, c.stream));
        if (diagS_host)
            CK(cudaMemcpyAsync(c.diagS, diagS_host, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        if (diagH_host)
            CK(cudaMemcpyAsync(c.diagH, diagH_host, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        c.bytes_h2d += (long long)(H_host ? n * w : 0) + (S_host ? n * w : 0) + (diagS_host ? n * 8 : 0) +
                       (diagH_host ? n * 8 : 0);
    }
    CK(cudaStreamSynchronize(c.stream));
    // the matrices changed: no row of an earlier factor may be reused
    c.fact_n = 0;
    c.blk_start.clear();
    return ECG_OK;
}

int ecg_get_vectors(ecg_ctx* ctx, int n, double* c_host, double* last_eigvec_host)
{
    if (!ctx || n < 0 || n > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    if (n > 0 && c_host) CK(cudaMemcpyAsync(c_host, c.c, n * sizeof(cd), cudaMemcpyDeviceToHost, c.stream));
    if (n > 0 && last_eigvec_host)
        CK(cudaMemcpyAsync(last_eigvec_host, c.x, n * sizeof(cd), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_set_vectors(ecg_ctx* ctx, int n, const double* c_host, const double* last_eigvec_host)
{
    if (!ctx || n < 0 || n > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    if (n > 0 && c_host) CK(cudaMemcpyAsync(c.c, c_host, n * sizeof(cd), cudaMemcpyHostToDevice, c.stream));
    if (n > 0 && last_eigvec_host)
        CK(cudaMemcpyAsync(c.x, last_eigvec_host, n * sizeof(cd), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_get_gradient(ecg_ctx* ctx, int nfo, double* grad_host)
{
    if (!ctx || !grad_host || nfo < 0 || nfo > ctx->c.ld) return ECG_EARG;
    Ctx& c = ctx->c;
    if (nfo > 0)
        CK(cudaMemcpyAsync(grad_host, c.grad, (size_t)nfo * c.npt * sizeof(double), cudaMemcpyDeviceToHost,
                           c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_get_deriv(ecg_ctx* ctx, int nfo, int nfa, double* D_host)
{
    if (!ctx || !D_host) return ECG_EARG;
    Ctx& c = ctx->c;
    if (!c.D || nfo < 1 || nfo > c.max_nfo || nfa < 1 || nfa > c.ld) return ECG_EARG;
    const size_t n2 = (size_t)2 * c.npt;
    CK(cudaMemcpy2DAsync(D_host, n2 * nfo * sizeof(cd), c.D, n2 * c.max_nfo * sizeof(cd), n2 * nfo * sizeof(cd), nfa,
                         cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return ECG_OK;
}

int ecg_matrix_elements(ecg_ctx* ctx, int count, const double* pk_host, const double* pl_host,
                        const int* term_host, int gradflag, double* hs_host, double* dk_host, double* dl_host)
{
    if (!ctx || count < 0 || !pk_host || !pl_host || !term_host || !hs_host) return ECG_EARG;
    Ctx& c = ctx->c;
    for (int i = 0; i < count; i++)
        if (term_host[i] < 0 || term_host[i] >= c.T) return ECG_EARG;
    if (((gradflag == 1 || gradflag == 3) && !dk_host) || ((gradflag == 2 || gradflag == 3) && !dl_host))
        return ECG_EARG;
    if (count == 0) return ECG_OK;
    const size_t npt = c.npt, nd = (size_t)4 * c.np;
    double *pk = nullptr, *pl = nullptr;
    int* term = nullptr;
    cd *hs = nullptr, *dk = nullptr, *dl = nullptr;
    int r = 0;
    r |= dalloc(&pk, npt * count);
    r |= dalloc(&pl, npt * count);
    r |= dalloc(&term, (size_t)count);
    r |= dalloc(&hs, (size_t)2 * count);
    r |= dalloc(&dk, nd * count);
    r |= dalloc(&dl, nd * count);
    int status = r ? ECG_ENOMEM : ECG_OK;
    if (!status) {
        bool ok = cudaMemcpyAsync(pk, pk_host, npt * count * sizeof(double), cudaMemcpyHostToDevice, c.stream) ==
                      cudaSuccess &&
                  cudaMemcpyAsync(pl, pl_host, npt * count * sizeof(double), cudaMemcpyHostToDevice, c.stream) ==
                      cudaSuccess &&
                  cudaMemcpyAsync(term, term_host, count * sizeof(int), cudaMemcpyHostToDevice, c.stream) ==
                      cudaSuccess;
        if (ok && launch_term_batch(c, count, pk, pl, term, gradflag, hs, dk, dl) == 0) {
            ok = cudaMemcpyAsync(hs_host, hs, 2 * count * sizeof(cd), cudaMemcpyDeviceToHost, c.stream) ==
                 cudaSuccess;
            if (ok && (gradflag == 1 || gradflag == 3))
                ok = cudaMemcpyAsync(dk_host, dk, nd * count * sizeof(cd), cudaMemcpyDeviceToHost, c.stream) ==
                     cudaSuccess;
            if (ok && (gradflag == 2 || gradflag == 3))
                ok = cudaMemcpyAsync(dl_host, dl, nd * count * sizeof(cd), cudaMemcpyDeviceToHost, c.stream) ==
                     cudaSuccess;
            ok = ok && cudaStreamSynchronize(c.stream) == cudaSuccess;
        } else {
            ok = false;
        }
        if (!ok) {
            cudaGetLastError();
            status = ECG_ECUDA;
        }
    }
    cudaStreamSynchronize(c.stream);
    void* ptrs[] = {pk, pl, term, hs, dk, dl};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    return status;
}

long long ecg_launch_count(ecg_ctx* ctx) { return ctx ? ctx->c.launches : -1; }

int ecg_set_timing(ecg_ctx* ctx, int on)
{
    if (!ctx) return ECG_EARG;
    ctx->c.timing = (on != 0);
    return ECG_OK;
}

int ecg_get_stage_ms(ecg_ctx* ctx, double* ms4)
{
    if (!ctx || !ms4) return ECG_EARG;
    for (int i = 0; i < 4; i++) ms4[i] = ctx->c.stage_ms[i];
    return ECG_OK;
}

int ecg_sync(ecg_ctx* ctx)
{
    if (!ctx) return ECG_EARG;
    CK(cudaStreamSynchronize(ctx->c.stream));
    return ECG_OK;
}

int ecg_timer_start(ecg_ctx* ctx)
{
    if (!ctx) return ECG_EARG;
    CK(cudaEventRecord(ctx->c.tev[0], ctx->c.stream));
    return ECG_OK;
}

int ecg_timer_stop(ecg_ctx* ctx, double* ms)
{
    if (!ctx || !ms) return ECG_EARG;
    Ctx& c = ctx->c;
    CK(cudaEventRecord(c.tev[1], c.stream));
    CK(cudaEventSynchronize(c.tev[1]));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c.tev[0], c.tev[1]));
    *ms = f;
    return ECG_OK;
}

int ecg_io_bytes(ecg_ctx* ctx, long long* h2d, long long* d2h)
{
    if (!ctx) return ECG_EARG;
    if (h2d) *h2d = ctx->c.bytes_h2d;
    if (d2h) *d2h = ctx->c.bytes_d2h;
    return ECG_OK;
}

}  // extern "C"
