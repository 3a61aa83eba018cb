/*
 * ecg_abi.h -- C ABI of libecgb200.so, the B200 drop-in for the variational
 * hot path of ATOM-MOL-nonBO (matrix elements over explicitly correlated
 * complex Gaussians, H/S assembly, the inverse-iteration solve of HC = ESC
 * and the gradient with respect to the nonlinear parameters).
 *
 * The reference's routines are Fortran module procedures that talk through
 * module globals (src/globvars.f90).  Here the globals live in an opaque
 * context, one per basis, whose device arrays mirror them:
 *     Glob_NonlinParam (npt x K)   Glob_H, Glob_S (ld x ld)   Glob_diagS,
 *     Glob_diagH   Glob_invD   Glob_c   Glob_LastEigvector   Glob_D.
 * Conventions:
 *   - every function returns an int status: 0 = success; 1 / 2 are the
 *     GHEPIIS ErrorCodes (1 = exactly zero pivot, 2 = not converged);
 *     negative values are ECG_E* below.  Nothing aborts the process.
 *   - basis indices are 1-based and inclusive, as in the Fortran callers;
 *     matrices are column-major; complex numbers are (re, im) double pairs
 *     (Fortran complex(8), C double _Complex).
 *   - pointers named *_host are host memory, copied during the call only.
 *   - one context is used by one host thread; all work is ordered on the
 *     context's CUDA stream.
 */
#ifndef ECG_ABI_H
#define ECG_ABI_H

#ifdef __cplusplus
extern "C" {
#endif

#define ECG_OK 0
#define ECG_ESINGULAR 1     /* GHEPIIS ErrorCode=1, src/linalg.f90:1862-1863 */
#define ECG_ENOCONV 2       /* GHEPIIS ErrorCode=2, src/linalg.f90:1864-1869 */
#define ECG_EARG (-1)       /* bad argument (size, index range, method) */
#define ECG_ECUDA (-2)      /* CUDA runtime error */
#define ECG_ENOMEM (-3)     /* device allocation failed */
#define ECG_ENODEV (-4)     /* no CUDA device */
#define ECG_ELIMIT (-5)     /* size above a fixed capacity of the call */

typedef struct ecg_ctx ecg_ctx;

/* Create a context for one system and basis capacity.
 * Replaces the array allocation and ProgramDataInit outputs consumed by the
 * hot path (src/workproc.f90:575-1202): n pseudo-particles (1..5),
 * mass_matrix_host = Glob_MassMatrix (n x n), charges_host = (q0, q1..qn)
 * = (Glob_PseudoCharge0, Glob_PseudoCharge), nterms Y^+Y terms with
 * yhy_mats_host = Glob_YHYMatr (n x n x nterms, integer) and
 * yhy_coeffs_host = Glob_YHYCoeff.  ld = Glob_HSLeadDim (max basis size),
 * max_nfo = the second extent of Glob_D (0: no plain derivative storage),
 * method = Glob_GSEPSolutionMethod ('I' or 'G').  device = CUDA ordinal. */
int ecg_ctx_create(int n, const double* mass_matrix_host, const double* charges_host, int nterms,
                   const int* yhy_mats_host, const int* yhy_coeffs_host, int ld, int max_nfo, char method,
                   int device, ecg_ctx** out);
int ecg_ctx_destroy(ecg_ctx* ctx);

/* Glob_NonlinParam(1:npt, first:first+count-1) = params_host (npt x count).
 * The optimisation drivers' parameter update before each evaluation, e.g.
 * src/workproc.f90:4157-4159 (BasisEnlI) and the FullOpt1I equivalent. */
int ecg_set_params(ecg_ctx* ctx, const double* params_host, int first, int count);
/* The same update from device memory (params_dev: npt x count doubles on the
 * context's device, e.g. an optimiser that keeps its iterate on the GPU);
 * ordered on the context's stream, no host copy. */
int ecg_set_params_device(ecg_ctx* ctx, const double* params_dev, int first, int count);

/* ComputeMatElem(Nmin,Nmax) + StoreHS, src/matform.f90:119-230 and :11-51.
 * approx_energy = Glob_ApproxEnergy (lambda~).  Rows Nmin..Nmax of the
 * lower triangle are computed; 'I' storage keeps H - lambda~ S in the lower
 * triangle of H and the full Hermitian S; 'G' storage keeps the strict lower
 * triangles of H and S plus diagS, diagH. */
int ecg_compute_mat_elem(ecg_ctx* ctx, int nmin, int nmax, double approx_energy);

/* ComputeMatElemAndDeriv(Nmin,Nmax) + StoreHSD, src/matform.f90:234-360 and
 * :55-115: as above plus Glob_D(1:2npt, i-nfru, j).  Requires
 * nfru < Nmin and Nmax - nfru <= max_nfo. */
int ecg_compute_mat_elem_and_deriv(ecg_ctx* ctx, int nmin, int nmax, int nfru, double approx_energy);

/* GHEPIIS(k,n,Glob_H,...,Glob_invD,Glob_S,...,apprlambda,Glob_c,w,Tol,
 * lambda,Glob_LastEigvector,RelAcc,MaxIter,SpecifNorm,NumIter,ErrorCode),
 * src/linalg.f90:1781-1926, on the context's device arrays: the LDL^H
 * factor of rows 1..k-1 is reused, rows k..n are factorised; the start
 * vector is Glob_c and the eigenvector lands in Glob_LastEigvector.
 * Returns ErrorCode. */
int ecg_ghepiis(ecg_ctx* ctx, int k, int n, double apprlambda, double tol, int max_iter, int specif_norm,
                double* lambda, double* rel_acc, int* num_iter);

/* EnergyIA / EnergyIAM, src/workproc.f90:1954-2060: optional
 * ComputeMatElem(Nmin,Nmax), then Glob_c = Glob_LastEigvector and GHEPIIS
 * with SpecifNorm -1 (IA) or 0 (IAM).  Returns ErrorCode. */
int ecg_energy_ia(ecg_ctx* ctx, int nmin, int nmax, int mat_elem_needed, double approx_energy, double tol,
                  int max_iter, int specif_norm, double* energy, int* num_iter);

/* EnergyIB, src/workproc.f90:2063-2154 (plain drop-in): optional
 * ComputeMatElemAndDeriv(nfru+1, nfa), GHEPIIS(nfru+1, nfa, ..., SpecifNorm
 * 0), then the gradient contraction over Glob_D.  grad_host receives npt*nfo
 * values ordered (vechL_i, vechB_i) for i = nfru+1..nfa; NULL leaves the
 * gradient on the device (ecg_get_gradient). */
int ecg_energy_ib(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, double approx_energy, double tol,
                  int max_iter, double* energy, double* grad_host, int* num_iter);

/* Same result as ecg_energy_ib from a fused adjoint pass: H, S without
 * derivatives, GHEPIIS, then one pass over the pairs of rows nfru+1..nfa
 * that recomputes each pair term and contracts its derivatives with
 * c_k^* c_l on the fly; Glob_D is neither formed nor read. */
int ecg_energy_ib_adjoint(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, double approx_energy, double tol,
                          int max_iter, double* energy, double* grad_host, int* num_iter);

/* The trial loop of BasisEnlI (src/workproc.f90:4054-4070) for `count`
 * candidate functions at once: for every candidate j, the energy that
 *     Glob_NonlinParam(1:npt, nbase+1) = cand_host(1:npt, j)
 *     E_j = EnergyIA(nbase+1, nbase+1, .true., ErrorCode_j)
 * would return, i.e. ComputeMatElem(nbase+1, nbase+1) followed by
 * GHEPIIS(nbase+1, nbase+1, ..., SpecifNorm -1) with the bordered LDL^H
 * step of LDLHF (src/linalg.f90:316-391) for the new row.
 * Requires: the context's H and S hold rows 1..nbase built with the same
 * approx_energy (lambda~), as after EnergyIA(1, nbase); the LDL^H factor of
 * those rows is reused when present, else computed first (ErrorCode 1 of
 * that factorisation is returned as the call's status).
 * Every candidate starts from Glob_LastEigvector(1:nbase+1) as the context
 * holds it at the call (the sequential reference starts each trial from
 * the previous trial's eigenvector; results agree to the tolerance).
 * The context's own state (parameters, H, S, factor, vectors) is left as
 * it was: install the chosen candidate with ecg_set_params and
 * ecg_energy_ia(nbase+1, nbase+1, ...), as BasisEnlI does after its loop.
 * Outputs per candidate: energies_host (undefined where the code is 1),
 * errcodes_host (0, 1 = zero pivot in the new row, 2 = not converged in
 * max_iter iterations), num_iter_host and rel_acc_host (NormOfDiff); the
 * last three may be NULL.  Returns 0 or a negative ECG_E* status. */
int ecg_eval_candidates(ecg_ctx* ctx, int nbase, int count, const double* cand_host, double approx_energy,
                        double tol, int max_iter, double* energies_host, int* errcodes_host, int* num_iter_host,
                        double* rel_acc_host);

/* ecg_eval_candidates plus, for every candidate j, the gradient that
 *     Glob_NonlinParam(1:npt, nbase+1) = cand_host(1:npt, j)
 *     call EnergyIB(E_j, grad_j, .true., ErrorCode_j)   with nfru = nbase,
 *                                                        nfa = nbase+1
 * returns (src/workproc.f90:2063-2154 with nfo = 1): dE_j / d(vech L,
 * vech B) of the candidate itself, from its eigenpair normalised c^H S c = 1
 * and a fused adjoint pass over row nbase+1 (no Glob_D).  This is the
 * energy + gradient the optimisation of a newly added function needs
 * (BasisEnlI's DRMNG loop, src/workproc.f90:4137-4170, and OptCycleI),
 * for all candidates at once.  grad_host receives npt x count values
 * (NaN for a candidate whose ErrorCode is 1); requires nbase >= 1.  Other
 * arguments and outputs as for ecg_eval_candidates. */
int ecg_eval_candidates_grad(ecg_ctx* ctx, int nbase, int count, const double* cand_host, double approx_energy,
                             double tol, int max_iter, double* energies_host, int* errcodes_host, int* num_iter_host,
                             double* rel_acc_host, double* grad_host);

/* EnergyGA (want_vector 0) / EnergyGAM (want_vector 1), src/workproc.f90:
 * 1697-1838, for contexts created with method 'G': optional
 * ComputeMatElem(Nmin,Nmax), then the which-th smallest eigenvalue of
 * H c = E S c with the semantics of the reference's
 * ZHEGVX(1, JOBZ, 'I', 'U', Nmax, ..., IL=IU=which) (src/workproc.f90:1750);
 * with want_vector, Glob_c = its eigenvector normalised c^H S c = 1.  As in
 * the reference, Glob_S's upper triangle is filled from its lower one.
 * Method: LDL^H of S for the positive-definiteness test; Sylvester-inertia
 * bisection on LDL^H(H - sigma S) (negative pivots = eigenvalues below
 * sigma) until the bracket holds the which-th eigenvalue alone; GHEPIIS at
 * the bracket's centre.  num_factorizations (may be NULL) receives the
 * number of LDL^H factorisations used.  Returns 0, or Nmax + i when the
 * leading minor of order i of S is not positive definite (ZHEGVX's INFO),
 * or a negative status. */
int ecg_energy_ga(ecg_ctx* ctx, int nmin, int nmax, int mat_elem_needed, int which, int want_vector, double* energy,
                  int* num_factorizations);

/* EnergyGB, src/workproc.f90:1841-1950 (plain drop-in, contexts created
 * with method 'G' and max_nfo >= nfa - nfru): optional
 * ComputeMatElemAndDeriv(nfru+1, nfa), EnergyGAM's eigenpair (Glob_c with
 * c^H S c = 1), then the gradient contraction over Glob_D
 * (src/workproc.f90:1927-1940).  grad_host as for ecg_energy_ib. */
int ecg_energy_gb(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, int which, double* energy, double* grad_host);

/* EnergyGB, src/workproc.f90:1841-1950, through the fused adjoint pass:
 * optional ComputeMatElem(nfru+1, nfa), EnergyGAM's eigenpair, then the
 * gradient of ecg_energy_ib_adjoint (same ordering) at that eigenpair. */
int ecg_energy_gb_adjoint(ecg_ctx* ctx, int nfru, int nfa, int mat_elem_needed, int which, double* energy,
                          double* grad_host);

/* ComputeOverlapPenalty (mode 0) and ComputeOverlapPenaltyAndAddGradient
 * (mode 1), src/workproc.f90:1491-1693: total_penalty = sum over pairs
 * i < j <= nfa with j > nfru of b (|S_ji|^2 - t2) / (1 - t2) where
 * |S_ji|^2 > t2, from the normalised overlaps in Glob_S (b =
 * max_pair_overlap_penalty = Glob_MaxOverlapPenalty, t2 =
 * overlap_threshold2 = Glob_OverlapPenaltyThreshold2).  Mode 1 adds the
 * reference's penalty gradient to the context's gradient (the one the last
 * ecg_energy_ib* / ecg_energy_gb_adjoint call left, Glob_WkGR), with the
 * derivatives it reads from Glob_D recomputed for the flagged pairs, so the
 * fused adjoint path needs no Glob_D.  Mode 2 adds instead the derivative
 * of the penalty itself: the reference's normalisation terms carry a factor
 * sqrt(diagS_i/diagS_j), and for the lower-index function S_ji^2 where the
 * derivative has |S_ji|^2.  grad_host (may be NULL) receives the updated gradient (npt x
 * (nfa - nfru)).  Requires Glob_S, Glob_diagS and the parameters of
 * functions 1..nfa current (any ComputeMatElem over them). */
int ecg_overlap_penalty(ecg_ctx* ctx, int nfru, int nfa, double max_pair_overlap_penalty, double overlap_threshold2,
                        int mode, double* total_penalty, double* grad_host);

/* The expectation-value pass of ExpectationValuesG, src/workproc.f90:
 * 8159-8366, with MatrixElementsForExpcVals (src/matelem.f90:949-1983) for
 * every pair of functions 1..nbasis and every symmetry term:
 *   symm_adapt_method 1: Y^+Y (the context's terms) on the ket; the error
 *                        bound adds 2|beta| per term;
 *   symm_adapt_method 2: Y on bra and ket, all (k, kk) pairs of the ny
 *                        terms y_mats_host (n x n x ny, Glob_YMatr) with
 *                        coefficients y_coeffs_host (Glob_YCoeff); 3|beta|.
 * masses_host = Glob_Mass (m0, m1..mn); energy = Glob_CurrEnergy (the
 * eigenvalue, used by the Drachmanised terms); c_host = the eigenvector
 * (nbasis complex), or NULL for Glob_c (left there by ecg_energy_ga with
 * want_vector).  Glob_diagS must hold functions 1..nbasis (any
 * ComputeMatElem(1, nbasis) has set it).
 * Outputs (NULL to skip): values_host / errors_host, 6np + 9 each in the
 * MEkl order of src/workproc.f90:8045-8060: 1/r^2, 1/r, r, r^2, delta(r),
 * Drachmanised delta(r) (np each, vech order (1,1),(1,2)..(n,n)), then H,
 * S, T, V, MV, drach_MV, Darwin, drach_Darwin, OO; errors_host are the
 * MEkl_e bounds (already times epsilon).  cf_host (np x ncf) and dens_host
 * ((n+1) x ndens): correlation functions on cf_grid_host and particle
 * densities on dens_grid_host (ncf / ndens may be 0). */
int ecg_expectation_values(ecg_ctx* ctx, int nbasis, const double* masses_host, int symm_adapt_method, int ny,
                           const int* y_mats_host, const int* y_coeffs_host, double energy, const double* c_host,
                           int ncf, const double* cf_grid_host, int ndens, const double* dens_grid_host,
                           double* values_host, double* errors_host, double* cf_host, double* dens_host);

/* Device -> host copies of the context arrays (any pointer may be NULL).
 * H_host, S_host: n x n with leading dimension ld_host. */
int ecg_get_matrices(ecg_ctx* ctx, int n, double* H_host, double* S_host, int ld_host, double* diagS_host,
                     double* diagH_host, double* invD_host);
/* The reverse of ecg_get_matrices: Glob_H, Glob_S (n x n, leading dimension
 * ld_host), Glob_diagS and Glob_diagH from host memory (any pointer may be
 * NULL), in the context's layout ('I' or 'G').  This is how the matrices
 * of the reference's swap file come back (ReadSwapFileAndDistributeData,
 * src/workproc.f90:2158-2240) so that EnergyIA / EnergyGA can run with
 * mat_elem_needed = 0.  The LDL^H factor of earlier rows is discarded. */
int ecg_set_matrices(ecg_ctx* ctx, int n, const double* H_host, const double* S_host, int ld_host,
                     const double* diagS_host, const double* diagH_host);
int ecg_get_vectors(ecg_ctx* ctx, int n, double* c_host, double* last_eigvec_host);
int ecg_set_vectors(ecg_ctx* ctx, int n, const double* c_host, const double* last_eigvec_host);
int ecg_get_gradient(ecg_ctx* ctx, int nfo, double* grad_host);
/* Glob_D(1:2npt, 1:nfo, 1:nfa) with leading extents (2npt, nfo). */
int ecg_get_deriv(ecg_ctx* ctx, int nfo, int nfa, double* D_host);

/* MatrixElements(Paramk, Paraml, P, Hkl, Skl, Dk, Dl, gradflag),
 * src/matelem.f90:12-750, for count independent calls.  P is the context's
 * Y^+Y matrix number term_host[i] (0-based).  hs_host receives (Hkl, Skl)
 * per call (4 doubles); dk_host / dl_host receive 4np complex values per
 * call when gradflag asks for them (may be NULL otherwise). */
int ecg_matrix_elements(ecg_ctx* ctx, int count, const double* pk_host, const double* pl_host,
                        const int* term_host, int gradflag, double* hs_host, double* dk_host, double* dl_host);

/* Diagnostics: kernel launches issued by this context so far, and the
 * device time (ms) of the stages of the last energy call:
 * [0] pair pass(es) for H,S  [1] LDL^H  [2] inverse iterations
 * [3] gradient (derivative pass + contraction, or adjoint pass). */
long long ecg_launch_count(ecg_ctx* ctx);
int ecg_set_timing(ecg_ctx* ctx, int on);
int ecg_get_stage_ms(ecg_ctx* ctx, double* ms4);
/* Block until all work queued on the context's stream has finished. */
int ecg_sync(ecg_ctx* ctx);
/* Device timer on the context's stream: start records an event; stop
 * records a second one, waits for it and returns the elapsed ms. */
int ecg_timer_start(ecg_ctx* ctx);
int ecg_timer_stop(ecg_ctx* ctx, double* ms);
/* One evaluation's pair work split over several GPUs (one context per GPU,
 * one process per GPU).  The reference deals its (pair, term) units to MPI
 * ranks and sums the H, S buffers and the gradient with MPI_ALLREDUCE
 * (src/matform.f90:170-213, src/workproc.f90:2129,2148); here each rank
 * takes a contiguous range of the 32 x 32 pair tiles of the lower
 * triangle, in the order the pair kernels walk them (ecg_pair_tiles gives
 * their number for rows nmin..nmax):
 *   ecg_compute_mat_elem_tiles  ComputeMatElem(nmin, nmax) for the range's
 *                               pairs plus every diagonal pair (StoreHS
 *                               needs all of diagS), into Glob_H / Glob_S;
 *   ecg_pack_tiles              the range's stored entries into packed_dev
 *                               (per tile 2 x 32 x 32 complex: H, then S);
 *   ecg_unpack_tiles            another rank's packed tiles into Glob_H,
 *                               Glob_S ('I' storage: S's upper mirror too).
 * After the exchange every rank holds the whole H and S, bit for bit what
 * ecg_compute_mat_elem writes, and runs the solve itself (ecg_energy_ia
 * with mat_elem_needed 0 and SpecifNorm 0).  Then
 *   ecg_adjoint_tiles           the fused adjoint pass of
 *                               ecg_energy_ib_adjoint over the range's
 *                               tiles of rows nfru+1..nfa (the tile list
 *                               of ecg_pair_tiles(nfru+1, nfa)) with
 *                               energy E and the eigenvector in
 *                               Glob_LastEigvector; part_dev receives
 *                               count x ecg_adjoint_part_doubles values;
 *   ecg_adjoint_finish          the gradient from the partials of all
 *                               tiles in list order (the ranks' ranges
 *                               concatenated): bit for bit that of
 *                               ecg_energy_ib_adjoint; grad_host as there.
 * Device buffers are the caller's, on the context's device; work is
 * ordered on the context's stream (ecg_sync before another stream or a
 * collective reads them). */
int ecg_pair_tiles(ecg_ctx* ctx, int nmin, int nmax, long long* ntiles);
int ecg_compute_mat_elem_tiles(ecg_ctx* ctx, int nmin, int nmax, double approx_energy, long long first,
                               long long count);
int ecg_pack_tiles(ecg_ctx* ctx, int nmin, int nmax, long long first, long long count, void* packed_dev);
int ecg_unpack_tiles(ecg_ctx* ctx, int nmin, int nmax, long long first, long long count, const void* packed_dev);
int ecg_adjoint_part_doubles(ecg_ctx* ctx, long long* per_tile);
int ecg_adjoint_tiles(ecg_ctx* ctx, int nfru, int nfa, double energy, long long first, long long count,
                      void* part_dev);
int ecg_adjoint_finish(ecg_ctx* ctx, int nfru, int nfa, const void* part_dev, double* grad_host);

/* Shapes the context's autotuner chose (-1: not tuned yet).  The pair
 * kernels' shape is chosen once per context by timing every candidate
 * shape on the first large launch (the outputs do not depend on it):
 *   pair_shape     k_pair_energy, 0..3: warps per 32 x 32 pair tile (8, 8,
 *                  4, 4) x register budget (2, 3, 2, 4 CTAs per SM);
 *   adjoint_shape  k_adjoint, 0..1: 1 or 2 CTAs per SM;
 *   cand_row_shape k_cand_row, 0..4: warps x candidates per warp.
 * times_ms (may be NULL) receives the 4 + 2 timings of the first two.  No
 * counterpart in the reference, whose linalg_setparam table
 * (src/linalg.f90:83-147) is the fixed tuning this replaces. */
int ecg_get_tuning(ecg_ctx* ctx, int* pair_shape, int* adjoint_shape, int* cand_row_shape, double* times_ms);

/* Pivots of the context's LDL^H factorisations (GHEPIIS, the candidates'
 * bordered step, the 'G' path): mode 0 (default) keeps them real, dropping
 * the rounding-level imaginary part that the complex arithmetic of
 * LDLHF (src/linalg.f90:370-381) leaves in them; mode 1 keeps the complex
 * pivot d = conj(x) and its exact x == 0 test as the reference does.  The
 * energies agree to rounding either way; the imaginary parts set a floor
 * of about 1e-13..1e-12 under GHEPIIS's NormOfDiff, so near
 * EIGVAL_TOLERANCE = 1e-12 mode 1 returns ErrorCode 2 where the reference
 * does and mode 0 converges.  Changing the mode discards the factor. */
int ecg_set_pivot_mode(ecg_ctx* ctx, int mode);
/* How the context factorises a whole matrix (LDLHF with m = 1, the first
 * step of every EnergyIA/IB(0, K) and of the 'G' path): mode 0 (default)
 * one persistent cooperative kernel over 64 x 64 tiles whose CTAs take
 * the diagonal eliminations, panel rows and trailing updates from a
 * critical-path-ordered task list; mode 1 one launch per panel step
 * (diagonal block, panel rows, trailing update on a second stream).  Both
 * give the same factor up to rounding.  No counterpart in the reference
 * (its LDLHF is one code path); kept for comparison and measurement. */
int ecg_set_factor_mode(ecg_ctx* ctx, int mode);
/* Factorise rows 1..n of the context's current matrix (the lower triangle
 * that ecg_compute_mat_elem / ecg_ghepiis leave: H - lambda~ S) once with
 * the persistent kernel, outside any graph, recording per task: the task
 * code (as ecg_ldl_schedule) | CTA << 32 | panels applied << 48 (0: found
 * already applied), and the GPU's globaltimer (ns) when the CTA began
 * waiting for the task's tiles, when they were ready and when the task was
 * published.  *count receives the number of records; records (capacity cap
 * values, 4 per record) is filled when large enough.  The factor is left as
 * GHEPIIS's factorisation leaves it.  No counterpart in the reference: a
 * measurement aid. */
int ecg_factor_trace(ecg_ctx* ctx, int n, unsigned long long* records, long long cap, long long* count);
/* Poll limit of the bounded device waits of the context (the triangular
 * solves of GHEPIIS and of the batched candidates, and the tile waits of
 * the persistent factorisation): every wait on another CTA's work gives up
 * after `polls` polls, records the timeout and the call returns ECG_ECUDA
 * with the context still usable.  polls < 0 restores the default (2^22).
 * No counterpart in the reference: a diagnostic that lets a test make a
 * wait run out without a fault. */
int ecg_set_wait_limit(ecg_ctx* ctx, int polls);
/* The task order of the persistent factorisation of n rows (n <= 12800)
 * for a grid of `workers` CTAs, on the host (no GPU needed): codes
 * type << 30 | h << 29 | s << 20 | R << 10 | C, type 0 = D(s) (diagonal
 * tile s), 1 = T(s, C) (panel rows of tile (s, C)), 2 = B(s, R, C) (update
 * of tile (R, C) by panel s; for R <= s + 2, other than (s+1, s+1), two
 * tasks on the column halves h = 0, 1), 64-row tiles.  *count receives the
 * length; out (capacity cap) is filled when it is large enough.  No
 * counterpart in the reference: exposes the task order to tests. */
int ecg_ldl_schedule(int n, int workers, unsigned* out, long long cap, long long* count);
/* Bytes this context has copied host->device and device->host so far. */
int ecg_io_bytes(ecg_ctx* ctx, long long* h2d, long long* d2h);
/* The fused adjoint gradient of ecg_energy_ib_adjoint, for callers that
 * cannot allocate device memory when they need it (a host that manages all
 * GPU memory through its own pool, an optimiser callback that must not fail
 * or fragment memory mid-run, a service with fixed memory budgets).  No
 * counterpart in the reference.  Every input and output is caller-owned:
 * params_dev = Glob_NonlinParam (npt x nfa doubles), c_dev = the normalised
 * eigenvector Glob_c (nfa complex), diagS_dev = Glob_diagS (nfa), energy =
 * its eigenvalue, grad_dev receives npt*(nfa-nfru) doubles ordered as
 * ecg_energy_ib's gradient.  The system arguments are those of
 * ecg_ctx_create.  Work is queued on `stream` (a cudaStream_t, NULL for the
 * default stream); the call issues no host-to-device copy (the projector
 * terms travel as kernel arguments) and returns without waiting for it.
 * Limits: nfa <= 512 and nterms <= 16, else ECG_ELIMIT and nothing runs.
 * The call allocates nothing: its working data lives in one fixed array of
 * about 4.3 MB compiled into the library, held by every GPU that loads it
 * until the process exits.  The first call on a device does a one-time
 * set-up (it looks up that array's device address): make that first call
 * before any stream capture on the device.  All calls on a device share the
 * array: calls whose GPU work overlaps race on it and must be serialised by
 * the caller. */
int ecg_adjoint_gradient_noalloc(int n, const double* mass_matrix_host, const double* charges_host, int nterms,
                                 const int* yhy_mats_host, const int* yhy_coeffs_host, const double* params_dev,
                                 const double* c_dev, const double* diagS_dev, double energy, int nfru, int nfa,
                                 double* grad_dev, void* stream);
/* Measured FP64 FMA throughput of the device (TFLOP/s, 2 flops per FMA):
 * a register-resident FMA loop over all SMs, timed with CUDA events. */
int ecg_probe_fp64_peak(int device, double* tflops);
/* Measured FP64 tensor-core throughput of the device (TFLOP/s, 2 flops per
 * multiply-add): register-resident mma.sync.m8n8k4.f64 chains over all SMs,
 * timed with CUDA events. */
int ecg_probe_fp64_tensor_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* ECG_ABI_H */
