/*
 * ecg_oracle.c -- CPU restatement of ATOM-MOL-nonBO's variational hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker and the timed
 * CPU baseline.  Nothing in the shipped library links, loads or calls it;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * It restates, in plain C99 double / double complex arithmetic, with the
 * same loop structure and operation order as the Fortran source, these
 * reference routines (paths relative to the reference project root):
 *
 *   MatrixElements            src/matelem.f90:12-750
 *   StoreHS / StoreHSD        src/matform.f90:11-115
 *   ComputeMatElem            src/matform.f90:119-230
 *   ComputeMatElemAndDeriv    src/matform.f90:234-360
 *   LDLHF (serial branch)     src/linalg.f90:316-392
 *   LDLHF (parallel branch)   src/linalg.f90:400-452, OpenMP threads as the
 *                             ranks; chosen as linalg_setparam does,
 *                             src/linalg.f90:113-121
 *   LDLHS (non-BLAS branch)   src/linalg.f90:618-653
 *   MHMV  (non-BLAS branch)   src/linalg.f90:1019-1043
 *   VMMHMV (serial branch)    src/linalg.f90:1180-1215
 *   CMaxAbsReOrIm, CVScale, CDotProdQuotient, CVDiffEucNorm, CDotProdItself
 *                             src/linalg.f90:1283-1311,1538-1563,1481-1515,
 *                                            1598-1629,1413-1443
 *   GHEPIIS                   src/linalg.f90:1781-1926
 *   EnergyIA/IAM/IB glue      src/workproc.f90:1954-2154
 *   ComputeOverlapPenalty(AndAddGradient)
 *                             src/workproc.f90:1491-1693
 *
 * The MPI work split of the reference is replaced by an OpenMP loop over
 * pairs; every pair element is computed exactly as one MPI rank computes it
 * with NumOfProcs = 1 (all Y^+Y terms summed in order j = 1..T), so the
 * values do not depend on the thread count.  BLAS calls are replaced by the
 * reference's own non-BLAS branches, which compute the same quantities.
 *
 * Compile with -O2 -fno-fast-math -ffp-contract=off so that no FMA
 * contraction changes the rounding of the restated expressions.
 */
#include <complex.h>
#include <math.h>
#include <float.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "ecg_oracle.h"

/* ---- module globals (the subset of src/globvars.f90 the path reads) ---- */
int g_n, g_np, g_npt, g_T;
double g_mass[NN][NN];             /* Glob_MassMatrix(i,j) -> g_mass[i][j] */
double g_q0, g_q[NN];              /* Glob_PseudoCharge0, Glob_PseudoCharge */
int g_P[TMAX][NN][NN];             /* Glob_YHYMatr(i,j,t) -> g_P[t][i][j] */
int g_coef[TMAX];                  /* Glob_YHYCoeff */
double g_2r3n2;                    /* Glob_2raised3n2 = 2^(3n/2) */

/* Set the system.  mass_cm is the n x n mass matrix column-major,
 * charges = (q0, q1..qn), yhy_cm = T column-major n x n integer matrices. */
int orc_set_system(int n, int T, const double *mass_cm, const double *charges,
                   const int *yhy_cm, const int *coef)
{
    if (n < 1 || n > NN || T < 1 || T > TMAX) return 1;
    g_n = n;
    g_np = n * (n + 1) / 2;
    g_npt = 2 * g_np;
    g_T = T;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) g_mass[i][j] = mass_cm[i + j * n];
    g_q0 = charges[0];
    for (int i = 0; i < n; i++) g_q[i] = charges[1 + i];
    for (int t = 0; t < T; t++) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) g_P[t][i][j] = yhy_cm[t * n * n + i + j * n];
        g_coef[t] = coef[t];
    }
    /* TWO**((3*Glob_n)/TWO), src/workproc.f90:76 */
    g_2r3n2 = pow(2.0, (3 * n) / 2.0);
    return 0;
}

/* ------------------------------------------------------------------------
 * MatrixElements, src/matelem.f90:12-750.  Pcm is the n x n permutation
 * matrix column-major.  Dk, Dl receive 4*np values each when requested.
 * ---------------------------------------------------------------------- */
static void matrix_elements(const double *Paramk, const double *Paraml, int P[NN][NN],
                            cplx *Hkl, cplx *Skl, cplx *Dk, cplx *Dl, int gradflag)
{
    const int n = g_n, np = g_np;
    double vechLk[NNP], vechBk[NNP], vechLl[NNP], vechBl[NNP];
    cplx dHdLk[NNP], dHdBk[NNP], dHdLl[NNP], dHdBl[NNP];
    cplx dSdLk[NNP], dSdBk[NNP], dSdLl[NNP], dSdBl[NNP];
    double Lk[NN][NN], Ll[NN][NN], inv_Lk[NN][NN], inv_Ll[NN][NN];
    double Ak[NN][NN], tAl[NN][NN], Bk[NN][NN], tBl[NN][NN];
    cplx Ck[NN][NN], tCl[NN][NN], tCkl[NN][NN];
    cplx inv_tCkl[NN][NN], inv_ttCkl[NN][NN], tr32[NN][NN];
    cplx F[NN][NN], G[NN][NN], tQ[NN][NN], ttQ[NN][NN];
    cplx Wc1[NN][NN], Wc2[NN][NN];
    cplx WVcLk[NNP], WVcLl[NNP], WVcBk[NNP], WVcBl[NNP];
    double Wr1[NN][NN], Wr2[NN][NN];
    double rtemp, rsum, rnumb;
    cplx ctemp, csum, cnumb, cmpnum, cRklij, det_tCkl, Tkl, Vkl, S, H;
    double det_Lk, det_Ll;
    int i, j, k, kk, kkk, indx;
    int grad_k = 0, grad_l = 0;

    for (i = 0; i < np; i++) {
        vechLk[i] = Paramk[i];
        vechBk[i] = Paramk[np + i];
        vechLl[i] = Paraml[i];
        vechBl[i] = Paraml[np + i];
    }
    if (gradflag == 1) grad_k = 1;
    if (gradflag == 2) grad_l = 1;
    if (gradflag == 3) { grad_k = 1; grad_l = 1; }

    /* matelem.f90:109-122 */
    indx = 0;
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            Lk[i][j] = 0.0; Lk[j][i] = vechLk[indx];
            Ll[i][j] = 0.0; Ll[j][i] = vechLl[indx];
            Bk[j][i] = vechBk[indx]; Bk[i][j] = vechBk[indx];
            tBl[j][i] = vechBl[indx]; tBl[i][j] = vechBl[indx];
            indx++;
        }
    /* matelem.f90:124-139 */
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            rtemp = 0.0;
            for (k = 0; k <= j; k++) rtemp = rtemp + Lk[i][k] * Lk[j][k];
            Ak[i][j] = rtemp; Ak[j][i] = rtemp;
            rtemp = 0.0;
            for (k = 0; k <= j; k++) rtemp = rtemp + Ll[i][k] * Ll[j][k];
            tAl[i][j] = rtemp; tAl[j][i] = rtemp;
        }
    /* matelem.f90:144-169: tAl = P' Al P, tBl = P' Bl P */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + P[k][i] * tAl[k][j];
                rtemp = rtemp + P[k][i] * tBl[k][j];
            }
            Wr1[i][j] = rnumb; Wr2[i][j] = rtemp;
        }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + Wr1[i][k] * P[k][j];
                rtemp = rtemp + Wr2[i][k] * P[k][j];
            }
            tAl[i][j] = rnumb; tAl[j][i] = rnumb;
            tBl[i][j] = rtemp; tBl[j][i] = rtemp;
        }
    /* matelem.f90:173-179 */
    det_Lk = 1.0; det_Ll = 1.0;
    for (i = 0; i < n; i++) { det_Lk = det_Lk * Lk[i][i]; det_Ll = det_Ll * Ll[i][i]; }
    /* matelem.f90:182-194: Ck holds Ck^* = Ak - iBk */
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            cnumb = CMPLX(Ak[j][i], -Bk[j][i]);
            Ck[j][i] = cnumb; Ck[i][j] = cnumb;
            cnumb = CMPLX(tAl[j][i], tBl[j][i]);
            tCl[j][i] = cnumb; tCl[i][j] = cnumb;
            cnumb = Ck[j][i] + tCl[j][i];
            tCkl[j][i] = cnumb; tCkl[i][j] = cnumb;
        }
    /* matelem.f90:203-217: pseudo-Cholesky tCkl = G G^T, det = prod pivots */
    det_tCkl = 1.0;
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            csum = tCkl[i][j];
            for (k = i - 1; k >= 0; k--) csum = csum - tCkl[i][k] * tCkl[j][k];
            if (i == j) {
                tCkl[i][i] = csqrt(csum);
                det_tCkl = det_tCkl * csum;
            } else {
                tCkl[j][i] = csum / tCkl[i][i];
            }
        }
    /* matelem.f90:221-241: invert G in place, then inv = G^-T G^-1 */
    for (i = 0; i < n; i++) {
        tCkl[i][i] = 1.0 / tCkl[i][i];
        for (j = i + 1; j < n; j++) {
            csum = 0.0;
            for (k = i; k <= j - 1; k++) csum = csum - tCkl[j][k] * tCkl[k][i];
            tCkl[j][i] = csum / tCkl[j][j];
        }
    }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            ctemp = 0.0;
            for (k = j; k < n; k++) ctemp = ctemp + tCkl[k][i] * tCkl[k][j];
            inv_tCkl[i][j] = ctemp; inv_tCkl[j][i] = ctemp;
        }
    /* matelem.f90:244-245 */
    cnumb = fabs(det_Ll * det_Lk) / det_tCkl;
    S = g_2r3n2 * cnumb * csqrt(cnumb);
    /* matelem.f90:248-274: kinetic energy */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            ctemp = 0.0;
            for (k = 0; k < n; k++) ctemp = ctemp + inv_tCkl[i][k] * Ck[k][j];
            Wc1[i][j] = ctemp;
        }
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            ctemp = 0.0;
            for (k = 0; k < n; k++) ctemp = ctemp + tCl[i][k] * Wc1[k][j];
            Wc2[i][j] = ctemp;
        }
    ctemp = 0.0;
    for (i = 0; i < n; i++)
        for (k = 0; k < n; k++) ctemp = ctemp + g_mass[i][k] * Wc2[k][i];
    Tkl = 6 * S * ctemp;
    /* matelem.f90:280-299: Coulomb */
    cnumb = (2.0 / SQRTPI) * S;
    ctemp = 0.0;
    for (i = 0; i < n; i++) {
        cmpnum = inv_tCkl[i][i];
        csum = csqrt(cmpnum);
        tr32[i][i] = 1.0 / (csum * cmpnum);
        cRklij = cnumb / csum;
        ctemp = ctemp + g_q[i] * cRklij;
    }
    ctemp = ctemp * g_q0;
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++) {
            cmpnum = inv_tCkl[i][i] + inv_tCkl[j][j] - inv_tCkl[j][i] - inv_tCkl[j][i];
            csum = csqrt(cmpnum);
            tr32[j][i] = 1.0 / (csum * cmpnum);
            cRklij = cnumb / csum;
            ctemp = ctemp + g_q[i] * g_q[j] * cRklij;
        }
    Vkl = ctemp;
    H = Tkl + Vkl;
    *Hkl = H;
    *Skl = S;
    if (!grad_k && !grad_l) return;

    /* ---- gradient of S, matelem.f90:306-423 ---- */
    if (grad_k) {
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = j; k < n; k++) csum = csum + inv_tCkl[i][k] * Lk[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) inv_Lk[j][i] = Lk[j][i];
        for (i = 0; i < n; i++) {
            inv_Lk[i][i] = 1.0 / inv_Lk[i][i];
            for (j = i + 1; j < n; j++) {
                inv_Lk[i][j] = 0.0;
                rsum = 0.0;
                for (k = i; k <= j - 1; k++) rsum = rsum - inv_Lk[j][k] * inv_Lk[k][i];
                inv_Lk[j][i] = rsum / inv_Lk[j][j];
            }
        }
        ctemp = S * 3.0 / 2.0;
        indx = 0;
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                dSdLk[indx] = (inv_Lk[i][j] - 2.0 * Wc1[j][i]) * ctemp;
                indx++;
            }
        ctemp = S * CMPLX(0.0, 3.0 / 2.0);
        cnumb = 2.0 * ctemp;
        indx = 0;
        for (i = 0; i < n; i++) {
            dSdBk[indx++] = inv_tCkl[i][i] * ctemp;
            for (j = i + 1; j < n; j++) dSdBk[indx++] = inv_tCkl[j][i] * cnumb;
        }
    }
    if (grad_l) {
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + P[i][k] * inv_tCkl[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * P[j][k];
                inv_ttCkl[i][j] = csum; inv_ttCkl[j][i] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + inv_ttCkl[i][k] * Ll[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) inv_Ll[j][i] = Ll[j][i];
        for (i = 0; i < n; i++) {
            inv_Ll[i][i] = 1.0 / inv_Ll[i][i];
            for (j = i + 1; j < n; j++) {
                inv_Ll[i][j] = 0.0;
                rsum = 0.0;
                for (k = i; k <= j - 1; k++) rsum = rsum - inv_Ll[j][k] * inv_Ll[k][i];
                inv_Ll[j][i] = rsum / inv_Ll[j][j];
            }
        }
        ctemp = S * 3.0 / 2.0;
        indx = 0;
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                dSdLl[indx] = (inv_Ll[i][j] - 2.0 * Wc1[j][i]) * ctemp;
                indx++;
            }
        ctemp = S * CMPLX(0.0, -3.0 / 2.0);
        cnumb = 2.0 * ctemp;
        indx = 0;
        for (i = 0; i < n; i++) {
            dSdBl[indx++] = inv_ttCkl[i][i] * ctemp;
            for (j = i + 1; j < n; j++) dSdBl[indx++] = inv_ttCkl[j][i] * cnumb;
        }
    }
    /* ---- gradient of T, matelem.f90:427-525 (ket), 527-598 (bra) ---- */
    if (grad_l) {
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Ck[i][k] * g_mass[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * Ck[k][j];
                Wc2[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + inv_tCkl[i][k] * Wc2[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * inv_tCkl[k][j];
                Wc2[i][j] = csum; Wc2[j][i] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + P[i][k] * Wc2[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * P[j][k];
                G[i][j] = csum; G[j][i] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = j; k < n; k++) csum = csum + G[i][k] * Ll[k][j];
                Wc1[i][j] = csum;
            }
        ctemp = Tkl / S;
        csum = 12 * S;
        indx = 0;
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                dHdLl[indx] = ctemp * dSdLl[indx] + csum * Wc1[j][i];
                indx++;
            }
        csum = S * CMPLX(0.0, 6.0);
        indx = 0;
        for (i = 0; i < n; i++) {
            dHdBl[indx] = ctemp * dSdBl[indx] + csum * G[i][i];
            indx++;
            for (j = i + 1; j < n; j++) {
                dHdBl[indx] = ctemp * dSdBl[indx] + 2.0 * csum * G[j][i];
                indx++;
            }
        }
    }
    if (grad_k) {
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + tCl[i][k] * g_mass[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * tCl[k][j];
                Wc2[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + inv_tCkl[i][k] * Wc2[k][j];
                Wc1[i][j] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                csum = 0.0;
                for (k = 0; k < n; k++) csum = csum + Wc1[i][k] * inv_tCkl[k][j];
                F[i][j] = csum; F[j][i] = csum;
            }
        for (i = 0; i < n; i++)
            for (j = 0; j < n; j++) {
                csum = 0.0;
                for (k = j; k < n; k++) csum = csum + F[i][k] * Lk[k][j];
                Wc1[i][j] = csum;
            }
        ctemp = Tkl / S;
        csum = 12 * S;
        indx = 0;
        for (i = 0; i < n; i++)
            for (j = i; j < n; j++) {
                dHdLk[indx] = ctemp * dSdLk[indx] + csum * Wc1[j][i];
                indx++;
            }
        csum = S * CMPLX(0.0, -6.0);
        indx = 0;
        for (i = 0; i < n; i++) {
            dHdBk[indx] = ctemp * dSdBk[indx] + csum * F[i][i];
            indx++;
            for (j = i + 1; j < n; j++) {
                dHdBk[indx] = ctemp * dSdBk[indx] + 2.0 * csum * F[j][i];
                indx++;
            }
        }
    }
    /* ---- gradient of V, matelem.f90:603-734 ---- */
    if (grad_k) for (i = 0; i < np; i++) { WVcLk[i] = 0.0; WVcBk[i] = 0.0; }
    if (grad_l) for (i = 0; i < np; i++) { WVcLl[i] = 0.0; WVcBl[i] = 0.0; }
    for (i = 0; i < n; i++)
        for (j = 0; j <= i; j++) {
            if (i == j) {
                for (k = 0; k < n; k++) {
                    tQ[k][k] = inv_tCkl[k][i] * inv_tCkl[i][k];
                    for (kk = k + 1; kk < n; kk++) {
                        cnumb = inv_tCkl[k][i] * inv_tCkl[i][kk];
                        tQ[k][kk] = cnumb; tQ[kk][k] = cnumb;
                    }
                }
            } else {
                for (k = 0; k < n; k++) {
                    tQ[k][k] = inv_tCkl[k][i] * inv_tCkl[i][k] + inv_tCkl[k][j] * inv_tCkl[j][k]
                             - inv_tCkl[k][i] * inv_tCkl[j][k] - inv_tCkl[k][j] * inv_tCkl[i][k];
                    for (kk = k + 1; kk < n; kk++) {
                        cnumb = inv_tCkl[k][i] * inv_tCkl[i][kk] + inv_tCkl[k][j] * inv_tCkl[j][kk]
                              - inv_tCkl[k][i] * inv_tCkl[j][kk] - inv_tCkl[k][j] * inv_tCkl[i][kk];
                        tQ[k][kk] = cnumb; tQ[kk][k] = cnumb;
                    }
                }
            }
            if (grad_k) {
                for (k = 0; k < n; k++)
                    for (kk = 0; kk <= k; kk++) {
                        csum = 0.0;
                        for (kkk = kk; kkk < n; kkk++) csum = csum + tQ[k][kkk] * Lk[kkk][kk];
                        Wc1[k][kk] = csum;
                    }
            }
            if (grad_l) {
                for (k = 0; k < n; k++)
                    for (kk = 0; kk < n; kk++) {
                        csum = 0.0;
                        for (kkk = 0; kkk < n; kkk++) csum = csum + P[k][kkk] * tQ[kkk][kk];
                        Wc2[k][kk] = csum;
                    }
                for (k = 0; k < n; k++)
                    for (kk = k; kk < n; kk++) {
                        csum = 0.0;
                        for (kkk = 0; kkk < n; kkk++) csum = csum + Wc2[k][kkk] * P[kk][kkk];
                        ttQ[k][kk] = csum; ttQ[kk][k] = csum;
                    }
                for (k = 0; k < n; k++)
                    for (kk = 0; kk <= k; kk++) {
                        csum = 0.0;
                        for (kkk = kk; kkk < n; kkk++) csum = csum + ttQ[k][kkk] * Ll[kkk][kk];
                        Wc2[k][kk] = csum;
                    }
            }
            if (i == j)
                cnumb = g_q0 * g_q[i] * tr32[i][i];
            else
                cnumb = g_q[i] * g_q[j] * tr32[i][j];
            if (grad_k) {
                indx = 0;
                for (k = 0; k < n; k++) {
                    WVcBk[indx] = WVcBk[indx] + cnumb * tQ[k][k];
                    WVcLk[indx] = WVcLk[indx] + cnumb * Wc1[k][k];
                    indx++;
                    for (kk = k + 1; kk < n; kk++) {
                        WVcBk[indx] = WVcBk[indx] + 2.0 * cnumb * tQ[kk][k];
                        WVcLk[indx] = WVcLk[indx] + cnumb * Wc1[kk][k];
                        indx++;
                    }
                }
            }
            if (grad_l) {
                indx = 0;
                for (k = 0; k < n; k++) {
                    WVcBl[indx] = WVcBl[indx] + cnumb * ttQ[k][k];
                    WVcLl[indx] = WVcLl[indx] + cnumb * Wc2[k][k];
                    indx++;
                    for (kk = k + 1; kk < n; kk++) {
                        WVcBl[indx] = WVcBl[indx] + 2.0 * cnumb * ttQ[kk][k];
                        WVcLl[indx] = WVcLl[indx] + cnumb * Wc2[kk][k];
                        indx++;
                    }
                }
            }
        }
    cnumb = (2.0 / SQRTPI) * S;
    ctemp = (CMPLX(0.0, 1.0) / SQRTPI) * S;
    if (grad_k)
        for (i = 0; i < np; i++) {
            dHdLk[i] = dHdLk[i] + (Vkl / S) * dSdLk[i] + cnumb * WVcLk[i];
            dHdBk[i] = dHdBk[i] + (Vkl / S) * dSdBk[i] - ctemp * WVcBk[i];
        }
    if (grad_l)
        for (i = 0; i < np; i++) {
            dHdLl[i] = dHdLl[i] + (Vkl / S) * dSdLl[i] + cnumb * WVcLl[i];
            dHdBl[i] = dHdBl[i] + (Vkl / S) * dSdBl[i] + ctemp * WVcBl[i];
        }
    /* matelem.f90:737-748 */
    if (grad_k)
        for (i = 0; i < np; i++) {
            Dk[i] = dHdLk[i]; Dk[np + i] = dHdBk[i];
            Dk[2 * np + i] = dSdLk[i]; Dk[3 * np + i] = dSdBk[i];
        }
    if (grad_l)
        for (i = 0; i < np; i++) {
            Dl[i] = dHdLl[i]; Dl[np + i] = dHdBl[i];
            Dl[2 * np + i] = dSdLl[i]; Dl[3 * np + i] = dSdBl[i];
        }
}

static void load_perm(const int *Pcm, int P[NN][NN])
{
    for (int i = 0; i < g_n; i++)
        for (int j = 0; j < g_n; j++) P[i][j] = Pcm[i + j * g_n];
}

/* Single MatrixElements call with an explicit permutation matrix. */
void orc_matrix_elements(const double *Paramk, const double *Paraml, const int *Pcm,
                         cplx *HS, cplx *Dk, cplx *Dl, int gradflag)
{
    int P[NN][NN];
    cplx dk[4 * NNP], dl[4 * NNP];
    load_perm(Pcm, P);
    matrix_elements(Paramk, Paraml, P, &HS[0], &HS[1], dk, dl, gradflag);
    if ((gradflag == 1 || gradflag == 3) && Dk) memcpy(Dk, dk, sizeof(cplx) * 4 * g_np);
    if ((gradflag == 2 || gradflag == 3) && Dl) memcpy(Dl, dl, sizeof(cplx) * 4 * g_np);
}

/* Sum over the Y^+Y terms as matform.f90:170-177 / 294-303 (one rank). */
static void pair_sum(const double *pk, const double *pl, int gradflag,
                     cplx *Hs, cplx *Ss, cplx *Dks, cplx *Dls)
{
    const int np4 = 4 * g_np;
    cplx Hkl, Skl, Dk[4 * NNP], Dl[4 * NNP];
    cplx Hsum = 0.0, Ssum = 0.0;
    if (gradflag) {
        for (int m = 0; m < np4; m++) Dks[m] = 0.0;
        if (gradflag == 3) for (int m = 0; m < np4; m++) Dls[m] = 0.0;
    }
    for (int t = 0; t < g_T; t++) {
        matrix_elements(pk, pl, g_P[t], &Hkl, &Skl, Dk, Dl, gradflag);
        Hsum = Hsum + g_coef[t] * Hkl;
        Ssum = Ssum + g_coef[t] * Skl;
        if (gradflag) {
            for (int m = 0; m < np4; m++) Dks[m] = Dks[m] + g_coef[t] * Dk[m];
            if (gradflag == 3) for (int m = 0; m < np4; m++) Dls[m] = Dls[m] + g_coef[t] * Dl[m];
        }
    }
    *Hs = Hsum;
    *Ss = Ssum;
}

#define IX(i, j, ld) ((size_t)((i) - 1) + (size_t)((j) - 1) * (size_t)(ld))

/* StoreHS, matform.f90:11-51.  i >= j, 1-based. */
static void store_hs(char method, double approx_e, int i, int j, cplx Hij, cplx Sij,
                     cplx *H, cplx *S, int ld, double *diagS, double *diagH)
{
    if (method == 'I') {
        if (i == j) {
            diagS[i - 1] = creal(Sij);
            S[IX(i, i, ld)] = 1.0;
            H[IX(i, i, ld)] = creal(Hij) / diagS[i - 1] - approx_e;
        } else {
            cplx f = 1.0 / sqrt(diagS[i - 1] * diagS[j - 1]);
            S[IX(i, j, ld)] = Sij * f;
            S[IX(j, i, ld)] = conj(S[IX(i, j, ld)]);
            H[IX(i, j, ld)] = (Hij - approx_e * Sij) * f;
        }
    } else {
        if (i == j) {
            diagS[i - 1] = creal(Sij);
            diagH[i - 1] = creal(Hij) / diagS[i - 1];
        } else {
            cplx f = 1.0 / sqrt(diagS[i - 1] * diagS[j - 1]);
            S[IX(i, j, ld)] = Sij * f;
            H[IX(i, j, ld)] = Hij * f;
        }
    }
}

/* ComputeMatElem + StoreHS (matform.f90:119-230).  params: npt x K col-major.
 * Diagonal pairs of rows nmin..nmax are stored first so that every
 * off-diagonal store finds both diagS entries, as in the reference's l=k..1
 * loop order. */
void orc_compute_mat_elem(const double *params, int nmin, int nmax, char method, double approx_e,
                          cplx *H, cplx *S, int ld, double *diagS, double *diagH)
{
    const int npt = g_npt;
    for (int k = nmin; k <= nmax; k++) {
        cplx h, s;
        pair_sum(params + (size_t)(k - 1) * npt, params + (size_t)(k - 1) * npt, 0, &h, &s, 0, 0);
        store_hs(method, approx_e, k, k, h, s, H, S, ld, diagS, diagH);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = nmax; k >= nmin; k--) {
        for (int l = k - 1; l >= 1; l--) {
            cplx h, s;
            pair_sum(params + (size_t)(k - 1) * npt, params + (size_t)(l - 1) * npt, 0, &h, &s, 0, 0);
            store_hs(method, approx_e, k, l, h, s, H, S, ld, diagS, diagH);
        }
    }
}

/* For the parity tests' tolerance scales: for every pair k >= l of
 * functions 1..K, aH = sum_t |coef_t| |H_t(k,l)| and aS likewise, as
 * (K x K) column-major arrays (lower triangle filled).  Not a reference
 * routine: the magnitude of the terms that ComputeMatElem sums. */
void orc_term_magnitudes(const double *params, int K, double *aH, double *aS)
{
    const int npt = g_npt;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 1; k <= K; k++) {
        for (int l = 1; l <= k; l++) {
            double h = 0.0, sm = 0.0;
            for (int t = 0; t < g_T; t++) {
                cplx Hkl, Skl;
                matrix_elements(params + (size_t)(k - 1) * npt, params + (size_t)(l - 1) * npt, g_P[t], &Hkl,
                                &Skl, 0, 0, 0);
                h += abs(g_coef[t]) * cabs(Hkl);
                sm += abs(g_coef[t]) * cabs(Skl);
            }
            aH[IX(k, l, K)] = h;
            aS[IX(k, l, K)] = sm;
        }
    }
}

/* StoreHSD, matform.f90:55-115.  D is (2npt, ldo, *) column-major. */
static void store_hsd(char method, double approx_e, int nfru, int i, int j, cplx Hij, cplx Sij,
                      const cplx *Di, const cplx *Dj, cplx *H, cplx *S, int ld, double *diagS,
                      double *diagH, cplx *D, int ldo)
{
    const int n2 = 2 * g_npt;
#define DX(m, a, b) ((size_t)(m) + (size_t)((a) - 1) * n2 + (size_t)((b) - 1) * (size_t)n2 * ldo)
    store_hs(method, approx_e, i, j, Hij, Sij, H, S, ld, diagS, diagH);
    if (i == j) {
        for (int m = 0; m < n2; m++) D[DX(m, i - nfru, i)] = 2 * creal(Di[m]) / diagS[i - 1];
    } else {
        cplx f = 1.0 / sqrt(diagS[i - 1] * diagS[j - 1]);
        for (int m = 0; m < n2; m++) D[DX(m, i - nfru, j)] = Di[m] * f;
        if (j > nfru)
            for (int m = 0; m < n2; m++) D[DX(m, j - nfru, i)] = conj(Dj[m] * f);
    }
#undef DX
}

/* ComputeMatElemAndDeriv + StoreHSD (matform.f90:234-360). */
void orc_compute_mat_elem_and_deriv(const double *params, int nmin, int nmax, int nfru, char method,
                                    double approx_e, cplx *H, cplx *S, int ld, double *diagS,
                                    double *diagH, cplx *D, int ldo)
{
    const int npt = g_npt;
    for (int k = nmin; k <= nmax; k++) {
        cplx h, s, Dk[4 * NNP], Dl[4 * NNP];
        pair_sum(params + (size_t)(k - 1) * npt, params + (size_t)(k - 1) * npt, 1, &h, &s, Dk, Dl);
        store_hsd(method, approx_e, nfru, k, k, h, s, Dk, Dl, H, S, ld, diagS, diagH, D, ldo);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = nmax; k >= nmin; k--) {
        for (int l = k - 1; l >= 1; l--) {
            cplx h, s, Dk[4 * NNP], Dl[4 * NNP];
            int gf = (l > nfru) ? 3 : 1;
            pair_sum(params + (size_t)(k - 1) * npt, params + (size_t)(l - 1) * npt, gf, &h, &s, Dk, Dl);
            store_hsd(method, approx_e, nfru, k, l, h, s, Dk, Dl, H, S, ld, diagS, diagH, D, ldo);
        }
    }
}

/* ---------------------------- linalg ---------------------------------- */

/* LDLHF serial branch, linalg.f90:356-392.  Returns ErrorCode. */
int orc_ldlhf(int m, int n, cplx *A, int ld, cplx *invD, cplx *w)
{
    for (int i = m; i <= n; i++) {
        for (int j = 1; j <= i; j++) {
            int jm = j - 1;
            cplx x;
            if (i == j) {
                for (int q = 1; q <= jm; q++) w[q - 1] = A[IX(q, i, ld)] * invD[q - 1];
                x = A[IX(i, j, ld)];
                for (int q = 1; q <= jm; q++) x = x - conj(A[IX(q, i, ld)]) * w[q - 1];
                x = conj(x);
                for (int q = 1; q <= jm; q++) A[IX(q, i, ld)] = w[q - 1];
                if (x == 0.0) return 1;
                invD[j - 1] = 1.0 / x;
            } else {
                x = A[IX(i, j, ld)];
                for (int q = 1; q <= jm; q++) x = x - conj(A[IX(q, i, ld)]) * A[IX(q, j, ld)];
                A[IX(j, i, ld)] = conj(x);
            }
        }
    }
    return 0;
}

/* LDLHF parallel branch (Glob_LDLHF_PMode /= 0), linalg.f90:400-452, with
 * the OpenMP threads of one team as the MPI ranks (Glob_NumOfProcs = team
 * size, Glob_ProcID = thread number).  Row i of L^H is built in chunks of
 * NumOfProcs entries: rank r forms entry ji+r of the chunk from the part of
 * the row before the chunk (one dot product), the chunk is gathered (the
 * reference's MPI_ALLREDUCE over entries that only one rank set), and every
 * entry then takes the within-chunk terms in order.  The diagonal term is a
 * strided partial sum per rank, reduced.  A barrier stands in for each
 * ALLREDUCE; the within-chunk steps, which every rank repeats identically
 * in the reference, run once.  Returns ErrorCode. */
int orc_ldlhf_par(int m, int n, cplx *A, int ld, cplx *invD, cplx *w)
{
    int err = 0;
    cplx part[256];
#pragma omp parallel
    {
#ifdef _OPENMP
        const int np = omp_get_num_threads() > 256 ? 256 : omp_get_num_threads();
        const int id = omp_get_thread_num();
#else
        const int np = 1, id = 0;
#endif
        for (int i = m; i <= n && !err; i++) {
            const int im = i - 1;
#pragma omp single
            for (int q = 1; q <= im; q++) A[IX(q, i, ld)] = 0.0;
            const int rows = im / np, rem = im % np;
            for (int k = 1; k <= rows + (rem > 0); k++) {
                const int ji = (k - 1) * np + 1, jim = ji - 1;
                const int jf = (k <= rows) ? k * np : im;
                const int jiR = ji + id;
                if (id < np && jiR <= jf) {
                    /* A(jiR,i) = conjg(-dot_product(A(1:jim,i), A(1:jim,jiR))) */
                    cplx d = 0.0;
                    for (int q = 1; q <= jim; q++) d = d + conj(A[IX(q, i, ld)]) * A[IX(q, jiR, ld)];
                    A[IX(jiR, i, ld)] = conj(-d);
                }
#pragma omp barrier
#pragma omp single
                for (int j = ji; j <= jf; j++) {
                    /* A(j,i) += conjg(A(i,j) - dot_product(A(ji:jm,i), A(ji:jm,j))) */
                    cplx d = 0.0;
                    for (int q = ji; q <= j - 1; q++) d = d + conj(A[IX(q, i, ld)]) * A[IX(q, j, ld)];
                    A[IX(j, i, ld)] = A[IX(j, i, ld)] + conj(A[IX(i, j, ld)] - d);
                }
            }
            /* the j == 1 (diagonal) case */
#pragma omp for schedule(static)
            for (int q = 1; q <= im; q++) w[q - 1] = A[IX(q, i, ld)] * invD[q - 1];
            cplx y = 0.0;
            for (int q = 1 + id; q <= im; q += np) y = y + conj(A[IX(q, i, ld)]) * w[q - 1];
            if (id < 256) part[id] = conj(y);
#pragma omp barrier
#pragma omp single
            {
                cplx x = 0.0;
                for (int r = 0; r < np; r++) x = x + part[r];
                x = A[IX(i, i, ld)] - x;
                for (int q = 1; q <= im; q++) A[IX(q, i, ld)] = w[q - 1];
                if (x == 0.0)
                    err = 1;
                else
                    invD[i - 1] = 1.0 / x;
            }
        }
    }
    return err;
}

/* Which LDLHF branch GHEPIIS calls: 0 serial, 1 parallel, -1 (default) as
 * linalg_setparam('marin') picks it for NumOfProcs = the thread count:
 * parallel when NumOfProcs >= 8 and n > 5000 or NumOfProcs >= 16 and
 * n > 3000 (src/linalg.f90:113-121). */
static int g_ldlhf_mode = -1;

void orc_set_ldlhf_mode(int mode) { g_ldlhf_mode = mode; }

static int ldlhf_parallel(int n)
{
    if (g_ldlhf_mode >= 0) return g_ldlhf_mode;
#ifdef _OPENMP
    const int procs = omp_get_max_threads();
#else
    const int procs = 1;
#endif
    return (procs >= 8 && n > 5000) || (procs >= 16 && n > 3000);
}

int orc_ldlhf_auto(int m, int n, cplx *A, int ld, cplx *invD, cplx *w)
{
    return ldlhf_parallel(n) ? orc_ldlhf_par(m, n, A, ld, invD, w) : orc_ldlhf(m, n, A, ld, invD, w);
}

/* LDLHS non-BLAS branch, linalg.f90:634-653 (the BLAS branch at :655-660
 * computes the same two unit triangular solves with ZTRSV). */
void orc_ldlhs(int n, const cplx *A, int ld, const cplx *invD, const cplx *b, cplx *x)
{
    for (int i = 0; i < n; i++) x[i] = b[i];
    for (int j = 1; j <= n; j++) {
        cplx t = x[j - 1];
        for (int i = 1; i <= j - 1; i++) t = t - conj(A[IX(i, j, ld)]) * x[i - 1];
        x[j - 1] = t;
    }
    for (int i = 0; i < n; i++) x[i] = x[i] * invD[i];
    for (int j = n; j >= 1; j--) {
        cplx t = x[j - 1];
        for (int i = j - 1; i >= 1; i--) x[i - 1] = x[i - 1] - t * A[IX(i, j, ld)];
    }
}

/* MHMV non-BLAS branch, linalg.f90:1033-1041: y = A^H x. */
static void mhmv(int n, const cplx *A, int ld, const cplx *x, cplx *y)
{
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= n; i++) {
        cplx t = 0.0;
        for (int j = 1; j <= n; j++) t = t + conj(A[IX(j, i, ld)]) * x[j - 1];
        y[i - 1] = t;
    }
}

/* VMMHMV serial branch, linalg.f90:1195-1206: x^H A x from the lower triangle. */
double orc_vmmhmv(int n, const cplx *A, int ld, const cplx *x)
{
    double v = 0.0;
    for (int k = 1; k <= n; k++) {
        double xr = creal(x[k - 1]), xi = cimag(x[k - 1]);
        v = v + (xr * xr + xi * xi) * creal(A[IX(k, k, ld)]);
        double sr = 0.0, si = 0.0;
        for (int j = k + 1; j <= n; j++) {
            cplx a = A[IX(j, k, ld)];
            sr = sr + (creal(x[j - 1]) * creal(a) + cimag(x[j - 1]) * cimag(a));
            si = si + (cimag(x[j - 1]) * creal(a) - creal(x[j - 1]) * cimag(a));
        }
        v = v + 2.0 * (xr * sr + xi * si);
    }
    return v;
}

static double cmax_abs_re_or_im(int n, const cplx *x)
{
    double m = 0.0, t;
    for (int j = 0; j < n; j++) {
        t = fabs(creal(x[j])); if (t > m) m = t;
        t = fabs(cimag(x[j])); if (t > m) m = t;
    }
    return m;
}

/* CVScale with a real alpha, linalg.f90:1548-1553. */
static void cvscale_real(int n, cplx *x, double a)
{
    for (int j = 0; j < n; j++) x[j] = CMPLX(a * creal(x[j]), a * cimag(x[j]));
}

static cplx cdot_quotient(int n, const cplx *x, const cplx *y)
{
    cplx a = 0.0;
    double r = 0.0;
    for (int j = 0; j < n; j++) {
        a = a + conj(x[j]) * y[j];
        r = r + creal(y[j]) * creal(y[j]) + cimag(y[j]) * cimag(y[j]);
    }
    return CMPLX(creal(a) / r, cimag(a) / r);
}

static double cvdiff_eucnorm(int n, const cplx *x, cplx alpha, const cplx *y)
{
    double s2 = 0.0;
    for (int j = 0; j < n; j++) {
        cplx s = x[j] - alpha * y[j];
        s2 = s2 + creal(s) * creal(s) + cimag(s) * cimag(s);
    }
    return sqrt(s2);
}

static double cdot_itself(int n, const cplx *x)
{
    double s = 0.0;
    for (int j = 0; j < n; j++) s = s + creal(x[j]) * creal(x[j]) + cimag(x[j]) * cimag(x[j]);
    return s;
}

/* GHEPIIS, linalg.f90:1781-1926.  v is overwritten (work), x receives the
 * eigenvector.  out[0]=lambda, out[1]=RelAcc; iout[0]=NumIter.  Returns
 * ErrorCode (0, 1 = singular pivot, 2 = not converged). */
int orc_ghepiis(int k, int n, cplx *M, int ldm, cplx *invD, const cplx *B, int ldb,
                double apprlambda, cplx *v, cplx *w, double tol, cplx *x, int maxiter,
                int specif_norm, double *out, int *iout)
{
    double NormOfDiff = 0.0, NormOfDiffPrev = DBL_MAX, t1, t2, sqrtn;
    int NumIter = 0, notconverged = 1, err;
    cplx tc;
    out[1] = DBL_MAX;
    iout[0] = 0;
    err = orc_ldlhf_auto(k, n, M, ldm, invD, w);
    if (err > 0) return err;
    sqrtn = sqrt(2 * n * 1.0);
    while (notconverged && NumIter < maxiter) {
        if (NumIter != 0) memcpy(v, x, sizeof(cplx) * n);
        mhmv(n, B, ldb, v, w);
        orc_ldlhs(n, M, ldm, invD, w, x);
        t1 = cmax_abs_re_or_im(n, x);
        cvscale_real(n, x, 1.0 / t1);
        tc = cdot_quotient(n, x, v);
        NormOfDiff = sqrtn * cvdiff_eucnorm(n, x, tc, v);
        if (tol > 0.0) {
            if (NormOfDiff <= tol) notconverged = 0;
        } else {
            if (NormOfDiff > NormOfDiffPrev && NormOfDiff <= fabs(tol)) notconverged = 0;
            NormOfDiffPrev = NormOfDiff;
        }
        NumIter++;
    }
    out[1] = NormOfDiff;
    err = notconverged ? 2 : 0;
    t1 = orc_vmmhmv(n, B, ldb, x);
    t2 = orc_vmmhmv(n, M, ldm, x);
    out[0] = t2 / t1 + apprlambda;
    if (specif_norm == 0) {
        cvscale_real(n, x, 1.0 / sqrt(t1));
    } else if (specif_norm == 1) {
        t1 = cdot_itself(n, x);
        cvscale_real(n, x, 1.0 / sqrt(t1));
    }
    iout[0] = NumIter;
    return err;
}

/* Gradient contraction of EnergyIB / EnergyGB, workproc.f90:2127-2142
 * (one rank).  D is (2npt, ldo, nfa); c has nfa entries; grad has npt*nfo. */
void orc_gradient_contract(int nfo, int nfa, int nfru, const cplx *D, int ldo, const cplx *c,
                           double E, double *grad)
{
    const int npt = g_npt, n2 = 2 * g_npt;
#define DX(m, a, b) ((size_t)(m) + (size_t)((a) - 1) * n2 + (size_t)((b) - 1) * (size_t)n2 * ldo)
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= nfo; k++) {
        cplx W[2 * NNP];
        for (int m = 0; m < npt; m++) W[m] = 0.0;
        for (int l = 1; l <= nfa; l++) {
            cplx t = c[l - 1];
            for (int m = 0; m < npt; m++)
                W[m] = W[m] + t * (D[DX(m, k, l)] - E * D[DX(m + npt, k, l)]);
        }
        cplx t = c[k + nfru - 1];
        for (int m = 0; m < npt; m++) grad[(size_t)(k - 1) * npt + m] = 2 * creal(conj(t) * W[m]);
        for (int m = 0; m < npt; m++)
            grad[(size_t)(k - 1) * npt + m] =
                creal(grad[(size_t)(k - 1) * npt + m] -
                      t * conj(t) * (D[DX(m, k, k + nfru)] - E * D[DX(m + npt, k, k + nfru)]));
    }
#undef DX
}

/* ComputeOverlapPenalty (WkGR == NULL) and ComputeOverlapPenaltyAndAddGradient
 * (WkGR != NULL: the penalty gradient is added to it), src/workproc.f90:
 * 1491-1693, NumOfProcs = 1 branch.  S is Glob_S (its strict lower triangle
 * is read, S(j,i) with j > i), D is Glob_D as orc_gradient_contract takes it.
 * Returns TotalPenalty.
 * exact = 1 replaces the reference's gradient by the derivative of its
 * penalty: the reference's normalisation terms carry a factor
 * sqrt(diagS_i/diagS_j) and, for the function of the lower index, S_ji^2
 * where the derivative has |S_ji|^2 and conj(Glob_D(.,i-nfru,j)). */
double orc_overlap_penalty(int nfru, int nfa, double max_pen, double thr2, const cplx *S, int ld,
                           const double *diagS, const cplx *D, int ldo, double *WkGR, int exact)
{
    const int npt = g_npt, n2 = 2 * g_npt;
#define DX(m, a, b) ((size_t)(m) + (size_t)((a) - 1) * n2 + (size_t)((b) - 1) * (size_t)n2 * ldo)
#define SX(j, i) ((size_t)((j) - 1) + (size_t)((i) - 1) * (size_t)ld)
    double tp = 0.0, aux, temp2;
    const double pen_coeff = max_pen / (1.0 - thr2);
    const double temp1 = 2 * pen_coeff;
    for (int i = 1; i <= nfru; i++)
        for (int j = nfru + 1; j <= nfa; j++) {
            const cplx Sji = S[SX(j, i)];
            aux = creal(Sji) * creal(Sji) + cimag(Sji) * cimag(Sji);
            if (aux > thr2) {
                tp = tp + pen_coeff * (aux - thr2);
                if (WkGR) {
                    temp2 = exact ? 1.0 : sqrt(diagS[i - 1] / diagS[j - 1]);
                    for (int m = 1; m <= npt; m++)
                        WkGR[(size_t)(j - nfru - 1) * npt + m - 1] =
                            WkGR[(size_t)(j - nfru - 1) * npt + m - 1] +
                            temp1 * creal(Sji * conj(D[DX(npt + m - 1, j - nfru, i)] -
                                                     0.5 * D[DX(npt + m - 1, j - nfru, j)] * Sji * temp2));
                }
            }
        }
    for (int i = nfru + 1; i <= nfa; i++)
        for (int j = i + 1; j <= nfa; j++) {
            const cplx Sji = S[SX(j, i)];
            aux = creal(Sji) * creal(Sji) + cimag(Sji) * cimag(Sji);
            if (aux > thr2) {
                tp = tp + pen_coeff * (aux - thr2);
                if (WkGR) {
                    temp2 = exact ? 1.0 : sqrt(diagS[i - 1] / diagS[j - 1]);
                    const cplx Sn = exact ? conj(Sji) : Sji;
                    for (int m = 1; m <= npt; m++)
                        WkGR[(size_t)(i - nfru - 1) * npt + m - 1] =
                            WkGR[(size_t)(i - nfru - 1) * npt + m - 1] +
                            temp1 * creal(Sji * (D[DX(npt + m - 1, i - nfru, j)] -
                                                 0.5 * D[DX(npt + m - 1, i - nfru, i)] * Sn / temp2));
                    for (int m = 1; m <= npt; m++)
                        WkGR[(size_t)(j - nfru - 1) * npt + m - 1] =
                            WkGR[(size_t)(j - nfru - 1) * npt + m - 1] +
                            temp1 * creal(Sji * conj(D[DX(npt + m - 1, j - nfru, i)] -
                                                     0.5 * D[DX(npt + m - 1, j - nfru, j)] * Sji * temp2));
                }
            }
        }
#undef DX
#undef SX
    return tp;
}

void orc_set_threads(int nt)
{
#ifdef _OPENMP
    if (nt > 0) omp_set_num_threads(nt);
#else
    (void)nt;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
