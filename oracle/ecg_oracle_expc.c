/*
 * ecg_oracle_expc.c -- CPU restatement of the expectation-value pair term
 * and of the accumulation loop of ExpectationValuesG.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker of ecg_expectation_values;
 * see the header of ecg_oracle.c).
 *
 * Restated, with the loop structure and operation order of the Fortran
 * source (paths relative to the reference project root):
 *
 *   MatrixElementsForExpcVals   src/matelem.f90:949-1983
 *   ME_rXr_over_rij             src/matelem.f90:753-818
 *   ME_rXr_rYr_over_rij         src/matelem.f90:821-945
 *   trace, ME_dXd_dYd, ME_dXd, ME_dXd_over_rij
 *                               src/matelem.f90:1986-2044
 *   ExpectationValuesG, main loop and error estimates
 *                               src/workproc.f90:8159-8366
 *   Glob_bvc                    src/workproc.f90:612-621
 *
 * The tensor TrCJCJ(i,j,p,q) of src/matelem.f90:1304-1330 is never assigned
 * for i = j < p < q (n >= 3), yet the 1/(r_ij r_pq) loop at :1334-1371 reads
 * it there.  The reference is built with ifort and no -save/-auto option,
 * which places local arrays in static, zero-initialised storage, so those
 * entries read as zero and take the `caux == 0` branch.  This restatement
 * clears the tensor on every call to keep exactly that behaviour.
 *
 * Fortran's matmul in the ME_dX* helpers is restated as the plain triple
 * loop with the inner sum in ascending order.
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

#ifdef ORC_LONG
/* Extended-precision build of the same source (x87 long double, 64-bit
 * significand), used by the tests as a more accurate evaluation of the
 * same formulas: public names get the suffix _ld. */
typedef long double xreal;
typedef long double complex xcplx;
#define XCSQRT csqrtl
#define XCLOG clogl
#define XCEXP cexpl
#define XFABS fabsl
#define XSQRT sqrtl
#define XCMPLX CMPLXL
#define XCREAL creall
#define XCIMAG cimagl
#define ORC_NAME(x) x##_ld
static const xreal PI_ = 3.14159265358979323846264338327950288L;
static const xreal XSQRTPI = 1.77245385090551602729816748334114518L;
#else
typedef double xreal;
typedef cplx xcplx;
#define XCSQRT csqrt
#define XCLOG clog
#define XCEXP cexp
#define XFABS fabs
#define XSQRT sqrt
#define XCMPLX CMPLX
#define XCREAL creal
#define XCIMAG cimag
#define ORC_NAME(x) x
static const xreal PI_ = 3.14159265358979323846264338327950;
#define XSQRTPI SQRTPI
#endif


static xreal g_pmass[NN + 1];     /* Glob_Mass(1..n+1): m0, m1..mn */
static xreal g_bvc[NN][NN + 1];   /* Glob_bvc(1:n, 1:n+1) */
static xreal g_curr_energy;       /* Glob_CurrEnergy */

/* Glob_Mass and Glob_bvc (src/workproc.f90:612-621). */
int ORC_NAME(orc_set_masses)(const double *masses)
{
    const int n = g_n, npart = n + 1;
    xreal Mtot = 0.0;
    for (int i = 0; i < npart; i++) g_pmass[i] = masses[i];
    for (int i = 0; i < npart; i++) Mtot += g_pmass[i];
    for (int i = 0; i < npart; i++)
        for (int p = 0; p < n; p++) g_bvc[p][i] = -g_pmass[p + 1] / Mtot;
    for (int i = 1; i < npart; i++) g_bvc[i - 1][i] = g_bvc[i - 1][i] + 1.0;
    return 0;
}

typedef xcplx Mat[NN][NN];

static xcplx trace(int k, Mat M)
{
    xcplx t = 0.0;
    for (int i = 0; i < k; i++) t = t + M[i][i];
    return t;
}

/* Fortran matmul of two n x n complex matrices. */
static void matmul(Mat A, Mat B, Mat C)
{
    const int n = g_n;
    Mat R;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            xcplx s = 0.0;
            for (int k = 0; k < n; k++) s = s + A[i][k] * B[k][j];
            R[i][j] = s;
        }
    memcpy(C, R, sizeof(Mat));
}

/* ME_rXr_over_rij, src/matelem.f90:753-818.  i, j 0-based. */
static xcplx me_rxr_over_rij(Mat X, int i, int j, Mat invCkl, xcplx me1, xcplx TrCJ)
{
    const int n = g_n;
    xcplx CXi[NN], CXj[NN], TrCX = 0.0, TrCXCJ;
    for (int m = 0; m < n; m++)
        for (int p = 0; p < n; p++) TrCX = TrCX + invCkl[m][p] * X[p][m];
    for (int m = 0; m < n; m++) {
        CXi[m] = 0.0;
        for (int p = 0; p < n; p++) CXi[m] = CXi[m] + invCkl[i][p] * X[p][m];
    }
    if (j != i)
        for (int m = 0; m < n; m++) {
            CXj[m] = 0.0;
            for (int p = 0; p < n; p++) CXj[m] = CXj[m] + invCkl[j][p] * X[p][m];
        }
    TrCXCJ = 0.0;
    if (i == j) {
        for (int m = 0; m < n; m++) TrCXCJ = TrCXCJ + CXi[m] * invCkl[m][i];
    } else {
        for (int m = 0; m < n; m++) TrCXCJ = TrCXCJ + (CXi[m] - CXj[m]) * (invCkl[m][i] - invCkl[m][j]);
    }
    return me1 * (3 * TrCX - TrCXCJ / TrCJ) / 2;
}

/* ME_rXr_rYr_over_rij, src/matelem.f90:821-945. */
static xcplx me_rxr_ryr_over_rij(Mat X, Mat Y, int i, int j, Mat invCkl, xcplx me1, xcplx TrCJ)
{
    const int n = g_n;
    Mat Ys, Xs, CX, CY;
    xcplx CXCYi[NN], CXCYj[NN];
    xcplx TrCX, TrCY, TrCXCY, TrCXCJ, TrCYCJ, TrCXCYCJ;
    for (int p = 0; p < n; p++) {
        Ys[p][p] = Y[p][p];
        for (int q = p + 1; q < n; q++) {
            Ys[p][q] = (Y[p][q] + Y[q][p]) / 2;
            Ys[q][p] = Ys[p][q];
        }
    }
    for (int p = 0; p < n; p++) {
        Xs[p][p] = X[p][p];
        for (int q = p + 1; q < n; q++) {
            Xs[p][q] = (X[p][q] + X[q][p]) / 2;
            Xs[q][p] = Xs[p][q];
        }
    }
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) {
            CY[p][q] = 0.0;
            for (int m = 0; m < n; m++) CY[p][q] = CY[p][q] + invCkl[p][m] * Ys[m][q];
        }
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) {
            CX[p][q] = 0.0;
            for (int m = 0; m < n; m++) CX[p][q] = CX[p][q] + invCkl[p][m] * Xs[m][q];
        }
    for (int m = 0; m < n; m++) {
        CXCYi[m] = 0.0;
        for (int p = 0; p < n; p++) CXCYi[m] = CXCYi[m] + CX[i][p] * CY[p][m];
    }
    if (j != i)
        for (int m = 0; m < n; m++) {
            CXCYj[m] = 0.0;
            for (int p = 0; p < n; p++) CXCYj[m] = CXCYj[m] + CX[j][p] * CY[p][m];
        }
    TrCY = 0.0;
    TrCX = 0.0;
    for (int m = 0; m < n; m++) {
        TrCY = TrCY + CY[m][m];
        TrCX = TrCX + CX[m][m];
    }
    TrCXCY = 0.0;
    for (int m = 0; m < n; m++)
        for (int p = 0; p < n; p++) TrCXCY = TrCXCY + CX[m][p] * CY[p][m];
    TrCXCJ = 0.0;
    TrCYCJ = 0.0;
    TrCXCYCJ = 0.0;
    if (i == j) {
        for (int m = 0; m < n; m++) TrCXCJ = TrCXCJ + CX[i][m] * invCkl[m][i];
        for (int m = 0; m < n; m++) TrCYCJ = TrCYCJ + CY[i][m] * invCkl[m][i];
        for (int m = 0; m < n; m++) TrCXCYCJ = TrCXCYCJ + CXCYi[m] * invCkl[m][i];
    } else {
        for (int m = 0; m < n; m++) TrCXCJ = TrCXCJ + (CX[i][m] - CX[j][m]) * (invCkl[m][i] - invCkl[m][j]);
        for (int m = 0; m < n; m++) TrCYCJ = TrCYCJ + (CY[i][m] - CY[j][m]) * (invCkl[m][i] - invCkl[m][j]);
        for (int m = 0; m < n; m++)
            TrCXCYCJ = TrCXCYCJ + (CXCYi[m] - CXCYj[m]) * (invCkl[m][i] - invCkl[m][j]);
    }
    return me1 * (9 * TrCY * TrCX + 6 * TrCXCY - (3 * (TrCY * TrCXCJ + TrCX * TrCYCJ) + 4 * TrCXCYCJ) / TrCJ +
                  3 * TrCXCJ * TrCYCJ / (TrCJ * TrCJ)) / 4;
}

/* ME_dXd_dYd, src/matelem.f90:1998-2016. */
static xcplx me_dxd_dyd(Mat X, Mat Y, Mat invCkl, Mat tCk, Mat tCl, xcplx Skl)
{
    const int n = g_n;
    Mat M, MM, Z, T1, T2;
    xcplx tr1, tr2, tr3, tr4, tr5;
    matmul(X, tCk, M);
    tr1 = trace(n, M);
    matmul(tCl, Y, M);
    tr2 = trace(n, M);
    matmul(X, tCk, T1);
    matmul(tCk, T1, T2);
    matmul(invCkl, T2, M);
    tr3 = trace(n, M);
    matmul(Y, tCl, T1);
    matmul(tCl, T1, T2);
    matmul(invCkl, T2, MM);
    tr4 = trace(n, MM);
    matmul(M, MM, Z);
    tr5 = trace(n, Z);
    return (36 * tr3 * tr4 + 24 * tr5 - 36 * tr1 * tr4 - 36 * tr2 * tr3 + 36 * tr1 * tr2) * Skl;
}

/* ME_dXd, src/matelem.f90:2018-2030. */
static xcplx me_dxd(Mat X, Mat invCkl, Mat tCl, xcplx Skl)
{
    const int n = g_n;
    Mat M, T1, T2;
    xcplx tr1, tr2;
    matmul(tCl, X, M);
    tr1 = trace(n, M);
    matmul(X, tCl, T1);
    matmul(tCl, T1, T2);
    matmul(invCkl, T2, M);
    tr2 = trace(n, M);
    return 6 * (tr2 - tr1) * Skl;
}

/* ME_dXd_over_rij, src/matelem.f90:2032-2044. */
static xcplx me_dxd_over_rij(Mat X, int i, int j, Mat invCkl, Mat tCl, xcplx me1, xcplx TrCJ)
{
    const int n = g_n;
    Mat M, Z, T1;
    xcplx tr1;
    matmul(X, tCl, T1);
    matmul(tCl, T1, M);
    matmul(tCl, X, Z);
    tr1 = trace(n, Z);
    return 4 * me_rxr_over_rij(M, i, j, invCkl, me1, TrCJ) - 6 * tr1 * me1;
}

/* Outputs of one MatrixElementsForExpcVals call.  The n x n arrays are
 * [row][col] as the Fortran (row, col). */
typedef struct {
    xcplx H, S, T, V, MV, drach_MV, Darwin, drach_Darwin, OO;
    xcplx rm2[NN][NN], rm[NN][NN], r[NN][NN], r2[NN][NN], deltar[NN][NN], drach_deltar[NN][NN];
} ExpcTerm;

/* MatrixElementsForExpcVals, src/matelem.f90:949-1983.  Pbra, Pket are
 * [row][col]; CFkl is np x ncf (column-major, vech order), Denskl is
 * (n+1) x ndens. */
static void expc_matrix_elements(const double *Paramk, const double *Paraml, int Pbra[NN][NN], int Pket[NN][NN],
                                 ExpcTerm *o, int ncf, const double *CFGrid, xcplx *CFkl, int ndens,
                                 const double *DensGrid, xcplx *Denskl)
{
    const int n = g_n, np = g_np;
    xreal vechLk[NNP], vechBk[NNP], vechLl[NNP], vechBl[NNP];
    xreal Lk[NN][NN], Ll[NN][NN];
    xreal tAk[NN][NN], tAl[NN][NN], tBk[NN][NN], tBl[NN][NN];
    Mat tCk, tCl, tCkl, tCkl_copy, inv_tCkl, Wc1, Wc2, Wc3, Wc4, Wc5;
    xreal Wr1[NN][NN], Wr2[NN][NN];
    xreal rtemp, rnumb;
    xcplx ctemp, csum, cnumb, cmpnum, caux, caux1, tr1, tr2, tr3, tr4, tr5;
    xreal det_Lk, det_Ll;
    xcplx det_tCkl, Skl, Tkl, Vkl;
    int i, j, k, p, q, indx;
    static __thread xcplx TrCJCJ[NN][NN][NN][NN];
    static __thread xcplx rmrmkl[NN][NN][NN][NN];
    Mat TrCJ;
    xreal Mass_For_Darwin[NN + 1];

    for (i = 0; i < np; i++) {
        vechLk[i] = Paramk[i];
        vechBk[i] = Paramk[np + i];
        vechLl[i] = Paraml[i];
        vechBl[i] = Paraml[np + i];
    }
    /* :1038-1072 */
    indx = 0;
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            Lk[i][j] = 0.0; Lk[j][i] = vechLk[indx];
            Ll[i][j] = 0.0; Ll[j][i] = vechLl[indx];
            tBk[j][i] = vechBk[indx]; tBk[i][j] = vechBk[indx];
            tBl[j][i] = vechBl[indx]; tBl[i][j] = vechBl[indx];
            indx++;
        }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            rtemp = 0.0;
            for (k = 0; k <= j; k++) rtemp = rtemp + Lk[i][k] * Lk[j][k];
            tAk[i][j] = rtemp; tAk[j][i] = rtemp;
            rtemp = 0.0;
            for (k = 0; k <= j; k++) rtemp = rtemp + Ll[i][k] * Ll[j][k];
            tAl[i][j] = rtemp; tAl[j][i] = rtemp;
        }
    /* :1074-1125: tAk = Pbra' Ak Pbra, tBk likewise; tAl, tBl with Pket */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + Pbra[k][i] * tAk[k][j];
                rtemp = rtemp + Pbra[k][i] * tBk[k][j];
            }
            Wr1[i][j] = rnumb; Wr2[i][j] = rtemp;
        }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + Wr1[i][k] * Pbra[k][j];
                rtemp = rtemp + Wr2[i][k] * Pbra[k][j];
            }
            tAk[i][j] = rnumb; tAk[j][i] = rnumb;
            tBk[i][j] = rtemp; tBk[j][i] = rtemp;
        }
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + Pket[k][i] * tAl[k][j];
                rtemp = rtemp + Pket[k][i] * tBl[k][j];
            }
            Wr1[i][j] = rnumb; Wr2[i][j] = rtemp;
        }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            rnumb = 0.0; rtemp = 0.0;
            for (k = 0; k < n; k++) {
                rnumb = rnumb + Wr1[i][k] * Pket[k][j];
                rtemp = rtemp + Wr2[i][k] * Pket[k][j];
            }
            tAl[i][j] = rnumb; tAl[j][i] = rnumb;
            tBl[i][j] = rtemp; tBl[j][i] = rtemp;
        }
    /* :1127-1134 */
    det_Lk = 1.0; det_Ll = 1.0;
    for (i = 0; i < n; i++) { det_Lk = det_Lk * Lk[i][i]; det_Ll = det_Ll * Ll[i][i]; }
    /* :1136-1150 */
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            cnumb = XCMPLX(tAk[j][i], -tBk[j][i]);
            tCk[j][i] = cnumb; tCk[i][j] = cnumb;
            cnumb = XCMPLX(tAl[j][i], tBl[j][i]);
            tCl[j][i] = cnumb; tCl[i][j] = cnumb;
            cnumb = tCk[j][i] + tCl[j][i];
            tCkl[j][i] = cnumb; tCkl[i][j] = cnumb;
        }
    /* :1159-1174 pseudo-Cholesky */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) tCkl_copy[i][j] = tCkl[i][j];
    det_tCkl = 1.0;
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            csum = tCkl_copy[i][j];
            for (k = i - 1; k >= 0; k--) csum = csum - tCkl_copy[i][k] * tCkl_copy[j][k];
            if (i == j) {
                tCkl_copy[i][i] = XCSQRT(csum);
                det_tCkl = det_tCkl * csum;
            } else {
                tCkl_copy[j][i] = csum / tCkl_copy[i][i];
            }
        }
    /* :1178-1197 inverse */
    for (i = 0; i < n; i++) {
        tCkl_copy[i][i] = 1.0 / tCkl_copy[i][i];
        for (j = i + 1; j < n; j++) {
            csum = 0.0;
            for (k = i; k <= j - 1; k++) csum = csum - tCkl_copy[j][k] * tCkl_copy[k][i];
            tCkl_copy[j][i] = csum / tCkl_copy[j][j];
        }
    }
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++) {
            ctemp = 0.0;
            for (k = j; k < n; k++) ctemp = ctemp + tCkl_copy[k][i] * tCkl_copy[k][j];
            inv_tCkl[i][j] = ctemp; inv_tCkl[j][i] = ctemp;
        }
    /* :1200-1201 overlap */
    cnumb = XFABS(det_Ll * det_Lk) / det_tCkl;
    Skl = g_2r3n2 * cnumb * XCSQRT(cnumb);
    /* :1203-1229 kinetic energy */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            ctemp = 0.0;
            for (k = 0; k < n; k++) ctemp = ctemp + inv_tCkl[i][k] * tCk[k][j];
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
    Tkl = 6 * Skl * ctemp;
    /* :1231-1268 potential, 1/r, r, r^2, delta(r) */
    cnumb = (2.0 / XSQRTPI) * Skl;
    caux = 1.5 * Skl;
    ctemp = 0.0;
    caux1 = Skl / (PI_ * XSQRTPI);
    for (i = 0; i < n; i++) {
        TrCJ[i][i] = inv_tCkl[i][i];
        csum = XCSQRT(TrCJ[i][i]);
        o->rm[i][i] = cnumb / csum;
        o->r[i][i] = cnumb * csum;
        o->r2[i][i] = caux * TrCJ[i][i];
        o->deltar[i][i] = caux1 / (csum * TrCJ[i][i]);
        ctemp = ctemp + g_q[i] * o->rm[i][i];
    }
    ctemp = ctemp * g_q0;
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++) {
            TrCJ[i][j] = inv_tCkl[i][i] + inv_tCkl[j][j] - inv_tCkl[j][i] - inv_tCkl[j][i];
            TrCJ[j][i] = TrCJ[i][j];
            csum = XCSQRT(TrCJ[i][j]);
            o->rm[i][j] = cnumb / csum;
            o->rm[j][i] = o->rm[i][j];
            o->r[i][j] = cnumb * csum;
            o->r[j][i] = o->r[i][j];
            o->r2[i][j] = caux * TrCJ[i][j];
            o->r2[j][i] = o->r2[i][j];
            o->deltar[i][j] = caux1 / (csum * TrCJ[i][j]);
            o->deltar[j][i] = o->deltar[i][j];
            ctemp = ctemp + g_q[i] * g_q[j] * o->rm[i][j];
        }
    Vkl = ctemp;
    o->H = Tkl + Vkl;
    o->S = Skl;
    o->T = Tkl;
    o->V = Vkl;

    /* :1270-1300 tr[invC Jij invC Jpq] (entries the loop skips stay zero) */
    memset(TrCJCJ, 0, sizeof(TrCJCJ));
    for (i = 0; i < n; i++) {
        caux = inv_tCkl[i][i] * inv_tCkl[i][i];
        TrCJCJ[i][i][i][i] = caux;
        for (j = i + 1; j < n; j++) {
            caux = inv_tCkl[j][i] * inv_tCkl[j][i];
            TrCJCJ[j][j][i][i] = caux;
            TrCJCJ[i][i][j][j] = caux;
            for (p = i; p < n; p++) {
                ctemp = inv_tCkl[p][i] - inv_tCkl[p][j];
                caux = ctemp * ctemp;
                TrCJCJ[i][j][p][p] = caux;
                TrCJCJ[j][i][p][p] = caux;
                TrCJCJ[p][p][i][j] = caux;
                TrCJCJ[p][p][j][i] = caux;
                for (q = p + 1; q < n; q++) {
                    ctemp = inv_tCkl[q][i] - inv_tCkl[p][i] - inv_tCkl[q][j] + inv_tCkl[p][j];
                    caux = ctemp * ctemp;
                    TrCJCJ[i][j][p][q] = caux;
                    TrCJCJ[j][i][p][q] = caux;
                    TrCJCJ[i][j][q][p] = caux;
                    TrCJCJ[j][i][q][p] = caux;
                    TrCJCJ[p][q][i][j] = caux;
                    TrCJCJ[p][q][j][i] = caux;
                    TrCJCJ[q][p][i][j] = caux;
                    TrCJCJ[q][p][j][i] = caux;
                }
            }
        }
    }
    /* :1302-1339 (1/r_ij 1/r_pq) */
    cnumb = 4 * Skl / PI_;
    cmpnum = 2 * Skl;
    for (i = 0; i < n; i++)
        for (j = i; j < n; j++)
            for (p = i; p < n; p++)
                for (q = p; q < n; q++) {
                    if ((p == i && q == j) || (p == j && q == i)) {
                        ctemp = cmpnum / TrCJ[i][j];
                    } else {
                        caux = XCSQRT(TrCJCJ[i][j][p][q]);
                        if (caux != 0.0) {
                            caux1 = caux / XCSQRT(TrCJ[i][j] * TrCJ[p][q]);
                            csum = XCMPLX(0.0, -1.0) * XCLOG(XCMPLX(0.0, 1.0) * caux1 + XCSQRT(1.0 - caux1 * caux1));
                            ctemp = cnumb * csum / caux;
                        } else {
                            ctemp = cnumb / XCSQRT(TrCJ[i][j] * TrCJ[p][q]);
                        }
                    }
                    rmrmkl[i][j][p][q] = ctemp;
                    rmrmkl[j][i][p][q] = ctemp;
                    rmrmkl[i][j][q][p] = ctemp;
                    rmrmkl[j][i][q][p] = ctemp;
                    rmrmkl[p][q][i][j] = ctemp;
                    rmrmkl[p][q][j][i] = ctemp;
                    rmrmkl[q][p][i][j] = ctemp;
                    rmrmkl[q][p][j][i] = ctemp;
                }
    /* :1342-1346 */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) o->rm2[j][i] = rmrmkl[j][i][j][i];
    /* :1349-1392 Drachmanised delta(r_ij): Wc2 = tCk M tCl */
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            ctemp = 0.0;
            for (k = 0; k < n; k++) ctemp = ctemp + g_mass[i][k] * tCl[k][j];
            Wc1[i][j] = ctemp;
        }
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            ctemp = 0.0;
            for (k = 0; k < n; k++) ctemp = ctemp + tCk[i][k] * Wc1[k][j];
            Wc2[i][j] = ctemp;
        }
    for (p = 0; p < n; p++)
        for (q = p; q < n; q++) {
            ctemp = 0.0;
            for (i = 0; i < n; i++) {
                ctemp = ctemp + g_q0 * g_q[i] * rmrmkl[p][q][i][i];
                for (j = i + 1; j < n; j++) ctemp = ctemp + g_q[i] * g_q[j] * rmrmkl[p][q][i][j];
            }
            if (p == q)
                caux = 2 * PI_ * g_mass[p][p];
            else
                caux = 2 * PI_ * (g_mass[p][p] + g_mass[q][q] - g_mass[p][q] - g_mass[p][q]);
            cnumb = me_rxr_over_rij(Wc2, p, q, inv_tCkl, o->rm[p][q], TrCJ[p][q]);
            o->drach_deltar[p][q] = (g_curr_energy * o->rm[p][q] - ctemp - 4 * cnumb) / caux;
            o->drach_deltar[q][p] = o->drach_deltar[p][q];
        }
    /* :1394-1485 orbit-orbit */
    o->OO = 0.0;
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++) {
            tr1 = tCl[j][i];
            tr2 = tr1;
            tr3 = 3 * tCl[j][j];
            for (p = 0; p < n; p++)
                for (q = 0; q < n; q++) Wc1[q][p] = tCl[q][i] * tCl[p][j] + tCl[q][j] * tCl[p][i];
            for (p = 0; p < n; p++) Wc1[p][j] = Wc1[p][j] + tCkl[p][j] * tCl[j][i];
            for (p = 0; p < n; p++) Wc1[j][p] = Wc1[j][p] + tCl[i][j] * tCl[p][j] + tr3 * tCl[p][i];
            for (p = 0; p < n; p++)
                for (q = 0; q < n; q++) Wc2[p][q] = tCkl[p][j] * tCl[q][j];
            memset(Wc3, 0, sizeof(Mat));
            for (p = 0; p < n; p++) Wc3[j][p] = tCl[p][i];
            cnumb = me_rxr_over_rij(Wc1, j, j, inv_tCkl, o->rm[j][j], TrCJ[j][j]);
            ctemp = me_rxr_ryr_over_rij(Wc2, Wc3, j, j, inv_tCkl, o->rm[j][j], TrCJ[j][j]);
            caux = -6 * (tr1 + tr2) * o->rm[j][j] + 4 * cnumb - 8 * ctemp;
            o->OO = o->OO - caux * g_q[j] / g_pmass[j + 1];
        }
    o->OO = o->OO * g_q0 / g_pmass[0];
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++) {
            tr1 = tCl[j][i];
            tr2 = tr1;
            tr3 = 3 * tCl[j][j];
            for (p = 0; p < n; p++)
                for (q = 0; q < n; q++) Wc1[q][p] = tCl[q][i] * tCl[p][j] + tCl[q][j] * tCl[p][i];
            for (p = 0; p < n; p++) {
                Wc1[p][j] = Wc1[p][j] + tCkl[p][j] * tCl[j][i];
                Wc1[p][i] = Wc1[p][i] - tCkl[p][j] * tCl[j][i];
            }
            for (p = 0; p < n; p++) {
                cnumb = tCl[i][j] * tCl[p][j] + tr3 * tCl[p][i];
                Wc1[j][p] = Wc1[j][p] + cnumb;
                Wc1[i][p] = Wc1[i][p] - cnumb;
            }
            for (p = 0; p < n; p++)
                for (q = 0; q < n; q++) Wc2[p][q] = tCkl[p][j] * tCl[q][j];
            memset(Wc3, 0, sizeof(Mat));
            for (p = 0; p < n; p++) {
                Wc3[j][p] = tCl[p][i];
                Wc3[i][p] = -tCl[p][i];
            }
            cnumb = me_rxr_over_rij(Wc1, i, j, inv_tCkl, o->rm[i][j], TrCJ[i][j]);
            ctemp = me_rxr_ryr_over_rij(Wc2, Wc3, i, j, inv_tCkl, o->rm[i][j], TrCJ[i][j]);
            caux = -6 * (tr1 + tr2) * o->rm[i][j] + 4 * cnumb - 8 * ctemp;
            o->OO = o->OO + caux * g_q[i] * g_q[j] / (g_pmass[i + 1] * g_pmass[j + 1]);
        }
    o->OO = o->OO / 2;

    /* :1487-1597 mass-velocity */
    for (p = 0; p < n; p++) {
        ctemp = 0.0;
        for (q = 0; q < n; q++) ctemp = ctemp + tCk[q][p];
        for (q = 0; q < n; q++) Wc3[q][p] = ctemp;
    }
    tr1 = 0.0;
    for (p = 0; p < n; p++) tr1 = tr1 + Wc3[p][p];
    for (p = 0; p < n; p++) {
        ctemp = 0.0;
        for (i = 0; i < n; i++) ctemp = ctemp + tCk[p][i] * Wc3[i][p];
        Wc1[p][p] = ctemp;
        for (q = p + 1; q < n; q++) {
            ctemp = 0.0;
            for (j = 0; j < n; j++) ctemp = ctemp + tCk[q][j] * Wc3[j][p];
            Wc1[q][p] = ctemp;
            Wc1[p][q] = ctemp;
        }
    }
    for (p = 0; p < n; p++) {
        ctemp = 0.0;
        for (q = 0; q < n; q++) ctemp = ctemp + tCl[q][p];
        for (q = 0; q < n; q++) Wc3[q][p] = ctemp;
    }
    tr2 = 0.0;
    for (p = 0; p < n; p++) tr2 = tr2 + Wc3[p][p];
    for (p = 0; p < n; p++) {
        ctemp = 0.0;
        for (i = 0; i < n; i++) ctemp = ctemp + tCl[p][i] * Wc3[i][p];
        Wc2[p][p] = ctemp;
        for (q = p + 1; q < n; q++) {
            ctemp = 0.0;
            for (j = 0; j < n; j++) ctemp = ctemp + tCl[q][j] * Wc3[j][p];
            Wc2[q][p] = ctemp;
            Wc2[p][q] = ctemp;
        }
    }
    for (p = 0; p < n; p++) {
        Wc3[p][p] = tr1 * Wc2[p][p] + tr2 * Wc1[p][p];
        for (q = p + 1; q < n; q++) {
            Wc3[q][p] = tr1 * Wc2[q][p] + tr2 * Wc1[q][p];
            Wc3[p][q] = Wc3[q][p];
        }
    }
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) {
            ctemp = 0.0;
            for (j = 0; j < n; j++) ctemp = ctemp + inv_tCkl[q][j] * Wc1[j][p];
            Wc4[q][p] = ctemp;
        }
    tr4 = 0.0;
    for (p = 0; p < n; p++) tr4 = tr4 + Wc4[p][p];
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) {
            ctemp = 0.0;
            for (j = 0; j < n; j++) ctemp = ctemp + inv_tCkl[q][j] * Wc2[j][p];
            Wc5[q][p] = ctemp;
        }
    tr5 = 0.0;
    for (p = 0; p < n; p++) tr5 = tr5 + Wc5[p][p];
    cnumb = 0.0;
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) cnumb = cnumb + Wc4[p][q] * Wc5[q][p];
    caux = 0.0;
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) caux = caux + inv_tCkl[p][q] * Wc3[q][p];
    o->MV = 36 * Skl * (tr4 * tr5 + ((xreal)2 / 3) * cnumb - caux + tr1 * tr2) /
            (g_pmass[0] * g_pmass[0] * g_pmass[0]);
    for (i = 0; i < n; i++) {
        for (p = 0; p < n; p++) {
            Wc1[p][p] = tCk[p][i] * tCk[i][p];
            for (q = p + 1; q < n; q++) {
                Wc1[q][p] = tCk[q][i] * tCk[i][p];
                Wc1[p][q] = Wc1[q][p];
            }
        }
        tr1 = tCk[i][i];
        for (p = 0; p < n; p++) {
            Wc2[p][p] = tCl[p][i] * tCl[i][p];
            for (q = p + 1; q < n; q++) {
                Wc2[q][p] = tCl[q][i] * tCl[i][p];
                Wc2[p][q] = Wc2[q][p];
            }
        }
        tr2 = tCl[i][i];
        caux = 0.0;
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) caux = caux + inv_tCkl[p][q] * (tr1 * Wc2[q][p] + tr2 * Wc1[q][p]);
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) {
                ctemp = 0.0;
                for (j = 0; j < n; j++) ctemp = ctemp + inv_tCkl[q][j] * Wc1[j][p];
                Wc4[q][p] = ctemp;
            }
        tr4 = 0.0;
        for (p = 0; p < n; p++) tr4 = tr4 + Wc4[p][p];
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) {
                ctemp = 0.0;
                for (j = 0; j < n; j++) ctemp = ctemp + inv_tCkl[q][j] * Wc2[j][p];
                Wc5[q][p] = ctemp;
            }
        tr5 = 0.0;
        for (p = 0; p < n; p++) tr5 = tr5 + Wc5[p][p];
        cnumb = 0.0;
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) cnumb = cnumb + Wc4[p][q] * Wc5[q][p];
        o->MV = o->MV + 36 * Skl * (tr4 * tr5 + ((xreal)2 / 3) * cnumb - caux + tr1 * tr2) /
                            (g_pmass[i + 1] * g_pmass[i + 1] * g_pmass[i + 1]);
    }
    o->MV = -o->MV / 8;

    /* :1675-1712 first term of the Drachmanised mass-velocity */
    cnumb = 1 / (g_pmass[0] * g_pmass[0]);
    for (p = 0; p < n; p++) {
        Wc1[p][p] = cnumb + 1 / (g_pmass[p + 1] * g_pmass[p + 1]);
        for (q = p + 1; q < n; q++) {
            Wc1[p][q] = cnumb;
            Wc1[q][p] = cnumb;
        }
    }
    tr1 = 0.0;
    for (p = 0; p < n; p++) {
        for (q = 0; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + tCl[j][q] * Wc1[j][p];
            Wc2[q][p] = cnumb;
        }
        tr1 = tr1 + Wc2[p][p];
    }
    for (p = 0; p < n; p++)
        for (q = p; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + Wc2[q][j] * tCl[j][p];
            Wc3[q][p] = cnumb;
            Wc3[p][q] = cnumb;
        }
    tr2 = 0.0;
    for (p = 0; p < n; p++)
        for (j = 0; j < n; j++) tr2 = tr2 + inv_tCkl[j][p] * Wc3[j][p];
    o->drach_MV = Skl * g_curr_energy * 6.0 * (tr2 - tr1) / 4;
    /* :1714-1726 second term (Wc3, tr1 reused) */
    cnumb = 0.0;
    for (i = 0; i < n; i++)
        cnumb = cnumb + g_q0 * g_q[i] *
                            (4 * me_rxr_over_rij(Wc3, i, i, inv_tCkl, o->rm[i][i], TrCJ[i][i]) - 6 * tr1 * o->rm[i][i]);
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++)
            cnumb = cnumb + g_q[i] * g_q[j] *
                                (4 * me_rxr_over_rij(Wc3, i, j, inv_tCkl, o->rm[i][j], TrCJ[i][j]) -
                                 6 * tr1 * o->rm[i][j]);
    o->drach_MV = o->drach_MV - cnumb / 4;
    /* :1728-1787 third term */
    tr1 = 0.0;
    for (p = 0; p < n; p++) {
        cnumb = 0.0;
        for (q = 0; q < n; q++) cnumb = cnumb + tCk[q][p];
        for (q = 0; q < n; q++) Wc1[q][p] = cnumb;
        tr1 = tr1 + cnumb;
    }
    tr2 = 0.0;
    for (p = 0; p < n; p++) {
        cnumb = (g_pmass[0] + g_pmass[p + 1]) / (g_pmass[0] * g_pmass[0] * g_pmass[p + 1] * g_pmass[p + 1]);
        for (q = 0; q < n; q++) Wc2[q][p] = cnumb * tCl[q][p];
        tr2 = tr2 + Wc2[p][p];
    }
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + inv_tCkl[q][j] * tCk[j][p];
            Wc5[q][p] = cnumb;
        }
    tr3 = 0.0;
    for (p = 0; p < n; p++) {
        for (q = 0; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + Wc5[q][j] * Wc1[j][p];
            Wc3[q][p] = cnumb;
        }
        tr3 = tr3 + Wc3[p][p];
    }
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + inv_tCkl[q][j] * Wc2[j][p];
            Wc5[q][p] = cnumb;
        }
    tr4 = 0.0;
    for (p = 0; p < n; p++) {
        for (q = 0; q < n; q++) {
            cnumb = 0.0;
            for (j = 0; j < n; j++) cnumb = cnumb + Wc5[q][j] * tCl[j][p];
            Wc4[q][p] = cnumb;
        }
        tr4 = tr4 + Wc4[p][p];
    }
    tr5 = 0.0;
    for (p = 0; p < n; p++)
        for (j = 0; j < n; j++) tr5 = tr5 + Wc3[p][j] * Wc4[j][p];
    o->drach_MV = o->drach_MV + Skl * (36 * tr3 * tr4 + 24 * tr5 - 36 * tr1 * tr4 - 36 * tr2 * tr3 + 36 * tr1 * tr2) / 8;
    /* :1789-1848 fourth term */
    for (k = 0; k < n - 1; k++) {
        tr1 = tCk[k][k];
        for (p = 0; p <= k; p++)
            for (q = 0; q < n; q++) Wc2[q][p] = 0.0;
        tr2 = 0.0;
        for (p = k + 1; p < n; p++) {
            cnumb = (g_pmass[k + 1] + g_pmass[p + 1]) /
                    (g_pmass[k + 1] * g_pmass[k + 1] * g_pmass[p + 1] * g_pmass[p + 1]);
            for (q = 0; q < n; q++) Wc2[q][p] = cnumb * tCl[q][p];
            tr2 = tr2 + Wc2[p][p];
        }
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) Wc5[q][p] = tCk[q][k] * tCk[p][k];
        tr3 = 0.0;
        for (p = 0; p < n; p++) {
            for (q = 0; q < n; q++) {
                cnumb = 0.0;
                for (j = 0; j < n; j++) cnumb = cnumb + inv_tCkl[q][j] * Wc5[j][p];
                Wc3[q][p] = cnumb;
            }
            tr3 = tr3 + Wc3[p][p];
        }
        for (p = 0; p < n; p++)
            for (q = 0; q < n; q++) {
                cnumb = 0.0;
                for (j = 0; j < n; j++) cnumb = cnumb + inv_tCkl[q][j] * Wc2[j][p];
                Wc5[q][p] = cnumb;
            }
        tr4 = 0.0;
        for (p = 0; p < n; p++) {
            for (q = 0; q < n; q++) {
                cnumb = 0.0;
                for (j = 0; j < n; j++) cnumb = cnumb + Wc5[q][j] * tCl[j][p];
                Wc4[q][p] = cnumb;
            }
            tr4 = tr4 + Wc4[p][p];
        }
        tr5 = 0.0;
        for (p = 0; p < n; p++)
            for (j = 0; j < n; j++) tr5 = tr5 + Wc3[p][j] * Wc4[j][p];
        o->drach_MV =
            o->drach_MV + Skl * (36 * tr3 * tr4 + 24 * tr5 - 36 * tr1 * tr4 - 36 * tr2 * tr3 + 36 * tr1 * tr2) / 8;
    }

    /* :1850-1873 Darwin */
    Mass_For_Darwin[0] = g_pmass[0];
    for (i = 1; i <= n; i++) Mass_For_Darwin[i] = g_pmass[i];
    o->Darwin = 0.0;
    for (i = 0; i < n; i++)
        o->Darwin = o->Darwin + (1.0 / (Mass_For_Darwin[0] * Mass_For_Darwin[0]) +
                                 1.0 / (Mass_For_Darwin[i + 1] * Mass_For_Darwin[i + 1])) *
                                    g_q0 * g_q[i] * o->deltar[i][i];
    for (i = 0; i < n; i++)
        for (j = 0; j < n; j++)
            if (j != i)
                o->Darwin = o->Darwin + 1.0 / (Mass_For_Darwin[i + 1] * Mass_For_Darwin[i + 1]) * g_q[i] * g_q[j] *
                                            o->deltar[i][j];
    o->Darwin = -o->Darwin * PI_ / 2;

    /* :1875-1929 Drachmanised Darwin */
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) Wc1[p][q] = 1.0 / (g_pmass[0] * g_pmass[0]);
    for (i = 0; i < n; i++) Wc1[i][i] = Wc1[i][i] + 1.0 / (g_pmass[i + 1] * g_pmass[i + 1]);
    o->drach_Darwin = g_curr_energy * me_dxd(Wc1, inv_tCkl, tCl, Skl) / 4;
    for (i = 0; i < n; i++)
        o->drach_Darwin = o->drach_Darwin - g_q0 * g_q[i] *
                                                me_dxd_over_rij(Wc1, i, i, inv_tCkl, tCl, o->rm[i][i], TrCJ[i][i]) / 4;
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++)
            o->drach_Darwin = o->drach_Darwin - g_q[i] * g_q[j] *
                                                    me_dxd_over_rij(Wc1, i, j, inv_tCkl, tCl, o->rm[i][j], TrCJ[i][j]) /
                                                    4;
    for (p = 0; p < n; p++)
        for (q = 0; q < n; q++) {
            Wc1[p][q] = 1.0;
            Wc2[p][q] = 0.0;
        }
    for (j = 0; j < n; j++)
        Wc2[j][j] = Wc2[j][j] + (g_pmass[0] + g_pmass[j + 1]) /
                                    (g_pmass[0] * g_pmass[0] * g_pmass[j + 1] * g_pmass[j + 1]);
    o->drach_Darwin = o->drach_Darwin + me_dxd_dyd(Wc1, Wc2, inv_tCkl, tCk, tCl, Skl) / 8;
    for (i = 0; i < n; i++)
        for (j = i + 1; j < n; j++) {
            memset(Wc1, 0, sizeof(Mat));
            Wc1[i][i] = 1.0;
            memset(Wc2, 0, sizeof(Mat));
            Wc2[j][j] = 1.0;
            cnumb = (g_pmass[i + 1] + g_pmass[j + 1]) /
                    (g_pmass[i + 1] * g_pmass[i + 1] * g_pmass[j + 1] * g_pmass[j + 1]);
            o->drach_Darwin = o->drach_Darwin + cnumb * me_dxd_dyd(Wc1, Wc2, inv_tCkl, tCk, tCl, Skl) / 8;
        }

    /* :1931-1960 correlation functions and particle densities */
    if (ncf > 0) {
        ctemp = Skl / (PI_ * XSQRTPI);
        for (k = 0; k < ncf; k++) {
            p = 0;
            rnumb = -CFGrid[k] * CFGrid[k];
            for (i = 0; i < n; i++)
                for (j = i; j < n; j++) {
                    CFkl[p + (size_t)k * np] = ctemp * XCEXP(rnumb / TrCJ[j][i]) / (XCSQRT(TrCJ[j][i]) * TrCJ[j][i]);
                    p++;
                }
        }
    }
    if (ndens > 0) {
        ctemp = Skl / (PI_ * XSQRTPI);
        for (k = 0; k < ndens; k++) {
            rnumb = -DensGrid[k] * DensGrid[k];
            for (i = 0; i <= n; i++) {
                caux = 0.0;
                for (p = 0; p < n; p++) {
                    caux = caux + g_bvc[p][i] * g_bvc[p][i] * inv_tCkl[p][p];
                    for (q = p + 1; q < n; q++) caux = caux + 2 * g_bvc[q][i] * g_bvc[p][i] * inv_tCkl[q][p];
                }
                Denskl[i + (size_t)k * (n + 1)] = ctemp * XCEXP(rnumb / caux) / (XCSQRT(caux) * caux);
            }
        }
    }
}

static void load_perm_cm(const int *Pcm, int P[NN][NN])
{
    for (int i = 0; i < g_n; i++)
        for (int j = 0; j < g_n; j++) P[i][j] = Pcm[i + j * g_n];
}

/* One MatrixElementsForExpcVals call packed into the MEkl order of
 * src/workproc.f90:8045-8060 / 8180-8215 (6 np + 9 complex values). */
static void expc_packed(const double *Paramk, const double *Paraml, const int *Pbra_cm, const int *Pket_cm,
                        xcplx *vals, int ncf, const double *cf_grid, xcplx *cf, int ndens, const double *dens_grid,
                        xcplx *dens)
{
    int Pb[NN][NN], Pk[NN][NN];
    ExpcTerm o;
    load_perm_cm(Pbra_cm, Pb);
    load_perm_cm(Pket_cm, Pk);
    expc_matrix_elements(Paramk, Paraml, Pb, Pk, &o, ncf, cf_grid, cf, ndens, dens_grid, dens);
    const int n = g_n;
    int c = 0;
    xcplx(*blocks[6])[NN] = {o.rm2, o.rm, o.r, o.r2, o.deltar, o.drach_deltar};
    for (int b = 0; b < 6; b++)
        for (int a = 0; a < n; a++)
            for (int bb = a; bb < n; bb++) vals[c++] = blocks[b][bb][a];
    vals[c++] = o.H;
    vals[c++] = o.S;
    vals[c++] = o.T;
    vals[c++] = o.V;
    vals[c++] = o.MV;
    vals[c++] = o.drach_MV;
    vals[c++] = o.Darwin;
    vals[c++] = o.drach_Darwin;
    vals[c++] = o.OO;
}

#ifndef ORC_LONG
/* A single MatrixElementsForExpcVals call with Glob_CurrEnergy = curr_energy. */
void orc_expc_matrix_elements(const double *Paramk, const double *Paraml, const int *Pbra_cm, const int *Pket_cm,
                              double curr_energy, cplx *vals, int ncf, const double *cf_grid, cplx *cf, int ndens,
                              const double *dens_grid, cplx *dens)
{
    g_curr_energy = curr_energy;
    expc_packed(Paramk, Paraml, Pbra_cm, Pket_cm, vals, ncf, cf_grid, cf, ndens, dens_grid, dens);
}

#endif

/*
 * The accumulation loop of ExpectationValuesG, src/workproc.f90:8159-8351,
 * for one rank (NumOfProcs = 1): pairs i = 1..K, j = 1..i, every term t of
 * the list (bra matrix, ket matrix, coefficients coef1[t], coef2[t]: the
 * weight is factor*coef1*coef2 as written there), values accumulated in the
 * reference's order.  SymmAdaptMethod 1 is the list (identity, Y^+Y_t,
 * YHYCoeff_t, 1) with err_mult 2; SymmAdaptMethod 2 the list
 * (Y_k, Y_kk, YCoeff_k, YCoeff_kk) over k outer, kk inner, with err_mult 3.
 * OpenMP threads take contiguous row ranges and their partial sums are
 * added in thread order, so the result depends only on the thread count.
 * Outputs: sums (6np+9), errs (6np+9, already times epsilon), cf (np x ncf),
 * dens ((n+1) x ndens).
 */
void ORC_NAME(orc_expectation_values)(const double *params, int K, const double *c_ri, const double *diagS, int nterms,
                            const int *pbra_cm, const int *pket_cm, const double *coef1, const double *coef2,
                            int err_mult,
                            double curr_energy, int ncf, const double *cf_grid, int ndens, const double *dens_grid,
                            double *sums, double *errs, double *cf, double *dens)
{
    const int n = g_n, np = g_np, npt = g_npt;
    const int nv = 6 * np + 9;
    const int ngrid = ncf * np + ndens * (n + 1);
    g_curr_energy = curr_energy;
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    xreal *part = calloc((size_t)nth * (2 * nv + ngrid), sizeof(xreal));
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        xreal *ps = part + (size_t)tid * (2 * nv + ngrid);
        xreal *pe = ps + nv, *pg = pe + nv;
        xcplx vals[6 * NNP + 9];
        xcplx *cfkl = ncf ? malloc(sizeof(xcplx) * (size_t)np * ncf) : NULL;
        xcplx *dkl = ndens ? malloc(sizeof(xcplx) * (size_t)(n + 1) * ndens) : NULL;
        /* rows split so that each thread gets about the same number of pairs */
        const xreal tot = 0.5 * (xreal)K * (K + 1);
        const int i0 = (int)ceil(XSQRT(2.0 * tot * tid / nth));
        const int i1 = (tid == nth - 1) ? K : (int)ceil(XSQRT(2.0 * tot * (tid + 1) / nth));
        for (int i = i0 + 1; i <= i1 && i <= K; i++) {
            if (i < 1) continue;
            for (int j = 1; j <= i; j++) {
                const xreal ReCi = c_ri[2 * (i - 1)], ImCi = c_ri[2 * (i - 1) + 1];
                const xreal ReCj = c_ri[2 * (j - 1)], ImCj = c_ri[2 * (j - 1) + 1];
                xreal factor;
                if (i == j)
                    factor = 1 / XSQRT(diagS[i - 1] * diagS[i - 1]);
                else
                    factor = 2 / XSQRT(diagS[i - 1] * diagS[j - 1]);
                for (int t = 0; t < nterms; t++) {
                    expc_packed(params + (size_t)(i - 1) * npt, params + (size_t)(j - 1) * npt,
                                pbra_cm + (size_t)t * n * n, pket_cm + (size_t)t * n * n, vals, ncf, cf_grid, cfkl,
                                ndens, dens_grid, dkl);
                    for (int a = 0; a < nv; a++) {
                        const xreal ReOij = XCREAL(vals[a]), ImOij = XCIMAG(vals[a]);
                        const xreal beta = (ReCi * ReCj + ImCi * ImCj) * ReOij + (ImCi * ReCj - ReCi * ImCj) * ImOij;
                        const xreal mu = XFABS(ReCi * (ReCj * ReOij - ImCj * ImOij)) +
                                          XFABS(ReCj * (ReCi * ReOij + ImCi * ImOij)) +
                                          XFABS(ImCi * (ImCj * ReOij + ReCj * ImOij)) +
                                          XFABS(ImCj * (ImCi * ReOij - ReCi * ImOij));
                        ps[a] = ps[a] + factor * coef1[t] * coef2[t] * beta;
                        pe[a] = pe[a] + XFABS(factor * coef1[t] * coef2[t] * (mu + err_mult * XFABS(beta)));
                    }
                    int g = 0;
                    for (int a = 0; a < ncf * np; a++, g++) {
                        const xreal ReOij = XCREAL(cfkl[a]), ImOij = XCIMAG(cfkl[a]);
                        const xreal beta = (ReCi * ReCj + ImCi * ImCj) * ReOij + (ImCi * ReCj - ReCi * ImCj) * ImOij;
                        pg[g] = pg[g] + factor * coef1[t] * coef2[t] * beta;
                    }
                    for (int a = 0; a < ndens * (n + 1); a++, g++) {
                        const xreal ReOij = XCREAL(dkl[a]), ImOij = XCIMAG(dkl[a]);
                        const xreal beta = (ReCi * ReCj + ImCi * ImCj) * ReOij + (ImCi * ReCj - ReCi * ImCj) * ImOij;
                        pg[g] = pg[g] + factor * coef1[t] * coef2[t] * beta;
                    }
                }
            }
        }
        free(cfkl);
        free(dkl);
    }
    /* thread partial sums added in thread order (into thread 0's slots) */
    for (int t = 1; t < nth; t++) {
        const xreal *ps = part + (size_t)t * (2 * nv + ngrid);
        for (int a = 0; a < 2 * nv + ngrid; a++) part[a] = part[a] + ps[a];
    }
    for (int a = 0; a < nv; a++) {
        sums[a] = (double)part[a];
        errs[a] = (double)(part[nv + a] * DBL_EPSILON);
    }
    for (int g = 0; g < ncf * np; g++) cf[g] = (double)part[2 * nv + g];
    for (int g = 0; g < ndens * (n + 1); g++) dens[g] = (double)part[2 * nv + ncf * np + g];
    free(part);
}
