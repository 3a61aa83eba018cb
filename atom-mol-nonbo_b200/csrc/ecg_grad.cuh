// ecg_grad.cuh -- derivatives of one ECG pair term.
//
// term_grad_plain: the derivative vectors Dk, Dl of src/matelem.f90:306-748
//   (dH/dvechL, dH/dvechB, dS/dvechL, dS/dvechB of the bra and/or ket), in the
//   reference's order, for the plain drop-in that materialises Glob_D.
//
// term_adjoint: the same derivatives already contracted into the form the
//   energy gradient needs.  For one term with energy E fixed,
//       dH/dvechL - E dS/dvechL  (entry (j,i), j >= i)
//            = a * delta_ij / L_ii - 2 (Z L)_ji
//       dH/dvechB - E dS/dvechB  (entry (i,j), weight 1 on the diagonal,
//                                 2 off it)
//            = +i Z_ij (bra)   or   -i Z_ij (ket),
//   with a = (3/2)(H - E S) and one complex symmetric matrix Z per side:
//       Z_k = a C^-1 - C^-1 [6 S tCl M tCl + S/sqrt(pi) Q] C^-1
//       Z_l = P ( a C^-1 - C^-1 [6 S Ck M Ck + S/sqrt(pi) Q] C^-1 ) P'
//   where Q(i,i) = w_ii + sum_{j!=i} w_ij, Q(i,j) = -w_ij collects the
//   Coulomb weights w_ij = cnumb of src/matelem.f90:677-681.  This follows
//   from the reference's formulas: every Coulomb matrix tQ of
//   src/matelem.f90:609-631 is the rank-one C^-1 (e_i-e_j)(e_i-e_j)' C^-1,
//   so their weighted sum is C^-1 Q C^-1; and dS, dT, dV share the factors
//   C^-1, F = C^-1 tCl M tCl C^-1 and G = P C^-1 Ck M Ck C^-1 P'.
#pragma once
#include "ecg_math.cuh"

namespace ecg {

// ---------------------------------------------------------------------------
// Plain transcription (src/matelem.f90:306-748).  Lk, Ll are lower
// triangular (upper entries zero), P the permutation matrix of this term.
// Dk, Dl receive 4*NP complex values each (H-L, H-B, S-L, S-B blocks).
// ---------------------------------------------------------------------------
template <int N, bool GK, bool GL>
__device__ __forceinline__ void term_grad_plain(const double (&Lk)[N][N], const double (&Ll)[N][N],
                                                const double (&P)[N][N], const cd (&Ck)[N][N],
                                                const cd (&tCl)[N][N], const TermEnergy<N>& te,
                                                const SysParams& sp, cd* Dk, cd* Dl)
{
    constexpr int NP = Sym<N>::NP;
    const cd S = te.S;
    const cd tos = cdiv(te.T, S);
    const cd vos = cdiv(te.V, S);
    cd Wc1[N][N];

    // ---- dS (matelem.f90:306-423) ----
    if (GK) {
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = j; k < N; k++) s = rfma(Lk[k][j], te.inv[i][k], s);
                Wc1[i][j] = s;
            }
        double iL[N][N];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) iL[j][i] = Lk[j][i];
#pragma unroll
        for (int i = 0; i < N; i++) {
            iL[i][i] = 1.0 / iL[i][i];
#pragma unroll
            for (int j = i + 1; j < N; j++) {
                double r = 0.0;
#pragma unroll
                for (int k = i; k <= j - 1; k++) r = fma(-iL[j][k], iL[k][i], r);
                iL[j][i] = r / iL[j][j];
            }
        }
        const cd ct = 1.5 * S;
        const cd cb = cmul(S, mk(0.0, 1.5));
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                const int x = vech_index(N, i, j);
                const double d = (i == j) ? iL[i][i] : 0.0;
                Dk[2 * NP + x] = cmul(mk(d - 2.0 * Wc1[j][i].x, -2.0 * Wc1[j][i].y), ct);
                Dk[3 * NP + x] = (i == j) ? cmul(te.inv[i][i], cb) : cmul(te.inv[j][i], 2.0 * cb);
            }
    }
    cd itt[N][N];  // inv_ttCkl = P C^-1 P'
    if (GL) {
        cd W[N][N];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[i][k], te.inv[k][j], s);
                W[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[j][k], W[i][k], s);
                itt[i][j] = s;
                itt[j][i] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(Ll[k][j], itt[i][k], s);
                Wc1[i][j] = s;
            }
        double iL[N][N];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) iL[j][i] = Ll[j][i];
#pragma unroll
        for (int i = 0; i < N; i++) {
            iL[i][i] = 1.0 / iL[i][i];
#pragma unroll
            for (int j = i + 1; j < N; j++) {
                double r = 0.0;
#pragma unroll
                for (int k = i; k <= j - 1; k++) r = fma(-iL[j][k], iL[k][i], r);
                iL[j][i] = r / iL[j][j];
            }
        }
        const cd ct = 1.5 * S;
        const cd cb = cmul(S, mk(0.0, -1.5));
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                const int x = vech_index(N, i, j);
                const double d = (i == j) ? iL[i][i] : 0.0;
                Dl[2 * NP + x] = cmul(mk(d - 2.0 * Wc1[j][i].x, -2.0 * Wc1[j][i].y), ct);
                Dl[3 * NP + x] = (i == j) ? cmul(itt[i][i], cb) : cmul(itt[j][i], 2.0 * cb);
            }
    }
    // ---- dT (matelem.f90:427-598) ----
    // X = C^-1 (Y M Y) C^-1 with Y = Ck (ket side, then G = P X P') or
    // Y = tCl (bra side, F = X).
    auto sandwich = [&](const cd (&Y)[N][N], cd (&X)[N][N]) {
        cd A[N][N], B[N][N];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(sp.M[k * NMAX + j], Y[i][k], s);
                A[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = cfma(A[i][k], Y[k][j], s);
                B[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = cfma(te.inv[i][k], B[k][j], s);
                A[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = cfma(A[i][k], te.inv[k][j], s);
                X[i][j] = s;
                X[j][i] = s;
            }
    };
    if (GL) {
        cd X[N][N], G[N][N], W[N][N];
        sandwich(Ck, X);
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[i][k], X[k][j], s);
                W[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[j][k], W[i][k], s);
                G[i][j] = s;
                G[j][i] = s;
            }
        const cd c12 = 12.0 * S;
        const cd c6 = cmul(S, mk(0.0, 6.0));
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                const int x = vech_index(N, i, j);
                cd gl = mk(0.0, 0.0);
#pragma unroll
                for (int k = i; k < N; k++) gl = rfma(Ll[k][i], G[j][k], gl);
                Dl[x] = cfma(tos, Dl[2 * NP + x], cmul(c12, gl));
                Dl[NP + x] = cfma(tos, Dl[3 * NP + x], (i == j) ? cmul(c6, G[i][i]) : cmul(2.0 * c6, G[j][i]));
            }
    }
    if (GK) {
        cd F[N][N];
        sandwich(tCl, F);
        const cd c12 = 12.0 * S;
        const cd c6 = cmul(S, mk(0.0, -6.0));
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                const int x = vech_index(N, i, j);
                cd fl = mk(0.0, 0.0);
#pragma unroll
                for (int k = i; k < N; k++) fl = rfma(Lk[k][i], F[j][k], fl);
                Dk[x] = cfma(tos, Dk[2 * NP + x], cmul(c12, fl));
                Dk[NP + x] = cfma(tos, Dk[3 * NP + x], (i == j) ? cmul(c6, F[i][i]) : cmul(2.0 * c6, F[j][i]));
            }
    }
    // ---- dV (matelem.f90:603-734) ----
    cd Qw[N][N];
    coulomb_weights<N>(te, sp, Qw);
    cd WLk[NP], WBk[NP], WLl[NP], WBl[NP];
#pragma unroll
    for (int x = 0; x < NP; x++) {
        WLk[x] = mk(0.0, 0.0); WBk[x] = mk(0.0, 0.0);
        WLl[x] = mk(0.0, 0.0); WBl[x] = mk(0.0, 0.0);
    }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j <= i; j++) {
            // tQ = C^-1 J_ij C^-1 = u u' with u = C^-1 (e_i - e_j) (u = C^-1 e_i if i == j)
            cd u[N];
#pragma unroll
            for (int k = 0; k < N; k++) u[k] = (i == j) ? te.inv[k][i] : te.inv[k][i] - te.inv[k][j];
            const cd cn = Qw[i][j];
            if (GK) {
#pragma unroll
                for (int k = 0; k < N; k++)
#pragma unroll
                    for (int kk = 0; kk <= k; kk++) {
                        // (tQ Lk)(k,kk) = u_k * sum_{m>=kk} u_m Lk(m,kk)
                        cd s = mk(0.0, 0.0);
#pragma unroll
                        for (int m = kk; m < N; m++) s = rfma(Lk[m][kk], u[m], s);
                        const cd tl = cmul(u[k], s);
                        const int x = vech_index(N, kk, k);
                        WLk[x] = cfma(cn, tl, WLk[x]);
                        const cd tq = cmul(u[k], u[kk]);
                        WBk[x] = cfma((k == kk) ? cn : 2.0 * cn, tq, WBk[x]);
                    }
            }
            if (GL) {
                cd pu[N];  // P u, so that ttQ = (P u)(P u)'
#pragma unroll
                for (int k = 0; k < N; k++) {
                    cd s = mk(0.0, 0.0);
#pragma unroll
                    for (int m = 0; m < N; m++) s = rfma(P[k][m], u[m], s);
                    pu[k] = s;
                }
#pragma unroll
                for (int k = 0; k < N; k++)
#pragma unroll
                    for (int kk = 0; kk <= k; kk++) {
                        cd s = mk(0.0, 0.0);
#pragma unroll
                        for (int m = kk; m < N; m++) s = rfma(Ll[m][kk], pu[m], s);
                        const cd tl = cmul(pu[k], s);
                        const int x = vech_index(N, kk, k);
                        WLl[x] = cfma(cn, tl, WLl[x]);
                        const cd tq = cmul(pu[k], pu[kk]);
                        WBl[x] = cfma((k == kk) ? cn : 2.0 * cn, tq, WBl[x]);
                    }
            }
        }
    const cd c2 = TWO_OVER_SQRTPI * S;
    const cd ci = cmul(mk(0.0, ONE_OVER_SQRTPI), S);
    if (GK)
#pragma unroll
        for (int x = 0; x < NP; x++) {
            Dk[x] = cfma(c2, WLk[x], cfma(vos, Dk[2 * NP + x], Dk[x]));
            Dk[NP + x] = cfms(ci, WBk[x], cfma(vos, Dk[3 * NP + x], Dk[NP + x]));
        }
    if (GL)
#pragma unroll
        for (int x = 0; x < NP; x++) {
            Dl[x] = cfma(c2, WLl[x], cfma(vos, Dl[2 * NP + x], Dl[x]));
            Dl[NP + x] = cfma(ci, WBl[x], cfma(vos, Dl[3 * NP + x], Dl[NP + x]));
        }
}

// ---------------------------------------------------------------------------
// Adjoint form: accumulate coef * Z_k, coef * Z_l (unpermuted) and coef * a.
// Zk, Zl are stored as packed lower triangles (vech order, NP entries).
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ void sym_sandwich(const cd (&inv)[N][N], const cd (&R)[N][N], cd (&X)[N][N])
{
    cd A[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = cfma(inv[i][k], R[k][j], s);
            A[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = cfma(A[i][k], inv[k][j], s);
            X[i][j] = s;
            X[j][i] = s;
        }
}

// R = 6 S (Y M Y) + S/sqrt(pi) Q for symmetric complex Y.
template <int N>
__device__ __forceinline__ void adj_middle(const cd (&Y)[N][N], const cd (&Qs)[N][N], cd s6,
                                           const SysParams& sp, cd (&R)[N][N])
{
    cd A[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = rfma(sp.M[k * NMAX + j], Y[i][k], s);
            A[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            cd s = mk(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < N; k++) s = cfma(A[i][k], Y[k][j], s);
            s = cfma(s6, s, Qs[i][j]);
            R[i][j] = s;
            R[j][i] = s;
        }
}

template <int N, bool KET>
__device__ __forceinline__ void term_adjoint(const double (&P)[N][N], const cd (&Ck)[N][N], const cd (&tCl)[N][N],
                                             const TermEnergy<N>& te, const SysParams& sp, double E, double coef,
                                             cd (&Zk)[Sym<N>::NP], cd (&Zl)[Sym<N>::NP], cd& a_acc)
{
    const cd S = te.S;
    const cd H = te.T + te.V;
    const cd a = 1.5 * (H - E * S);
    a_acc = rfma(coef, a, a_acc);
    // Qs = S/sqrt(pi) * Q
    cd Qw[N][N], Qs[N][N];
    coulomb_weights<N>(te, sp, Qw);
    const cd sq = ONE_OVER_SQRTPI * S;
#pragma unroll
    for (int i = 0; i < N; i++) {
        cd d = Qw[i][i];
#pragma unroll
        for (int j = 0; j < N; j++)
            if (j != i) d = d + Qw[i][j];
        Qs[i][i] = cmul(sq, d);
#pragma unroll
        for (int j = i + 1; j < N; j++) {
            Qs[i][j] = -cmul(sq, Qw[i][j]);
            Qs[j][i] = Qs[i][j];
        }
    }
    const cd s6 = 6.0 * S;
    cd R[N][N], X[N][N];
    adj_middle<N>(tCl, Qs, s6, sp, R);
    sym_sandwich<N>(te.inv, R, X);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = i; j < N; j++) {
            const int x = vech_index(N, i, j);
            Zk[x] = rfma(coef, cfms(mk(1.0, 0.0), X[j][i], cmul(a, te.inv[j][i])), Zk[x]);
        }
    if (KET) {
        adj_middle<N>(Ck, Qs, s6, sp, R);
        sym_sandwich<N>(te.inv, R, X);
        // Zt = a C^-1 - X, then Zl += coef * P Zt P'
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                const cd z = cfms(mk(1.0, 0.0), X[j][i], cmul(a, te.inv[j][i]));
                X[i][j] = z;
                X[j][i] = z;
            }
        cd W[N][N];
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = 0; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[i][k], X[k][j], s);
                W[i][j] = s;
            }
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int j = i; j < N; j++) {
                cd s = mk(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < N; k++) s = rfma(P[j][k], W[i][k], s);
                const int x = vech_index(N, i, j);
                Zl[x] = rfma(coef, s, Zl[x]);
            }
    }
}

}  // namespace ecg
