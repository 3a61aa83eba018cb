/*
 * ecg_oracle.h -- declarations shared by the translation units of the CPU
 * oracle (test infrastructure only; see the header of ecg_oracle.c).
 */
#pragma once
#include <complex.h>

#define NN 5                  /* Glob_MaxAllowedNumOfPseudoParticles */
#define NNP (NN * (NN + 1) / 2)
#define TMAX 720              /* 6! terms is the largest symmetric group here */

typedef double complex cplx;

static const double SQRTPI = 1.77245385090551602729816748334115;

/* module globals set by orc_set_system (ecg_oracle.c) */
extern int g_n, g_np, g_npt, g_T;
extern double g_mass[NN][NN];      /* Glob_MassMatrix(i,j) -> g_mass[i][j] */
extern double g_q0, g_q[NN];       /* Glob_PseudoCharge0, Glob_PseudoCharge */
extern double g_2r3n2;             /* Glob_2raised3n2 = 2^(3n/2) */
