/* Golbal.h -- drop-in for the reference's include/Golbal.h: the test-case
 * enumeration and the file-static settings of the calling translation unit.
 * Names, order, types and defaults are those of the reference, so that
 * src/RP_FVM.c compiles and behaves unchanged. */
#ifndef GLOBAL_H
#define GLOBAL_H

#include <stdbool.h>

/* include/Golbal.h:8-30, same enumerators in the same order (values 0..20). */
typedef enum {
    TEST_PRECISION,
    TEST_1D_SHOCKTUBE,
    TEST_1D_CONTACTWAVE,
    TEST_1D_SHOCKIMPACT,
    TEST_1D_IMPACTWALL,
    TEST_1D_DOUBLERARE,
    TEST_1D_NOHPROBLEM,
    TEST_2D_SHOCKTUBE_CASE1,
    TEST_2D_SHOCKTUBE_CASE2,
    TEST_2D_SHOCKTUBE_CASE3,
    TEST_2D_SHOCKTUBE_CASE4,
    TEST_2D_SHOCKTUBE_CASE5,
    TEST_TAYLOR_GREEN_VORTEX,
    TEST_GAUSSIAN_PULSE,
    TEST_KELVIN_HELMHOLTZ,
    TEST_RAYLEIGH_TAYLOR,
    TEST_DOUBLE_MACH_REFLECTION,
    TEST_BLAST_WAVE,
    TEST_NOH_PROBLEM,
    TEST_OddEven_Decoupling,
    TEST_BACKWARD_STEP
} TestCase2D;

/* include/Golbal.h:33-70: per-translation-unit settings and their defaults. */
const int var = 4;
static bool Control_Out = false;
const int Block = 2;
static double Time = 0;
static int Ite = 0;
static int GhostCell = 4;
static double CFL = 0.5;
static int Recon_Accur = 5;
static bool Characteriz = false;
static bool Source;
static double Gravity;
static int Control_Compution;
static int Control_output;
static double M_gamma;

#endif
