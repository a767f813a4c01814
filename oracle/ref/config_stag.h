/*
 * config_stag.h -- build configuration for compiling the reference's staggered
 * sources (staggered/*.cpp) into oracle/_ref/.  Force-included (-include) ahead of
 * the sources, it defines CONFIG_H so the reference's own staggered/config.h is
 * skipped, and re-declares that header's interface (the `real` type, the
 * compile-time switches, struct main_params, struct t_cmdline_params) with the
 * mesh size and scheme taken from -D REF_* flags.  The member order of
 * main_params must equal staggered/config.h:47-73 because the reference code
 * copies it between host and device images.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef TCREF_CONFIG_STAG_H
#define TCREF_CONFIG_STAG_H
#define CONFIG_H

#ifndef REF_DOUBLE
#define REF_DOUBLE 1
#endif
#ifndef REF_GENERAL_WRAP
#define REF_GENERAL_WRAP 0
#endif
#ifndef REF_TURB
#define REF_TURB 0
#endif
#ifndef REF_VISC_NAIVE
#define REF_VISC_NAIVE REF_TURB
#endif

#define USE_DOUBLE_PRECISION REF_DOUBLE
#if USE_DOUBLE_PRECISION
#define real double
#else
#define real float
#endif

#define NORMALIZE_PRESSURE_AFTER_EACH_SOLVE
#define ENABLE_TURB_VISC REF_TURB

enum struct tViscApproximation { CROSS, NAIVE, GALERKIN };
#define VISC_APPR_TYPE (REF_VISC_NAIVE ? tViscApproximation::NAIVE : tViscApproximation::CROSS)

#define CONV_HW 0
#define CONV_VV 1
#define CONV_APPR_TYPE REF_CONV

#if REF_GENERAL_WRAP
#include "index_wrap.h" /* NX, NY of any size (sizes that are not powers of two) */
#else
#define NX REF_NX
#define NY REF_NY
#endif
#define NXY (NX * NY)
#define NZ_MAX REF_NZMAX

#define BLK_1D 256
#define BLK_X 8
#define BLK_Y 8
#define BLK_Z 4

struct main_params {
    real visc;
    real sour_dpdx;
    real inv_length_scale;
    real xmin, ymin;
    real hx, hy, inv_hx, inv_hy, area;
    int NZ, N3D;
    real ZZ[NZ_MAX + 1];
    real DZ[NZ_MAX];
#if (CONV_APPR_TYPE == CONV_HW)
    real MAT_A[NZ_MAX];
#endif
#if (CONV_APPR_TYPE == CONV_VV)
    real DZW[NZ_MAX];
    real GC1[NZ_MAX];
    real GC2[NZ_MAX];
    real GCZ[NZ_MAX];
    real MAT_A[NZ_MAX * 3], MAT_D[6];
    real KERG[NZ_MAX], KERG_norm2;
#endif
};

struct t_cmdline_params {
    int DeviceID = 0;
    int NZ = NZ_MAX;
    double TimeMax = 100.;
    double TimeStartAveraging = 0.;
    int TimeStepsMax = 0x7FFFFFFF;
    double tau = 1e-3;
    double CFLmin = 0.05;
    double CFLmax = 0.5;
    int SProgress = 200;
    int FProgress = 1000000;
    int PProgress = 100000;
};
int ReadCmdlineParams(int argc, char** argv, int DeviceCount, t_cmdline_params& PM);
#endif
