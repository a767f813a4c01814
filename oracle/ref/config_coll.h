/*
 * config_coll.h -- build configuration for compiling the reference's
 * collocated_AB3 sources into oracle/_ref/ (see config_stag.h for the mechanism).
 * Re-declares the interface of collocated_AB3/config.h (struct main_params member
 * order as in collocated_AB3/config.h:39-56) with size and options from -D REF_*.
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef TCREF_CONFIG_COLL_H
#define TCREF_CONFIG_COLL_H
#define CONFIG_H

#ifndef REF_DOUBLE
#define REF_DOUBLE 1
#endif
#ifndef REF_GENERAL_WRAP
#define REF_GENERAL_WRAP 0
#endif
#ifndef REF_GALERKIN
#define REF_GALERKIN 1
#endif
#define USE_DOUBLE_PRECISION REF_DOUBLE
#if USE_DOUBLE_PRECISION
#define real double
#else
#define real float
#endif

#define NORMALIZE_PRESSURE_AFTER_EACH_SOLVE
#define RE_TAU 395
#define ENABLE_TURB_VISC REF_GALERKIN
#define VISC_TERM_GALERKIN REF_GALERKIN

#if REF_GENERAL_WRAP
#include "index_wrap.h" /* NX, NY of any size (sizes that are not powers of two) */
#else
#define NX REF_NX
#define NY REF_NY
#endif
#define NZ_MAX REF_NZMAX

#define BLK_1D 256
#define BLK_X 8
#define BLK_Y 8
#define BLK_Z 4

struct main_params {
    int EnableTurbVisc;
    real visc;
    real sour_dpdx;
    real inv_length_scale;
    real xmin, ymin;
    real hx, hy, inv_hx, inv_hy, area;
    int NZ, N3D;
    int StabType;
    int FDmode;
};
#endif
