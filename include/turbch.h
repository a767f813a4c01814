/*
 * turbch.h -- C ABI of turbchannel_b200, the B200 (sm_100a) implementation of the
 * per-time-step path of TurbChannel's channel-flow solvers.
 *
 * Every entry point returns 0 on success and a negative TC_E* code on failure;
 * tc_last_error() then holds a message (per host thread).  Plain pointers and
 * sizes only.  One handle = one solver object = one CUDA device + one stream;
 * handles are independent (the reference keeps a single global object per
 * process, staggered/func_cuda.cpp:41).
 *
 * Field layout at this boundary is the reference's: velocity AoS (u,v,w) per
 * cell, pressure one value per cell, linear index in = ix + NX*(iy + NY*iz),
 * x (streamwise) fastest, wall-normal z slowest, and four ring levels per field
 * (staggered/data_global_inc.h:4-9, :35-38).  Host buffers are always double.
 * Inside the library fields are stored structure-of-arrays in the precision
 * selected by tc_params.precision.
 */
#ifndef TURBCH_H
#define TURBCH_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ---- */
#define TC_OK 0
#define TC_E_ARG (-1)     /* invalid argument / unsupported configuration   */
#define TC_E_CUDA (-2)    /* CUDA runtime error                              */
#define TC_E_NOMEM (-3)   /* device allocation failed                        */
#define TC_E_NUMERIC (-4) /* singular pivot / non-finite value               */
#define TC_E_STATE (-5)   /* call out of order                               */

/* ---- schemes, options ---- */
#define TC_SCHEME_HW2 0    /* staggered Harlow-Welch, 2nd order      */
#define TC_SCHEME_VV4 1    /* staggered Verstappen-Veldman, 4th order */
#define TC_SCHEME_COLLOC 2 /* collocated, 2nd order (collocated_AB3)  */

#define TC_VISC_CROSS 0    /* 7-point Laplacian, constant viscosity   */
#define TC_VISC_NAIVE 1    /* staggered stress divergence with nu_t   */
#define TC_VISC_GALERKIN 2 /* collocated 27-point Galerkin with nu_t  */

#define TC_FP64 0  /* everything in double                                       */
#define TC_MIXED 1 /* float storage/stencils/FFTs; double for the low-wavenumber
                      banded solves (incl. the pinned mean mode), the flow-rate
                      forcing and every global reduction                         */

#define TC_TURB_NONE 0
#define TC_TURB_SMAGORINSKY 1 /* Smagorinsky-van Driest, staggered/func_global.h:875-890 */
#define TC_TURB_MLP 2         /* learned closure (tc_set_turb_model)                       */

/* Mirrors struct main_params (staggered/config.h:47-73, collocated_AB3/config.h:
 * 39-56) plus the reference's compile-time switches (config.h:5-43) as runtime
 * values.  NZ: staggered = number of cells (NZ+1 z-faces), collocated = number of
 * nodes (walls included), as in the reference. */
typedef struct tc_params {
    int scheme;     /* TC_SCHEME_*                                   */
    int precision;  /* TC_FP64 / TC_MIXED                            */
    int visc_type;  /* TC_VISC_*                                     */
    int turb_model; /* TC_TURB_*                                     */
    int NX, NY, NZ; /* NX, NY: 2^a 3^b, even                         */
    int stab_type;  /* collocated StabType: 0 or 1                   */
    int fd_mode;    /* collocated FDmode: 0 or 1                     */
    int device;     /* CUDA device ordinal (-d/--device)              */
    double visc, sour_dpdx, inv_length_scale;
    double xmin, ymin;
    double hx, hy, area;
    int low_modes; /* TC_MIXED: modes with kx < low_modes and min(ky, NY-ky) < low_modes
                      are solved in double (0 selects the default, 4)               */
} tc_params;

typedef struct tc_handle tc_handle;

const char* tc_last_error(void);
const char* tc_version(void);

/* Create a solver.  zz: z-coordinates of the NZ+1 cell faces (staggered) or of the
 * NZ nodes (collocated); replaces data::alloc_all + InitDerivativeMeshData +
 * InitFourier + CopyDataToDevice (staggered/func_global.h:944-963,
 * staggered/main.cpp:112-156, :245-262). */
int tc_create(const tc_params* prm, const double* zz, tc_handle** out);
int tc_destroy(tc_handle* h); /* data::dealloc_all, func_global.h:964-974 */

/* Ring levels 0..3 of vel/pres.  Host AoS double.  Either pointer may be NULL. */
int tc_upload_level(tc_handle* h, int level, const double* vel_aos, const double* p);
int tc_download_level(tc_handle* h, int level, double* vel_aos, double* p);
int tc_download_flux(tc_handle* h, int level, double* flux_aos);
/* Zero-copy device pointers (structure-of-arrays: u[N], v[N], w[N]; pressure p[N]);
 * element type double (TC_FP64) or float (TC_MIXED). */
int tc_device_level(tc_handle* h, int level, void** vel_soa, void** p);
int tc_get_stream(tc_handle* h, void** cuda_stream);
int tc_sync(tc_handle* h);

/* One SBDF3 time step: data::Step(t, tau, current_field, bdf_order),
 * staggered/func_global.h:897-942, collocated_AB3/func_global.h:387-450.
 * Writes vel/pres[(current_field+1)%4] and flux[current_field], flux[next].
 * Enqueued on the handle's stream; returns without waiting. */
int tc_step(tc_handle* h, double t, double tau, int current_field, int bdf_order);

/* Forcing: mode 0 = constant dp/dx source (the reference's sour_dpdx);
 * mode 1 = constant flow rate with target bulk velocity `value`: each step the
 * mean pressure gradient is chosen so that the bulk velocity after the step equals
 * the target.  tc_last_dpdx returns the gradient applied by the last step. */
int tc_set_forcing(tc_handle* h, int mode, double value);
int tc_last_dpdx(tc_handle* h, double* dpdx);

/* Binary checkpoint for an exact restart (replaces the reference's single-level VTK
 * ASCII q*.vtk / input.vtk, staggered/io.cpp:6-68, whose restart loses the BDF history):
 * a 256-byte header (scheme, precision, grid, current field, time t, forcing state) and
 * the four ring levels' velocity, flux and pressure in the device layout and working
 * precision.  Load checks scheme, precision and grid against the solver; the turbulence
 * model and its parameters are set by the caller, as at creation. */
int tc_checkpoint_save(tc_handle* h, const char* path, int current_field, double t);
int tc_checkpoint_load(tc_handle* h, const char* path, int* current_field, double* t);

/* Time-averaged plane statistics on the device (the reference's driver averages the
 * per-step profiles on the host, staggered/main.cpp:316-326): tc_stats_accumulate adds
 * weight x the per-plane means of level `level` (tc_profiles' 12 quantities per plane)
 * to a device accumulator without synchronising; tc_stats_read returns the weighted
 * means (NZ x 12) and the total weight; tc_stats_reset clears them. */
int tc_stats_accumulate(tc_handle* h, int level, double weight);
int tc_stats_read(tc_handle* h, double* profiles, double* total_weight);
int tc_stats_reset(tc_handle* h);

/* Device-controlled run (the reference's driver loop with its CFL control,
 * staggered/main.cpp:308-370, without a host synchronisation per step): up to `nsteps`
 * SBDF3 steps of time step `tau` from ring level `current_field`, replayed by a CUDA
 * graph whose while-loop repeats `check_every` steps (a multiple of 4, so the ring comes
 * back to `current_field`) and then computes on the device the CFL number of that level
 * (mode as tc_cfl); the loop ends when the CFL leaves [cfl_min, cfl_max] or the steps
 * are done.  Returns the steps done and the last CFL.  The caller has ramped the BDF
 * order to 3 with tc_step, and reacts to the returned CFL as the reference does (new
 * tau, order restart).  The graph is kept for the next call with the same tau,
 * current_field, check_every and mode.  Phase timing must be off. */
int tc_run_graph(tc_handle* h, double tau, int current_field, int nsteps, int check_every, int cfl_mode,
                 double cfl_min, double cfl_max, int* steps_done, double* cfl);

/* Turbulence model: kind TC_TURB_*; weights only for TC_TURB_MLP (see
 * tc_mlp_* in turbch_les.h).  Requires visc_type NAIVE (staggered) or GALERKIN. */
int tc_set_turb_model(tc_handle* h, int kind, const void* weights);

/* Diagnostics (FP64 accumulation), synchronous.
 * data::CalcIntegral / CalcKineticEnergy / CalcCFL / CalcProfiles
 * (staggered/func_global.h:678-808).  A NaN or Inf anywhere in the level's u, v, w,
 * p or nu_t makes these calls (and tc_diagnostics) return TC_E_NUMERIC, with the
 * outputs still written and the plane named in tc_last_error(); the reference reports
 * nothing here (its only numeric signal is the -1e50 written for a singular pivot,
 * staggered/func_global.h:169). */
int tc_integral(tc_handle* h, int level, double out[3]);
int tc_kinetic_energy(tc_handle* h, int level, double* out);
int tc_cfl(tc_handle* h, int level, double tau, int mode, double* out);
/* out: NZ x 12 doubles per plane: <u>,<v>,<w>, <uu>,<vv>,<ww>,<uv>,<uw>,<vw>, <nu_t>, <p>, <pp>
 * (the real9 layout of staggered/real3.h:39-50; w cell-centred for staggered). */
int tc_profiles(tc_handle* h, int level, double* out);
/* Fused per-step diagnostics: integral, CFL and profiles in one pass over the level
 * (main.cpp:313-338 calls the three separately).  Any output may be NULL. */
int tc_diagnostics(tc_handle* h, int level, double tau, double integral[3], double* cfl, double* profiles);

/* Where the diagnostics are computed (no counterpart in the reference, whose driver runs
 * separate reduction passes after the step).  mode 0: a separate pass over the level per
 * call (default); 1: the step's correction kernel also reduces the new level (staggered
 * schemes, NX % 4 == 0), a diagnostics call for that level and tau only adds the planes;
 * 2: as 1 while the caller reads the diagnostics of every step's output, as 0 otherwise.
 * The results agree to round-off (summation order). */
int tc_set_diag_fusion(tc_handle* h, int mode);

/* How the pressure solve's horizontal FFTs run (no counterpart in the reference, which
 * calls its FFT library per direction).  mode 1 (default): where (NX, NY) has a plane
 * kernel that fits the device, the x- and y-FFTs of each z-plane run in one launch, a
 * thread-block cluster holding the plane's half spectrum in its shared memory; 0: the
 * separate x- and y-FFT kernels.  The arithmetic is the same (round-off may differ by
 * FMA contraction). */
int tc_set_fft_fusion(tc_handle* h, int mode);

/* How the float flux kernel (mixed precision, staggered CROSS) fills its shared-memory
 * ring of velocity planes (no counterpart in the reference).  mode 0 (default): every
 * thread copies 16-byte chunks (cp.async); 1: tiles whose halo does not wrap (NX % 64 ==
 * 0, NY % 8 == 0) are filled by TMA tensor-map boxes, one per component and plane,
 * completed on an mbarrier (bounded waits: a load that never completes makes tc_sync
 * return TC_E_CUDA), the border tiles by cp.async in a second launch.  Same results. */
int tc_set_flux_staging(tc_handle* h, int mode);

/* Segregated IMEX Runge-Kutta step of the collocated scheme (collocated_SRK:
 * data::Step, func_global.h:317-408; method tables as collocated_SRK/imex.h:10-41).
 * The handle must be collocated with cross viscosity and no turbulence model; the
 * explicit term is then collocated_SRK's ExplicitTerm (func_global.h:270-307), the
 * source term the handle's sour_dpdx.  tc_srk_init takes the method as the reference's
 * main.cpp copies it into its data object (main.cpp:342-352): type TC_IMEX_*, stage
 * count S <= TC_SRK_MAX_STAGES, Butcher tables of (S+1) x S row-major values (last row
 * b), StabType 0 (Du + Sp = 0) or 1 (Du + S dp/dt = 0) and alpha_tau (the reference
 * uses half the method's alpha_tau_max).  It allocates the stage buffers (S+2 vectors,
 * 2S+3 scalars of the working precision) and switches the handle's pressure
 * normalisation to collocated_SRK's (shift sum(p vol)/area, func_global.h:130-137).
 * tc_srk_step advances ring level 0 (velocity, pressure) by tau, with dp/dt (StabType
 * 1) in the pressure slot of level 1 (the reference's qressure); t is accepted for the
 * reference's signature.  The reference's implicit term is identically zero
 * (func_global.h:310-315), so its Ku terms are left out (exact zeros). */
#define TC_SRK_MAX_STAGES 6
#define TC_IMEX_A 0
#define TC_IMEX_ARS 1
#define TC_IMEX_CK 2
int tc_srk_init(tc_handle* h, int imex_type, int nstages, const double* butcher_e, const double* butcher_i,
                int stab_type, double alpha_tau);
int tc_srk_step(tc_handle* h, double t, double tau);

/* Operator-level entry points on host buffers (the reference's operator methods,
 * used by its CPU/GPU self-checks, staggered/selftest.cpp:360-438). */
int tc_op_explicit_term(tc_handle* h, const double* vel_aos, double* flux_aos);    /* ExplicitTerm    */
int tc_op_apply_gradient(tc_handle* h, const double* p, double* grad_aos);         /* ApplyGradient   */
int tc_op_apply_divergence(tc_handle* h, const double* vel_aos, double* div);      /* ApplyDivergence */
int tc_op_unapply_gradient(tc_handle* h, const double* vel_aos, double* p);        /* UnapplyGradient */
int tc_op_pressure_solve(tc_handle* h, const double* rhs, double* p);              /* LinearSystemSolveFFT */
/* LinearSystemSolveFFT on device arrays (staggered/func_global.h:214-248 works on the
 * data object's device members): rhs and p are device buffers of N values in the working
 * precision (double for TC_FP64, float for TC_MIXED), cells [z][y][x]; rhs may equal p.
 * Asynchronous on the solver's stream (tc_get_stream); the same kernels as
 * tc_op_pressure_solve. */
int tc_pressure_solve_device(tc_handle* h, const void* rhs, void* p);
int tc_op_turb_visc(tc_handle* h, const double* vel_aos, double* nu_t);            /* RecalcTurbVisc  */
int tc_set_nu_t(tc_handle* h, const double* nu_t);
int tc_get_nu_t(tc_handle* h, double* nu_t);

/* Pressure solve (tc_op_pressure_solve's result up to round-off) on DEVICE buffers of N cells in
 * the handle's working precision (double for TC_FP64, float for TC_MIXED; rhs and p
 * may alias), enqueued on the handle's stream; no counterpart in the reference.  It
 * allocates nothing: the z-solve's elimination coefficients live in a static device
 * array of 32 MiB shared by all calls on a device, so the z-solve's
 * (NX/2+1)*NY*NZ*c*8 bytes (c = 3 for VV4, 1 otherwise) must fit (else TC_E_ARG),
 * and calls whose launches overlap in time race on it.  tc_create loads the module
 * that holds the array on the handle's device, so its 32 MiB are taken from device
 * memory when the handle is created (create handles before handing the rest of HBM
 * to a pool); each call then only looks the array's address up. */
int tc_op_pressure_solve_static(tc_handle* h, const void* rhs, void* p);

/* Seeded channel initial field on level `level`: u = 1.5(1 - y^2) + noise, v, w =
 * noise, noise uniform in [-amp, amp] from MT19937-64(seed) drawn 3 per cell in
 * index order; wall DOFs zero; projected divergence-free with the solver's own
 * operators when project != 0; pressure zero.  (Replaces SetInitialFields,
 * staggered/main.cpp:158-185, for seeded synthetic runs.) */
int tc_init_channel(tc_handle* h, int level, unsigned long long seed, double amp, int project);

/* Instrumentation.  With phase timing on, every tc_step records CUDA events around
 * its phases on the handle's stream (no synchronisation): 0 turbulence model,
 * 1 flux+combine, 2 divergence+x-FFT, 3 y-FFT, 4 banded z-solve, 5 inverse y-FFT,
 * 6 inverse x-FFT, 7 correction.  tc_phase_times waits for the stream, returns the
 * summed milliseconds per phase and the number of steps, and resets the sums.
 * tc_launch_count returns the number of kernels this handle has launched. */
#define TC_NPHASE 8
int tc_phase_timing(tc_handle* h, int enable);
int tc_phase_times(tc_handle* h, double ms[TC_NPHASE], int* nsteps);
int tc_launch_count(tc_handle* h, unsigned long long* n);

/* Wall-normal tanh mesh: z_j = H (1 + tanh(gamma (2j/n - 1)) / tanh gamma), j = 0..n. */
void tc_mesh_tanh(int n, double gamma, double H, double* z);

#ifdef __cplusplus
}
#endif
#endif
