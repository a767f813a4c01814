/*
 * tc_oracle.h -- CPU restatement of TurbChannel's per-time-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/, the
 * smoke() entry of __graft_entry__.py and bench.py's CPU-baseline / reference
 * legs load it.  The product (turbchannel_b200) never links or calls it.
 *
 * The oracle restates, in plain C, the numerics of
 *   staggered/func_global.h      (HW2 and VV4 staggered schemes, NAIVE/CROSS
 *                                 viscosity, Smagorinsky, FFT pressure solve,
 *                                 SBDF3 Step, reductions)
 *   staggered/main.cpp:12-156    (FillMatrix, solve_banded, mesh-derived data)
 *   collocated_AB3/func_global.h (collocated scheme, StabType 0/1)
 *   collocated_AB3/func_fluxes.h (collocated convection + Galerkin viscosity)
 * with runtime NX/NY/NZ (any 2^a*3^b periodic sizes).  Field layout is the
 * reference's: AoS real3, x fastest, wall-normal z slowest, 4-level rings.
 *
 * Compiled twice: ORC_REAL=double (FP64) and ORC_REAL=float (mirrors the
 * reference's USE_DOUBLE_PRECISION 0 build).  The host-facing API is always
 * double so one ctypes binding serves both.
 */
#ifndef TC_ORACLE_H
#define TC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_HW2 = 0, ORC_VV4 = 1, ORC_COLLOC = 2 };
enum { ORC_VISC_CROSS = 0, ORC_VISC_NAIVE = 1, ORC_VISC_GALERKIN = 2 };

typedef struct orc_params {
    int scheme;      /* ORC_HW2 / ORC_VV4 / ORC_COLLOC                         */
    int visc_type;   /* ORC_VISC_*                                              */
    int turb;        /* 0: DNS, 1: Smagorinsky-van Driest nu_t                  */
    int stab_type;   /* collocated StabType (collocated_AB3/config.h:52)       */
    int fd_mode;     /* collocated FDmode   (collocated_AB3/config.h:55)       */
    int NX, NY, NZ;  /* staggered: NZ cells (NZ+1 z-faces); colloc: NZ nodes   */
    double visc, sour_dpdx, inv_length_scale;
    double xmin, ymin, hx, hy, area;
} orc_params;

typedef struct orc orc;

orc* orc_create(const orc_params* p, const double* zz, int* err);
void orc_destroy(orc* o);
int  orc_real_size(void);

/* Mesh-derived arrays (staggered/main.cpp:112-156).  name: "DZ","DZW","GC1","GC2",
   "GCZ","MAT_A","MAT_D","KERG","KERG_norm2","cMAT_A". Returns count written. */
int  orc_get_mesh(const orc* o, const char* name, double* out);

/* Ring-level access, host AoS real3 (double) + pressure. */
void orc_set_level(orc* o, int level, const double* vel, const double* p);
void orc_get_level(const orc* o, int level, double* vel, double* p);
void orc_get_flux(const orc* o, int level, double* flux);
void orc_set_nu_t(orc* o, const double* nu_t);
void orc_get_nu_t(const orc* o, double* nu_t);

/* Operators on host AoS buffers (double in/out). */
void orc_apply_gradient(orc* o, const double* p, double* gp);
void orc_apply_divergence(orc* o, const double* v, double* dv);
void orc_unapply_gradient(orc* o, const double* v, double* p);
void orc_pressure_solve(orc* o, const double* rhs, double* p);
void orc_normalize_pressure(orc* o, double* p);
void orc_explicit_term(orc* o, const double* v, double* f);
void orc_flux_fd(orc* o, const double* v, int do_conv, int do_visc, double* f);
void orc_recalc_turb_visc(orc* o, const double* v);

/* One SBDF3 step (staggered/func_global.h:897-942, collocated_AB3/func_global.h:387-450).
   cfr_on: constant flow rate; after the step the bulk velocity is brought to
   cfr_target by a uniform shift of u (returned dp/dx in *dpdx_out). */
int  orc_step(orc* o, double t, double tau, int current_field, int bdf_order,
              int cfr_on, double cfr_target, double* dpdx_out);

/* Diagnostics (FP64 accumulation). */
void   orc_integral(const orc* o, int level, double out[3]);
double orc_kinetic_energy(const orc* o, int level);
double orc_cfl(const orc* o, int level, double tau, int mode);
void   orc_profiles(const orc* o, int level, double* out /* NZ x 12 */);

/* Seeded channel initial field: u = 1.5(1-y^2) + noise, v,w = noise, noise uniform
   in [-amp, amp] from MT19937-64(seed); projected divergence-free when project!=0. */
void orc_init_channel(orc* o, int level, unsigned long long seed, double amp, int project);
void orc_mt64_fill(unsigned long long seed, int n, unsigned long long* out);

/* Tanh wall-normal mesh: z_j = H*(1 + tanh(gamma*(2j/n - 1))/tanh(gamma)), j=0..n. */
void orc_mesh_tanh(int n, double gamma, double H, double* z);

/* Self-tests restated from staggered/selftest.cpp; return the printed norms. */
double orc_check_gradient_kernel(orc* o);
double orc_check_normalization_projection(orc* o);
double orc_check_matrix_symmetry(orc* o);
double orc_check_pressure_matrix(orc* o);
double orc_check_pressure_solver(orc* o, int itest);
double orc_check_conservation(orc* o, int itest, double out_K[3]);

/* Threads used by the OpenMP loops (0: leave the runtime default). */
void orc_set_threads(int n);
int  orc_get_threads(void);

/* Complex FFT used by the pressure solve (exposed for testing against numpy).
   n must be 2^a 3^b; sign -1 forward, +1 backward (unnormalised). */
int  orc_fft(int n, int sign, double* data /* 2n interleaved */);

#ifdef __cplusplus
}
#endif
#endif
