/*
 * ref_srk_driver.cu -- C entry points over the reference's collocated_SRK CPU solver
 * object (its data::Step, collocated_SRK/func_global.h:317-408).  The reference keeps
 * main() and both solver namespaces in one translation unit, so this file compiles
 * that unit in place (its main renamed) plus imex.cpp (CalcD), and adds the entry
 * points after it.  Setup follows collocated_SRK/main.cpp:336-398 with the node
 * coordinates, physical parameters and the IMEX method supplied by the caller; the
 * mesh size in x and y is the reference's compile-time NX = 128, NY = 64.
 * TEST INFRASTRUCTURE ONLY (oracle/_ref/).
 */
#include <thrust/execution_policy.h>  // thrust::host / thrust::device (not pulled in by newer Thrust)
#define main tcref_srk_reference_main
#include "main.cpp"
#undef main
#include "imex.cpp"

extern "C" {
int ref_srk_nx(void) { return NX; }
int ref_srk_ny(void) { return NY; }
int ref_srk_nzmax(void) { return NZ_MAX; }

int ref_srk_setup(int nz, const double* zz, double visc, double sour_dpdx, double hx, double hy, double area,
                  int imex_type, int nstages, const double* be, const double* bi, int stab_type, double alpha_tau,
                  int threads) {
    if (nz > NZ_MAX || nz < 4 || nstages < 1 || nstages > MAX_N_STAGES) return 1;
    if (threads > 0) omp_set_num_threads(threads);
    for (int i = 0; i < nz; i++) Z_CPU[i] = zz[i];
    for (int i = 0; i < nz - 1; i++) data_cpu::DZ[i] = Z_CPU[i + 1] - Z_CPU[i];
    main_params& MD = DATA_CPU;
    MD.IMEXtype = imex_type == 0 ? tIMEXtype::IMEX_A : (imex_type == 1 ? tIMEXtype::IMEX_ARS : tIMEXtype::IMEX_CK);
    MD.NStages = nstages;
    const int size = nstages * (nstages + 1);
    std::vector<double> I(bi, bi + size);
    for (int i = 0; i < size; i++) {
        MD.ButcherE[i] = be[i];
        MD.ButcherI[i] = bi[i];
    }
    std::vector<double> d = tIMEXMethod::CalcD(nstages, I);
    for (int i = 0; i < nstages; i++) MD.d[i] = d[i];
    MD.StabType = stab_type;
    MD.alpha_tau = alpha_tau;
    MD.visc = visc;
    MD.sour_dpdx = sour_dpdx;
    MD.NZ = nz;
    MD.N3D = NX * NY * nz;
    MD.hx = hx;
    MD.hy = hy;
    MD.inv_hx = 1. / hx;
    MD.inv_hy = 1. / hy;
    MD.area = area;
    MD.xmin = 0.;
    MD.ymin = 0.;
    MD.FDmode = 1;
    DATA_CPU.alloc_all();
    DATA_CPU.InitFourier();
    double* A = data_cpu::MAT_A;
    A[0] = 0.;
    for (int j = 1; j < nz; j++) A[j] = DATA_CPU.hx * DATA_CPU.hy / data_cpu::DZ[j - 1];
    if (DATA_CPU.FDmode) {
        A[1] *= 0.5;
        A[nz - 1] *= 0.5;
    }
    return 0;
}

void ref_srk_set(const double* vel, const double* p, const double* dpdt) {
    for (int i = 0; i < DATA_CPU.N3D; i++) {
        for (int c = 0; c < 3; c++) DATA_CPU.velocity[i][c] = vel[3 * i + c];
        DATA_CPU.pressure[i] = p[i];
        DATA_CPU.qressure[i] = dpdt[i];
    }
}

void ref_srk_get(double* vel, double* p, double* dpdt) {
    for (int i = 0; i < DATA_CPU.N3D; i++) {
        for (int c = 0; c < 3; c++) vel[3 * i + c] = DATA_CPU.velocity[i][c];
        p[i] = DATA_CPU.pressure[i];
        dpdt[i] = DATA_CPU.qressure[i];
    }
}

void ref_srk_step(double t, double tau) { DATA_CPU.Step(t, tau, DATA_CPU.velocity, DATA_CPU.pressure, DATA_CPU.qressure); }
}
