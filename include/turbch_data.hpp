// turbch_data.hpp -- header-only C++ stand-in for the reference's GPU solver object
// (`data_cuda::data`, staggered/data_global_inc.h:11-76 and
// collocated_AB3/data_global.h:74-170) built on the C ABI of include/turbch.h.
//
// The reference driver keeps raw device pointers to AoS real3 ring levels and passes
// them back into the diagnostics (staggered/main.cpp:308-338).  Here the ring lives
// inside the library in structure-of-arrays form, so levels are named by their ring
// index instead of by pointer; everything else (Step arguments, ring convention,
// diagnostics, host AoS copies) is unchanged.  Errors throw turbch::Error carrying
// tc_last_error() (the reference prints and exits, staggered/func_cuda.cpp:23-35).
#ifndef TURBCH_DATA_HPP
#define TURBCH_DATA_HPP
#include <stdexcept>
#include <string>
#include <vector>

#include "turbch.h"

namespace turbch {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != TC_OK) throw Error(rc, tc_last_error());
}

class Data {
   public:
    // zz: NZ+1 face coordinates (staggered) or NZ node coordinates (collocated).
    Data(const tc_params& p, const std::vector<double>& zz) : prm_(p) { check(tc_create(&p, zz.data(), &h_)); }
    ~Data() { tc_destroy(h_); }
    Data(const Data&) = delete;
    Data& operator=(const Data&) = delete;

    int NX() const { return prm_.NX; }
    int NY() const { return prm_.NY; }
    int NZ() const { return prm_.NZ; }
    long long N3D() const { return (long long)prm_.NX * prm_.NY * prm_.NZ; }
    tc_handle* handle() { return h_; }

    // data::Step (staggered/func_global.h:897-942); enqueued, returns immediately.
    void Step(double t_start, double tau, int current_field, int bdf_order) {
        check(tc_step(h_, t_start, tau, current_field, bdf_order));
    }
    void Sync() { check(tc_sync(h_)); }

    // Host copies of a ring level (AoS (u,v,w) per cell + pressure), replacing the
    // cudaMemcpy calls of staggered/main.cpp:283-286, 348-349.
    void Upload(int level, const double* vel_aos, const double* p) { check(tc_upload_level(h_, level, vel_aos, p)); }
    void Download(int level, double* vel_aos, double* p) { check(tc_download_level(h_, level, vel_aos, p)); }

    // Diagnostics of staggered/func_global.h:678-808 on ring level `level`.
    void CalcIntegral(int level, double out[3]) { check(tc_integral(h_, level, out)); }
    double CalcKineticEnergy(int level) {
        double e;
        check(tc_kinetic_energy(h_, level, &e));
        return e;
    }
    double CalcCFL(int level, double tau, int mode = 3) {
        double c;
        check(tc_cfl(h_, level, tau, mode, &c));
        return c;
    }
    // av_u[NZ] of real9 (u[3], uu[6], nu_t, p, pp), as 12 doubles per plane.
    void CalcProfiles(int level, double* av_u) { check(tc_profiles(h_, level, av_u)); }

    // Operator methods used by the reference's CPU/GPU self-checks (selftest.cpp:360-438).
    void ApplyGradient(const double* p, double* grad_aos) { check(tc_op_apply_gradient(h_, p, grad_aos)); }
    void UnapplyGradient(const double* vel_aos, double* p) { check(tc_op_unapply_gradient(h_, vel_aos, p)); }
    void ExplicitTerm(const double* vel_aos, double* flux_aos) { check(tc_op_explicit_term(h_, vel_aos, flux_aos)); }

    // Forcing: constant dp/dx (the reference's sour_dpdx) or constant flow rate.
    void SetConstantPressureGradient(double dpdx) { check(tc_set_forcing(h_, 0, dpdx)); }
    void SetConstantFlowRate(double bulk_velocity) { check(tc_set_forcing(h_, 1, bulk_velocity)); }
    double LastPressureGradient() {
        double d;
        check(tc_last_dpdx(h_, &d));
        return d;
    }

    // restart, time averaging and device-controlled runs (no counterpart in the reference's object)
    void SaveCheckpoint(const std::string& path, int current_field, double t) {
        check(tc_checkpoint_save(h_, path.c_str(), current_field, t));
    }
    void LoadCheckpoint(const std::string& path, int& current_field, double& t) {
        check(tc_checkpoint_load(h_, path.c_str(), &current_field, &t));
    }
    void StatsAccumulate(int level, double weight = 1.0) { check(tc_stats_accumulate(h_, level, weight)); }
    double StatsRead(double* profiles) {
        double w;
        check(tc_stats_read(h_, profiles, &w));
        return w;
    }
    void StatsReset() { check(tc_stats_reset(h_)); }
    // steps done; cfl receives the CFL number of the last device-side check
    int RunGraph(double tau, int current_field, int nsteps, int check_every, int cfl_mode, double cfl_min,
                 double cfl_max, double& cfl) {
        int done;
        check(tc_run_graph(h_, tau, current_field, nsteps, check_every, cfl_mode, cfl_min, cfl_max, &done, &cfl));
        return done;
    }

   private:
    tc_params prm_;
    tc_handle* h_ = nullptr;
};

}  // namespace turbch
#endif
