// turbch_run -- channel-flow driver over the C ABI, with the reference driver's
// command line (staggered/io.cpp:102-125: -d, --nz, -t, -a, --TimeStepsMax, --tau,
// --CFLmin, --CFLmax, -s, -f, -p) and time loop (staggered/main.cpp:290-371: SBDF
// order ramp, per-step bulk velocity, profiles and CFL, dt halving / x1.5 with order
// restart, log.dat, time-averaged profiles).  Options not in the reference select the
// scheme and sizes that the reference fixes at compile time.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "turbch_data.hpp"

struct Opts {
    int device = 0, NZ = 64, NX = 64, NY = 64, steps_max = 0x7FFFFFFF;
    double time_max = 100.0, t_avg = 0.0, tau = 1e-3, cflmin = 0.05, cflmax = 0.5;
    int sprog = 200, fprog = 1000000, pprog = 100000;
    std::string scheme = "vv4", precision = "fp64";
    bool les = false, cfr = false;
    double re_bulk = 5600, gamma = 1.8, lx = 4 * M_PI, ly = 4 * M_PI / 3, re_tau = 0;
    unsigned long long seed = 12345;
};

static void usage() {
    std::printf(
        "Turbulent flow between parallel plates (B200)\n"
        "  -d,--device N            device to use\n"
        "  --nz N                   number of cells (staggered) / nodes (collocated) in the normal direction\n"
        "  -t,--TimeMax T           maximal integration time\n"
        "  -a,--TimeStartAveraging T time where averaging should be started\n"
        "  --TimeStepsMax N         maximal number of iterations\n"
        "  --tau T                  initial timestep size\n"
        "  --CFLmin C, --CFLmax C   timestep adaptation thresholds\n"
        "  -s,--SProgress N         timesteps between writing to screen and log\n"
        "  -f,--FProgress N         timesteps between writing a field (binary dump)\n"
        "  -p,--PProgress N         timesteps between writing a profile\n"
        "  --scheme hw2|vv4|colloc  --nx N --ny N --precision fp64|mixed --les\n"
        "  --re-bulk R --gamma G --lx L --ly L --cfr --seed S\n");
}

static bool parse(int argc, char** argv, Opts& o) {
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&](void) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", a.c_str());
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "-h" || a == "--help") { usage(); return false; }
        else if (a == "-d" || a == "--device") o.device = std::atoi(val());
        else if (a == "--nz") o.NZ = std::atoi(val());
        else if (a == "--nx") o.NX = std::atoi(val());
        else if (a == "--ny") o.NY = std::atoi(val());
        else if (a == "-t" || a == "--TimeMax") o.time_max = std::atof(val());
        else if (a == "-a" || a == "--TimeStartAveraging") o.t_avg = std::atof(val());
        else if (a == "--TimeStepsMax") o.steps_max = std::atoi(val());
        else if (a == "--tau") o.tau = std::atof(val());
        else if (a == "--CFLmin") o.cflmin = std::atof(val());
        else if (a == "--CFLmax") o.cflmax = std::atof(val());
        else if (a == "-s" || a == "--SProgress") o.sprog = std::atoi(val());
        else if (a == "-f" || a == "--FProgress") o.fprog = std::atoi(val());
        else if (a == "-p" || a == "--PProgress") o.pprog = std::atoi(val());
        else if (a == "--scheme") o.scheme = val();
        else if (a == "--precision") o.precision = val();
        else if (a == "--les") o.les = true;
        else if (a == "--cfr") o.cfr = true;
        else if (a == "--re-bulk") o.re_bulk = std::atof(val());
        else if (a == "--gamma") o.gamma = std::atof(val());
        else if (a == "--lx") o.lx = std::atof(val());
        else if (a == "--ly") o.ly = std::atof(val());
        else if (a == "--seed") o.seed = std::strtoull(val(), nullptr, 10);
        else {
            std::fprintf(stderr, "unknown option %s\n", a.c_str());
            usage();
            std::exit(2);
        }
    }
    return true;
}

int main(int argc, char** argv) {
    Opts o;
    if (!parse(argc, argv, o)) return 0;
    tc_params p = {};
    p.scheme = o.scheme == "hw2" ? TC_SCHEME_HW2 : o.scheme == "colloc" ? TC_SCHEME_COLLOC : TC_SCHEME_VV4;
    p.precision = o.precision == "mixed" ? TC_MIXED : TC_FP64;
    p.visc_type = p.scheme == TC_SCHEME_COLLOC ? (o.les ? TC_VISC_GALERKIN : TC_VISC_CROSS)
                                               : (o.les ? TC_VISC_NAIVE : TC_VISC_CROSS);
    p.turb_model = o.les ? TC_TURB_SMAGORINSKY : TC_TURB_NONE;
    p.NX = o.NX;
    p.NY = o.NY;
    p.NZ = o.NZ;
    p.stab_type = p.scheme == TC_SCHEME_COLLOC ? 1 : 0;
    p.fd_mode = 1;
    p.device = o.device;
    const double H = 1.0, visc = 2.0 * H / o.re_bulk;
    const double re_tau = 0.09 * std::pow(o.re_bulk, 0.88), u_tau = re_tau * visc / H;
    p.visc = visc;
    p.sour_dpdx = u_tau * u_tau / H;
    p.inv_length_scale = u_tau / visc;
    p.hx = o.lx / o.NX;
    p.hy = o.ly / o.NY;
    const int nint = p.scheme == TC_SCHEME_COLLOC ? o.NZ - 1 : o.NZ;
    std::vector<double> zz(nint + 1);
    tc_mesh_tanh(nint, o.gamma, H, zz.data());
    p.area = o.lx * o.ly * (zz.back() - zz.front());
    try {
        turbch::Data S(p, zz);
        if (o.cfr) S.SetConstantFlowRate(1.0);
        turbch::check(tc_init_channel(S.handle(), 0, o.seed, 0.1, 1));
        const int NZ = o.NZ;
        std::vector<double> prof(12 * NZ), avg(12 * NZ, 0.0);
        FILE* log = std::fopen("log.dat", "wt");
        double t = 0, tau = o.tau, tavg = 0;
        int cur = 0, start = 0;
        const int max_order = 3;
        std::printf("Start of time integration (N=%i,%i,%i)\n", o.NX, o.NY, o.NZ);
        for (int it = 0;; it++) {
            S.Step(it * tau, tau, cur, std::min(it - start + 1, max_order));
            cur = (cur + 1) % 4;
            double I[3], cfl;
            turbch::check(tc_diagnostics(S.handle(), cur, tau, I, &cfl, prof.data()));
            if (t >= o.t_avg) {
                for (int k = 0; k < 12 * NZ; k++) avg[k] += tau * prof[k];
                tavg += tau;
            }
            t += tau;
            const bool last = t >= o.time_max || it + 1 == o.steps_max;
            const double dz0 = zz[1] - zz[0];
            const double dudy = p.scheme == TC_SCHEME_COLLOC ? prof[12 * 1] / dz0 : prof[0] / (0.5 * dz0);
            const double uf = dudy < 0 ? 0 : std::sqrt(dudy * visc);
            const double dudy_av = tavg > 0 ? (p.scheme == TC_SCHEME_COLLOC ? avg[12] / (dz0 * tavg) : avg[0] / (0.5 * dz0 * tavg)) : 0;
            const double uf_av = dudy_av < 0 ? 0 : std::sqrt(dudy_av * visc);
            const double ub = I[0] / p.area;
            if (it % o.sprog == 0 || last) {
                std::printf("T=%f Ubulk=%.04f tau=%.1e CFL=%.04f Ufric=%.04f UfricAv=%.04f\n", t, ub, tau, cfl, uf, uf_av);
                std::fprintf(log, "%f %f %e %f %f %f\n", t, ub, tau, cfl, uf, uf_av);
            }
            if (it != 0 && it % o.fprog == 0) {
                std::vector<double> v(3 * S.N3D()), q(S.N3D());
                S.Download(cur, v.data(), q.data());
                char fn[64];
                std::snprintf(fn, sizeof fn, "q%05i.bin", it);
                FILE* f = std::fopen(fn, "wb");
                std::fwrite(v.data(), sizeof(double), v.size(), f);
                std::fwrite(q.data(), sizeof(double), q.size(), f);
                std::fclose(f);
            }
            if (it != 0 && it % o.pprog == 0) {
                char fn[64];
                std::snprintf(fn, sizeof fn, "r%05i.dat", it);
                FILE* f = std::fopen(fn, "wt");
                for (int z = 0; z < NZ; z++) {
                    for (int k = 0; k < 12; k++) std::fprintf(f, "%e ", prof[12 * z + k]);
                    std::fprintf(f, "\n");
                }
                std::fclose(f);
            }
            if (last) break;
            while (cfl > o.cflmax) {  // staggered/main.cpp:361-370
                cfl *= 0.5;
                tau *= 0.5;
                start = it + 1;
            }
            if (cfl < o.cflmin) {
                cfl *= 1.5;
                tau *= 1.5;
                start = it + 1;
            }
        }
        std::fclose(log);
        if (tavg > 0) {
            FILE* f = std::fopen("res.dat", "wt");
            for (int z = 0; z < NZ; z++) {
                for (int k = 0; k < 12; k++) std::fprintf(f, "%e ", avg[12 * z + k] / tavg);
                std::fprintf(f, "\n");
            }
            std::fclose(f);
        }
    } catch (const turbch::Error& e) {
        std::fprintf(stderr, "turbch error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}
