// cc_euler2d_main: drop-in for the reference's Euler/HLLC driver
// (euler2d_gravity_hllc.cpp main(), EH:645-737) on top of the C ABI: the
// reference's default parameters and init_random_blob initial condition, the
// same loop (while t < t_end - 1e-14: dt with the bad-dt abort, clamp to t_end,
// RK2 step) on the GPU, the same snapshot rule (t = 0, then after a step with
// t + 1e-14 >= next_store or t >= t_end - 1e-14) and the same fields rho, P,
// Mach.  The reference writes out2d_hllc.h5 (/x /y /t /rho /P /Mach); libhdf5
// is not available to this build, so the same datasets go to
// <out>/{x,y,t,rho,P,Mach}.npy (default out2d_hllc/).
//
// Usage: cc_euler2d_main [--precision fp64|fp32] [--Nx N] [--Ny N]
//                        [--t_end T] [--dt_store D] [--out DIR] [--checkpoint FILE] [--restart FILE]
// --checkpoint writes a restart file at the end of the run; --restart starts
// from one (same grid) instead of the initial condition, its first snapshot
// being the restored state at the restored time.
#include <sys/stat.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/cc_ic.h"
#include "../../include/cc_step.h"
#include "npy_out.h"

using namespace ccmain;

int main(int argc, char** argv) {
    cc_euler2d_params p;
    cc_euler2d_params_default(&p);   // the reference's Params defaults (EH:29-56)
    std::string out = "out2d_hllc";
    std::string ckpt, restart;
    for (int a = 1; a < argc; a++) {
        const std::string k = argv[a];
        if (a + 1 >= argc) {
            std::fprintf(stderr, "%s needs a value\n", k.c_str());
            return 2;
        }
        const std::string v = argv[++a];
        if (k == "--precision") p.precision = v == "fp32" ? CC_FP32 : CC_FP64;
        else if (k == "--Nx") p.Nx = std::atoi(v.c_str());
        else if (k == "--Ny") p.Ny = std::atoi(v.c_str());
        else if (k == "--t_end") p.t_end = std::atof(v.c_str());
        else if (k == "--dt_store") p.dt_store = std::atof(v.c_str());
        else if (k == "--out") out = v;
        else if (k == "--checkpoint") ckpt = v;
        else if (k == "--restart") restart = v;
        else {
            std::fprintf(stderr, "unknown option %s\n", k.c_str());
            return 2;
        }
    }
    const int Nx = p.Nx, Ny = p.Ny;
    const size_t N = (size_t)Nx * Ny;
    const double dx = (p.x1 - p.x0) / Nx, dy = (p.y1 - p.y0) / Ny;
    std::vector<double> x(Nx), y(Ny);
    for (int i = 0; i < Nx; i++) x[i] = p.x0 + (i + 0.5) * dx;
    for (int j = 0; j < Ny; j++) y[j] = p.y0 + (j + 0.5) * dy;

    cc_handle* h = nullptr;
    auto check = [&](int r, const char* what) {
        if (r != CC_OK) std::fprintf(stderr, "%s failed (%d): %s\n", what, r, h ? cc_last_error(h) : "");
        return r;
    };
    if (check(cc_euler2d_create(&p, &h), "cc_euler2d_create")) return 1;
    std::vector<std::vector<double>> f(4, std::vector<double>(N));
    double* fp[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
    double t = 0.0;
    if (restart.empty()) {
        if (cc_ic_euler2d_random_blob(&p, fp) != 0) {
            std::fprintf(stderr, "initial condition failed\n");
            return 1;
        }
        if (check(cc_euler2d_upload(h, fp[0], fp[1], fp[2], fp[3]), "upload")) return 1;
    } else {
        if (check(cc_euler2d_checkpoint_load(h, restart.c_str()), "cc_euler2d_checkpoint_load")) return 1;
        cc_diag d0;
        if (check(cc_euler2d_diagnostics(h, &d0), "diagnostics")) return 1;
        t = d0.t;
    }

    const char* names[3] = {"rho", "P", "Mach"};
    mkdir(out.c_str(), 0755);
    SeriesFile series[3];
    for (int k = 0; k < 3; k++)
        if (!series[k].open(out + "/" + names[k] + ".npy", {Ny, Nx})) {
            std::fprintf(stderr, "cannot write %s/%s.npy\n", out.c_str(), names[k]);
            return 1;
        }
    std::vector<double> times;
    std::vector<std::vector<double>> snap(3, std::vector<double>(N));
    double* sp[3] = {snap[0].data(), snap[1].data(), snap[2].data()};
    auto store = [&](double tt) {
        times.push_back(tt);
        if (check(cc_euler2d_derived(h, sp), "cc_euler2d_derived")) return false;
        for (int k = 0; k < 3; k++)
            if (!series[k].append(sp[k])) return false;
        return true;
    };

    // the main loop (EH:692-715)
    double next_store = t;
    if (!store(t)) return 1;
    next_store += p.dt_store;
    cc_diag d;
    while (t < p.t_end - 1e-14) {
        if (check(cc_euler2d_advance(h, 1, &t), "cc_euler2d_advance")) return 1;   // bad dt: CC_ERR_NONFINITE
        if (t + 1e-14 >= next_store || t >= p.t_end - 1e-14) {
            if (!store(t)) return 1;
            next_store += p.dt_store;
            if (check(cc_euler2d_diagnostics(h, &d), "diagnostics")) return 1;
            std::fprintf(stderr, "t=%.10g dt=%.10g snapshots=%zu\n", t, d.dt_last, times.size());
        }
    }
    if (!ckpt.empty() && check(cc_euler2d_checkpoint_save(h, ckpt.c_str()), "cc_euler2d_checkpoint_save")) return 1;
    bool ok = true;
    for (int k = 0; k < 3; k++) ok = series[k].finish() && ok;
    ok = write_npy(out + "/x.npy", {Nx}, x.data(), x.size()) && ok;
    ok = write_npy(out + "/y.npy", {Ny}, y.data(), y.size()) && ok;
    ok = write_npy(out + "/t.npy", {(long long)times.size()}, times.data(), times.size()) && ok;
    if (!ok) {
        std::fprintf(stderr, "writing %s failed\n", out.c_str());
        return 1;
    }
    std::printf("wrote %zu snapshots to %s/\n", times.size(), out.c_str());
    cc_destroy(h);
    return 0;
}
