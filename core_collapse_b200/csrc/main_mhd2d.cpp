// cc_mhd2d_main: drop-in for the reference's 2D driver
// (mhd2d_resistive_hlld_ct_gravity.cpp main(), M2:928-1130) on top of the
// C ABI: the reference's default parameters and core-collapse initial
// condition, the same time loop (Poisson, dt clamped to t_end, RK2 step) run
// on the GPU, the same snapshot rule (store at t = 0 and after every step with
// t >= next_store - 1e-15, next_store += dt_store) and the same ten derived
// fields per snapshot.
//
// Output: the reference writes out2d_mhd.h5 (datasets x, y, t and the ten
// fields of shape (Nt, Ny, Nx)).  libhdf5 is not available to this build, so
// the same datasets are written as NumPy .npy files (little-endian FP64) into
// a directory, default out2d_mhd/: x.npy, y.npy, t.npy, rho.npy, P.npy,
// Mach.npy, u.npy, v.npy, vabs.npy, Bx.npy, By.npy, Bz.npy, divB.npy.
// Field files grow one snapshot at a time; their headers are rewritten with
// the final Nt at the end.
//
// Usage: cc_mhd2d_main [--precision fp64|fp32] [--poisson sor|fft|lex]
//                      [--Nx N] [--Ny N] [--t_end T] [--dt_store D]
//                      [--out DIR] [--checkpoint FILE] [--restart FILE]
//                      [--max_steps N]
// --checkpoint writes a restart file at the end of the run; --restart starts
// from one (same grid) instead of the initial condition.  --poisson lex runs
// the reference's own lexicographic SOR (CC_POISSON_SOR_LEX: its sweep order
// and sums, slow; the default red-black SOR is the production solve).
// --max_steps ends the loop after N steps even before t_end (the output then
// holds the snapshots stored so far): with its default parameters the
// reference's collapse makes dt fall by orders of magnitude near t = 0.275.
#include <sys/stat.h>

#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cc_ic.h"
#include "../../include/cc_step.h"
#include "npy_out.h"

namespace {

using namespace ccmain;

const char* const FIELD_NAMES[10] = {"rho", "P", "Mach", "u", "v", "vabs", "Bx", "By", "Bz", "divB"};

int check(cc_handle* h, int r, const char* what) {
    if (r != CC_OK) std::fprintf(stderr, "%s failed (%d): %s\n", what, r, h ? cc_last_error(h) : "");
    return r;
}

}  // namespace

int main(int argc, char** argv) {
    cc_mhd2d_params p;
    cc_mhd2d_params_default(&p);   // the reference's Params defaults (M2:44-86)
    std::string out = "out2d_mhd", ckpt, restart;
    long long max_steps = -1;
    for (int a = 1; a < argc; a++) {
        const std::string k = argv[a];
        const char* v = (a + 1 < argc) ? argv[a + 1] : nullptr;
        auto need = [&]() {
            if (!v) {
                std::fprintf(stderr, "%s needs a value\n", k.c_str());
                std::exit(2);
            }
            a++;
            return std::string(v);
        };
        if (k == "--precision") p.precision = need() == "fp32" ? CC_FP32 : CC_FP64;
        else if (k == "--poisson") {
            const std::string kind = need();
            p.poisson_kind = kind == "fft" ? CC_POISSON_FFT : kind == "lex" ? CC_POISSON_SOR_LEX : CC_POISSON_SOR;
        }
        else if (k == "--Nx") p.Nx = std::atoi(need().c_str());
        else if (k == "--Ny") p.Ny = std::atoi(need().c_str());
        else if (k == "--t_end") p.t_end = std::atof(need().c_str());
        else if (k == "--dt_store") p.dt_store = std::atof(need().c_str());
        else if (k == "--out") out = need();
        else if (k == "--checkpoint") ckpt = need();
        else if (k == "--restart") restart = need();
        else if (k == "--max_steps") max_steps = std::atoll(need().c_str());
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
    if (check(h, cc_mhd2d_create(&p, &h), "cc_mhd2d_create")) return 1;
    double t = 0.0;
    if (restart.empty()) {
        // the reference main()'s initial condition (M2:957-1048)
        std::vector<std::vector<double>> f = {std::vector<double>(N), std::vector<double>(N), std::vector<double>(N),
                                              std::vector<double>(N), std::vector<double>(N), std::vector<double>(N),
                                              std::vector<double>((size_t)(Nx + 1) * Ny),
                                              std::vector<double>((size_t)Nx * (Ny + 1))};
        double* fp[8];
        for (int k = 0; k < 8; k++) fp[k] = f[k].data();
        cc_mhd2d_ic_knobs kn;
        cc_mhd2d_ic_knobs_default(&kn);
        if (cc_ic_mhd2d_reference(&p, &kn, fp) != 0) {
            std::fprintf(stderr, "initial condition failed\n");
            return 1;
        }
        const double* cf[8];
        for (int k = 0; k < 8; k++) cf[k] = fp[k];
        if (check(h, cc_mhd2d_upload(h, cf[0], cf[1], cf[2], cf[3], cf[4], cf[5], cf[6], cf[7]), "upload")) return 1;
    } else {
        if (check(h, cc_mhd2d_checkpoint_load(h, restart.c_str()), "cc_mhd2d_checkpoint_load")) return 1;
    }
    cc_diag d;
    if (check(h, cc_mhd2d_diagnostics(h, &d), "diagnostics")) return 1;
    t = d.t;
    std::printf("init max|divB|=%.12g\n", d.max_divB);

    mkdir(out.c_str(), 0755);   // an existing directory is fine
    SeriesFile series[10];
    for (int k = 0; k < 10; k++)
        if (!series[k].open(out + "/" + FIELD_NAMES[k] + ".npy", {Ny, Nx})) {
            std::fprintf(stderr, "cannot write %s/%s.npy\n", out.c_str(), FIELD_NAMES[k]);
            return 1;
        }
    std::vector<double> tstore;
    std::vector<std::vector<double>> snap(10, std::vector<double>(N));
    double* sp[10];
    for (int k = 0; k < 10; k++) sp[k] = snap[k].data();
    auto store = [&](double tt) {
        tstore.push_back(tt);
        if (check(h, cc_mhd2d_derived(h, sp), "cc_mhd2d_derived")) return false;
        for (int k = 0; k < 10; k++)
            if (!series[k].append(sp[k])) return false;
        return true;
    };

    // the main loop (M2:1111-1129)
    double next_store = t;
    if (!store(t)) return 1;
    long long steps = 0;
    while (t < p.t_end) {
        if (max_steps >= 0 && steps >= max_steps) {
            if (check(h, cc_mhd2d_diagnostics(h, &d), "diagnostics")) return 1;
            std::printf("stopped after %lld steps: t=%.7g dt=%.7g\n", steps, t, d.dt_last);
            break;
        }
        if (check(h, cc_mhd2d_advance(h, 1, &t), "cc_mhd2d_advance")) return 1;
        steps++;
        if (t >= next_store - 1e-15) {
            if (check(h, cc_mhd2d_diagnostics(h, &d), "diagnostics")) return 1;
            std::printf("t=%.7g dt=%.7g max|divB|=%.12g\n", t, d.dt_last, d.max_divB);
            if (!store(t)) return 1;
            next_store += p.dt_store;
        }
    }
    bool ok = true;
    for (int k = 0; k < 10; k++) ok = series[k].finish() && ok;
    ok = write_npy(out + "/x.npy", {Nx}, x.data(), x.size()) && ok;
    ok = write_npy(out + "/y.npy", {Ny}, y.data(), y.size()) && ok;
    ok = write_npy(out + "/t.npy", {(long long)tstore.size()}, tstore.data(), tstore.size()) && ok;
    if (!ok) {
        std::fprintf(stderr, "writing %s failed\n", out.c_str());
        return 1;
    }
    if (!ckpt.empty() && check(h, cc_mhd2d_checkpoint_save(h, ckpt.c_str()), "cc_mhd2d_checkpoint_save")) return 1;
    std::printf("wrote %zu snapshots to %s/\n", tstore.size(), out.c_str());
    cc_destroy(h);
    return 0;
}
