// cc_mhd3d_main: drop-in for the reference's 3D driver
// (mhd3d_resistive_hlld_ct.cpp main(), M3:1131-1338) on top of the C ABI: the
// reference's default parameters and core-collapse IC, the same loop (dt
// clamped to t_end, RK2 step) on the GPU, the same snapshot rule (after a step
// with t >= t_next - 1e-12, t_next += dt_store; no snapshot at t = 0) and the
// same eleven fields.  The reference writes out3d_mhd.h5 (/x /y /z /t and
// /rho /P /Mach /u /v /w /vabs /Bx /By /Bz /divB of shape (Nt, Nz, Ny, Nx));
// libhdf5 is not available to this build, so the same datasets go to
// <out>/<name>.npy (default out3d_mhd/).
//
// Usage: cc_mhd3d_main [--precision fp64|fp32] [--Nx N] [--Ny N] [--Nz N]
//                      [--t_end T] [--dt_store D] [--out DIR] [--checkpoint FILE] [--restart FILE]
// --checkpoint writes a restart file at the end of the run; --restart starts
// from one (same grid) instead of the initial condition; frames then follow
// the same rule from the restored time (the first after the first step).
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
    cc_mhd3d_params p;
    cc_mhd3d_params_default(&p);   // the reference's Params defaults (M3:43-89)
    std::string out = "out3d_mhd";
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
        else if (k == "--Nz") p.Nz = std::atoi(v.c_str());
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
    const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
    const size_t N = (size_t)Nx * Ny * Nz;
    std::vector<double> x(Nx), y(Ny), z(Nz);
    // cell centres as the reference forms them (M3:1134-1143): x0 + (i + 0.5) * dx
    const double dx = (p.x1 - p.x0) / Nx, dy = (p.y1 - p.y0) / Ny, dz = (p.z1 - p.z0) / Nz;
    for (int i = 0; i < Nx; i++) x[i] = p.x0 + (i + 0.5) * dx;
    for (int j = 0; j < Ny; j++) y[j] = p.y0 + (j + 0.5) * dy;
    for (int k = 0; k < Nz; k++) z[k] = p.z0 + (k + 0.5) * dz;

    cc_handle* h = nullptr;
    auto check = [&](int r, const char* what) {
        if (r != CC_OK) std::fprintf(stderr, "%s failed (%d): %s\n", what, r, h ? cc_last_error(h) : "");
        return r;
    };
    if (check(cc_mhd3d_create(&p, &h), "cc_mhd3d_create")) return 1;
    std::vector<std::vector<double>> f = {std::vector<double>(N), std::vector<double>(N), std::vector<double>(N),
                                          std::vector<double>(N), std::vector<double>(N),
                                          std::vector<double>((size_t)(Nx + 1) * Ny * Nz),
                                          std::vector<double>((size_t)Nx * (Ny + 1) * Nz),
                                          std::vector<double>((size_t)Nx * Ny * (Nz + 1))};
    double* fp[8];
    for (int k = 0; k < 8; k++) fp[k] = f[k].data();
    double t = 0.0;
    if (restart.empty()) {
        cc_mhd3d_ic_knobs kn;
        cc_mhd3d_ic_knobs_default(&kn);
        if (cc_ic_mhd3d_reference(&p, &kn, fp) != 0) {
            std::fprintf(stderr, "initial condition failed\n");
            return 1;
        }
        if (check(cc_mhd3d_upload(h, fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7]), "upload")) return 1;
    } else {
        if (check(cc_mhd3d_checkpoint_load(h, restart.c_str()), "cc_mhd3d_checkpoint_load")) return 1;
        cc_diag d0;
        if (check(cc_mhd3d_diagnostics(h, &d0), "diagnostics")) return 1;
        t = d0.t;
    }

    const char* names[11] = {"rho", "P", "Mach", "u", "v", "w", "vabs", "Bx", "By", "Bz", "divB"};
    mkdir(out.c_str(), 0755);
    SeriesFile series[11];
    for (int k = 0; k < 11; k++)
        if (!series[k].open(out + "/" + names[k] + ".npy", {Nz, Ny, Nx})) {
            std::fprintf(stderr, "cannot write %s/%s.npy\n", out.c_str(), names[k]);
            return 1;
        }
    std::vector<double> tstore;
    std::vector<std::vector<double>> snap(11, std::vector<double>(N));
    double* sp[11];
    for (int k = 0; k < 11; k++) sp[k] = snap[k].data();

    // the main loop (M3:1285-1327)
    double tnext = t;
    while (t < p.t_end) {
        if (check(cc_mhd3d_advance(h, 1, &t), "cc_mhd3d_advance")) return 1;
        if (t >= tnext - 1e-12) {
            tstore.push_back(t);
            if (check(cc_mhd3d_derived(h, sp), "cc_mhd3d_derived")) return 1;
            for (int k = 0; k < 11; k++)
                if (!series[k].append(sp[k])) return 1;
            std::printf("Stored frame %zu at t=%g\n", tstore.size() - 1, t);
            tnext += p.dt_store;
        }
    }
    if (!ckpt.empty() && check(cc_mhd3d_checkpoint_save(h, ckpt.c_str()), "cc_mhd3d_checkpoint_save")) return 1;
    bool ok = true;
    for (int k = 0; k < 11; k++) ok = series[k].finish() && ok;
    ok = write_npy(out + "/x.npy", {Nx}, x.data(), x.size()) && ok;
    ok = write_npy(out + "/y.npy", {Ny}, y.data(), y.size()) && ok;
    ok = write_npy(out + "/z.npy", {Nz}, z.data(), z.size()) && ok;
    ok = write_npy(out + "/t.npy", {(long long)tstore.size()}, tstore.data(), tstore.size()) && ok;
    if (!ok) {
        std::fprintf(stderr, "writing %s failed\n", out.c_str());
        return 1;
    }
    std::printf("wrote %zu snapshots to %s/\n", tstore.size(), out.c_str());
    cc_destroy(h);
    return 0;
}
