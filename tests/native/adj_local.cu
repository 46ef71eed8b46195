// Test harness (host code only): exposes the forward pointwise physics of the
// 2D MHD step and its reverse-mode versions (core_collapse_b200/csrc/
// mhd2d_adjoint.cuh) through a C ABI, so that tests/test_adjoint_local.py can
// compare every vector-Jacobian product with central finite differences.
#include "mhd2d_adjoint.cuh"

using namespace ccb;

namespace {
M2Const<double> mk(const double* k) {
    M2Const<double> c{};
    c.gamma = k[0]; c.gm1 = k[0] - 1.0; c.floor_rho = k[1]; c.floor_P = k[2]; c.eta = k[3];
    c.dx = k[4]; c.dy = k[5];
    c.inv_dx = 1.0 / k[4]; c.inv_dy = 1.0 / k[5];
    c.idx2 = 1.0 / (k[4] * k[4]); c.idy2 = 1.0 / (k[5] * k[5]);
    c.two_dx = 2.0 * k[4]; c.two_dy = 2.0 * k[5];
    c.resistive = k[3] > 0.0;
    return c;
}
Prim<double> P8(const double* a) {
    Prim<double> p;
    p.r = a[0]; p.u = a[1]; p.v = a[2]; p.w = a[3]; p.P = a[4]; p.bx = a[5]; p.by = a[6]; p.bz = a[7];
    return p;
}
void put8(const Prim<double>& p, double* a) {
    a[0] = p.r; a[1] = p.u; a[2] = p.v; a[3] = p.w; a[4] = p.P; a[5] = p.bx; a[6] = p.by; a[7] = p.bz;
}
void put7(const Flux<double>& f, double* a) {
    a[0] = f.f0; a[1] = f.f1; a[2] = f.f2; a[3] = f.f3; a[4] = f.f4; a[5] = f.f5; a[6] = f.f6;
}
Flux<double> F7(const double* a) {
    Flux<double> f;
    f.f0 = a[0]; f.f1 = a[1]; f.f2 = a[2]; f.f3 = a[3]; f.f4 = a[4]; f.f5 = a[5]; f.f6 = a[6];
    return f;
}
}  // namespace

extern "C" {

void fwd_hlld(const double* k, int dir, const double* L, const double* R, double Bn, double* F) {
    const M2Const<double> c = mk(k);
    put7(dir == 0 ? hlld_x(c, P8(L), P8(R), Bn) : hlld_y(c, P8(L), P8(R), Bn), F);
}

void vjp_hlld(const double* k, int dir, const double* L, const double* R, double Bn, const double* lF, double* lL,
              double* lR, double* lBn) {
    const M2Const<double> c = mk(k);
    Prim<double> a = prim_zero<double>(), b = prim_zero<double>();
    double bn = 0.0;
    if (dir == 0) hlld_x_vjp(c, P8(L), P8(R), Bn, F7(lF), a, b, bn);
    else hlld_y_vjp(c, P8(L), P8(R), Bn, F7(lF), a, b, bn);
    put8(a, lL); put8(b, lR); *lBn = bn;
}

void fwd_to_prim(const double* k, const double* U, double* W) {
    const M2Const<double> c = mk(k);
    put8(to_prim(c, U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7]), W);
}

void vjp_to_prim(const double* k, const double* U, const double* lW, double* lU) {
    const M2Const<double> c = mk(k);
    for (int i = 0; i < 8; i++) lU[i] = 0.0;
    to_prim_vjp(c, U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P8(lW), lU[0], lU[1], lU[2], lU[3], lU[4],
                lU[5], lU[6], lU[7]);
}

void fwd_floors(const double* k, const double* U, double* out) {
    const M2Const<double> c = mk(k);
    double rho = U[0], E = U[4];
    floors(c, rho, U[1], U[2], U[3], E, U[5], U[6], U[7]);
    for (int i = 0; i < 8; i++) out[i] = U[i];
    out[0] = rho; out[4] = E;
}

void vjp_floors(const double* k, const double* U, const double* lout, double* lU) {
    const M2Const<double> c = mk(k);
    for (int i = 0; i < 8; i++) lU[i] = lout[i];
    floors_vjp(c, U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], lU[0], lU[1], lU[2], lU[3], lU[4], lU[5], lU[6],
               lU[7]);
}

double fwd_mc(double a, double b, double cc) { return mc_slope(a, b, cc); }

void vjp_mc(double a, double b, double cc, double ls, double* out) {
    out[0] = out[1] = out[2] = 0.0;
    mc_slope_vjp(a, b, cc, ls, out[0], out[1], out[2]);
}

// Joule: in[16] = rho mx my mz E Bz Bx By bzE bzW bzN bzS byE byC bxN bxC; out[6] = rho..Bz after
void fwd_joule(const double* k, double dt, const double* in, double* out) {
    const M2Const<double> c = mk(k);
    double rho = in[0], mx = in[1], my = in[2], mz = in[3], E = in[4], Bz = in[5];
    const double bzE = in[8], bzW = in[9], bzN = in[10], bzS = in[11];
    const double dBzdy = (bzN - bzS) / c.two_dy, dBzdx = (bzE - bzW) / c.two_dx;
    const double dBydx = (in[12] - in[13]) / c.dx, dBxdy = (in[14] - in[15]) / c.dy;
    const double Jx = dBzdy, Jy = -dBzdx, Jz = dBydx - dBxdy;
    E = E + dt * c.eta * (Jx * Jx + Jy * Jy + Jz * Jz);
    const double lap = (bzE - 2.0 * Bz + bzW) * c.idx2 + (bzN - 2.0 * Bz + bzS) * c.idy2;
    Bz = Bz + dt * c.eta * lap;
    floors(c, rho, mx, my, mz, E, in[6], in[7], Bz);
    out[0] = rho; out[1] = mx; out[2] = my; out[3] = mz; out[4] = E; out[5] = Bz;
}

// lin[17]: adjoints of the 16 inputs, then eta
void vjp_joule(const double* k, double dt, const double* in, const double* lout, double* lin) {
    const M2Const<double> c = mk(k);
    JouleIn<double> J;
    J.rho = in[0]; J.mx = in[1]; J.my = in[2]; J.mz = in[3]; J.E = in[4]; J.Bz = in[5]; J.Bx = in[6]; J.By = in[7];
    J.bzE = in[8]; J.bzW = in[9]; J.bzN = in[10]; J.bzS = in[11];
    J.byE = in[12]; J.byC = in[13]; J.bxN = in[14]; J.bxC = in[15];
    JouleAdj<double> a{};
    for (int i = 0; i < 6; i++) a.l[i] = lout[i];
    joule_vjp(c, dt, J, a);
    for (int i = 0; i < 6; i++) lin[i] = a.l[i];
    lin[6] = a.Bx; lin[7] = a.By;
    lin[8] = a.bzE; lin[9] = a.bzW; lin[10] = a.bzN; lin[11] = a.bzS;
    lin[12] = a.byE; lin[13] = a.byC; lin[14] = a.bxN; lin[15] = a.bxC;
    lin[16] = a.eta;
}
}
