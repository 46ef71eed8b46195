// Reverse-mode (vector-Jacobian) versions of the pointwise physics of the 2D
// resistive-MHD step (mhd2d_physics.cuh, which follows
// mhd2d_resistive_hlld_ct_gravity.cpp, cited M2:<line>).
//
// Every *_vjp function takes the forward inputs, recomputes the forward
// intermediates with the same expressions as the forward function (so every
// branch -- floors, limiter choices, HLLD region, guards -- is decided exactly
// as in the forward pass), and accumulates adjoint-times-partial-derivative
// into the input adjoints (+=).  The derivative of a branch is that of the
// branch taken; boundaries between branches (measure zero) get the taken
// side's derivative.  Host and device callable, so the local derivatives are
// checked against finite differences on the CPU.
#pragma once
#include "mhd2d_physics.cuh"

namespace ccb {

#define CC_HD __host__ __device__ __forceinline__

template <class T> CC_HD Prim<T> prim_zero() {
    Prim<T> p;
    p.r = p.u = p.v = p.w = p.P = p.bx = p.by = p.bz = T(0);
    return p;
}

template <class T> CC_HD void prim_acc(Prim<T>& a, const Prim<T>& b) {
    a.r += b.r; a.u += b.u; a.v += b.v; a.w += b.w; a.P += b.P; a.bx += b.bx; a.by += b.by; a.bz += b.bz;
}

// energy (M2:357): P/gm1 + 0.5 r |v|^2 + 0.5 |B|^2
template <class T>
CC_HD void energy_vjp(const M2Const<T>& c, const Prim<T>& W, T lE, Prim<T>& lW) {
    lW.P += lE * (T(1) / c.gm1);
    lW.r += T(0.5) * (W.u * W.u + W.v * W.v + W.w * W.w) * lE;
    lW.u += W.r * W.u * lE;
    lW.v += W.r * W.v * lE;
    lW.w += W.r * W.w * lE;
    lW.bx += W.bx * lE;
    lW.by += W.by * lE;
    lW.bz += W.bz * lE;
}

// fast magnetosonic speed (M2:148-174)
template <class T>
CC_HD void fast_speed_vjp(const M2Const<T>& c, const Prim<T>& W, T bn, T lcf, Prim<T>& lW, T& lbn) {
    if (lcf == T(0)) return;
    const T rf = vmax(W.r, c.floor_rho);
    const T a2 = c.gamma * W.P / rf;
    const T b2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
    const T rr = vmax(W.r, tiny_pos<T>());
    const T vA2 = b2 / rr;
    const T vn2 = (bn * bn) / rr;
    const T s = a2 + vA2;
    const T disc0 = s * s - T(4.0) * a2 * vn2;
    const T disc = vmax(T(0.0), disc0);
    const T sq = sqrt(disc);
    const T cf2 = T(0.5) * (s + sq);
    const T cf = sqrt(vmax(T(0.0), cf2));
    const T lcf2 = (T(0.0) < cf2 && cf > T(0)) ? lcf / (T(2) * cf) : T(0);
    T ls = T(0.5) * lcf2;
    const T lsq = T(0.5) * lcf2;
    const T ldisc = (T(0.0) < disc0 && sq > T(0)) ? lsq / (T(2) * sq) : T(0);
    ls += T(2) * s * ldisc;
    T la2 = -T(4.0) * vn2 * ldisc;
    const T lvn2 = -T(4.0) * a2 * ldisc;
    la2 += ls;
    const T lvA2 = ls;
    const T i_rr = T(1) / rr, i_rf = T(1) / rf;
    const T lb2 = lvA2 * i_rr;
    const T lrr = -(lvA2 * vA2 + lvn2 * vn2) * i_rr;
    lbn += T(2) * bn * lvn2 * i_rr;
    if (!(W.r < tiny_pos<T>())) lW.r += lrr;
    lW.P += c.gamma * la2 * i_rf;
    const T lrf = -la2 * a2 * i_rf;
    if (!(W.r < c.floor_rho)) lW.r += lrf;
    lW.bx += T(2) * W.bx * lb2;
    lW.by += T(2) * W.by * lb2;
    lW.bz += T(2) * W.bz * lb2;
}

// x-normal ideal flux (M2:351-370)
template <class T>
CC_HD void ideal_flux_vjp(const M2Const<T>& c, const Prim<T>& W, const Flux<T>& lF, Prim<T>& lW) {
    const T r = W.r, u = W.u, v = W.v, w = W.w, Bx = W.bx, By = W.by, Bz = W.bz;
    const T B2 = Bx * Bx + By * By + Bz * Bz;
    const T pt = W.P + T(0.5) * B2;
    const T E = energy(c, W);
    const T vdotB = u * Bx + v * By + w * Bz;
    lW.r += lF.f0 * u + lF.f1 * u * u + lF.f2 * u * v + lF.f3 * u * w;
    lW.u += lF.f0 * r + lF.f1 * T(2) * r * u + lF.f2 * r * v + lF.f3 * r * w + lF.f4 * (E + pt) + lF.f5 * By +
            lF.f6 * Bz;
    lW.v += lF.f2 * r * u - lF.f5 * Bx;
    lW.w += lF.f3 * r * u - lF.f6 * Bx;
    const T lpt = lF.f1 + lF.f4 * u;
    const T lE = lF.f4 * u;
    const T lvdotB = -Bx * lF.f4;
    lW.u += Bx * lvdotB;
    lW.v += By * lvdotB;
    lW.w += Bz * lvdotB;
    lW.P += lpt;
    const T lB2 = T(0.5) * lpt;
    lW.bx += -T(2) * Bx * lF.f1 - By * lF.f2 - Bz * lF.f3 - vdotB * lF.f4 - v * lF.f5 - w * lF.f6 + u * lvdotB +
             T(2) * Bx * lB2;
    lW.by += -Bx * lF.f2 + u * lF.f5 + v * lvdotB + T(2) * By * lB2;
    lW.bz += -Bx * lF.f3 + u * lF.f6 + w * lvdotB + T(2) * Bz * lB2;
    energy_vjp(c, W, lE, lW);
}

// HLLD (M2:372-530), reverse.  lL / lR receive the adjoints of the left and
// right states except their normal B (the forward replaces it by Bn), whose
// adjoint goes to lBn together with Bn's own.
template <class T>
CC_HD void hlld_x_vjp(const M2Const<T>& c, Prim<T> L, Prim<T> R, const T Bn, const Flux<T>& lF, Prim<T>& lL,
                      Prim<T>& lR, T& lBn) {
    L.bx = Bn;
    R.bx = Bn;
    Prim<T> aL = prim_zero<T>(), aR = prim_zero<T>();
    T aBn = T(0), lSL = T(0), lSR = T(0);
    const T cfL = fast_speed(c, L, Bn), cfR = fast_speed(c, R, Bn);
    const T uLm = L.u - cfL, uRm = R.u - cfR, uLp = L.u + cfL, uRp = R.u + cfR;
    const T SL = vmin(uLm, uRm);
    const T SR = vmax(uLp, uRp);

    do {   // one exit: the common tail below runs once, whatever the region
        if (T(0.0) <= SL) { ideal_flux_vjp(c, L, lF, aL); break; }
        if (T(0.0) >= SR) { ideal_flux_vjp(c, R, lF, aR); break; }

        const T EL = energy(c, L), ER = energy(c, R);
        const T ptL = L.P + T(0.5) * (L.bx * L.bx + L.by * L.by + L.bz * L.bz);
        const T ptR = R.P + T(0.5) * (R.bx * R.bx + R.by * R.by + R.bz * R.bz);
        T lEL = T(0), lER = T(0), lptL = T(0), lptR = T(0);

        if (fabs(Bn) < T(1e-12)) {  // HLL (M2:449-467)
            const Flux<T> FL = ideal_flux(c, L), FR = ideal_flux(c, R);
            const T inv = T(1.0) / (SR - SL);
            const T s2 = SL * SR;
            const T fl[7] = {FL.f0, FL.f1, FL.f2, FL.f3, FL.f4, FL.f5, FL.f6};
            const T fr[7] = {FR.f0, FR.f1, FR.f2, FR.f3, FR.f4, FR.f5, FR.f6};
            const T ul[7] = {L.r, L.r * L.u, L.r * L.v, L.r * L.w, EL, L.by, L.bz};
            const T ur[7] = {R.r, R.r * R.u, R.r * R.v, R.r * R.w, ER, R.by, R.bz};
            const T lf[7] = {lF.f0, lF.f1, lF.f2, lF.f3, lF.f4, lF.f5, lF.f6};
            T lfl[7], lfr[7], lul[7], lur[7];
            T linv = T(0), ls2 = T(0);
    #pragma unroll
            for (int k = 0; k < 7; k++) {
                const T num = SR * fl[k] - SL * fr[k] + s2 * (ur[k] - ul[k]);
                const T lnum = lf[k] * inv;
                linv += lf[k] * num;
                lSR += lnum * fl[k];
                lfl[k] = lnum * SR;
                lSL -= lnum * fr[k];
                lfr[k] = -lnum * SL;
                ls2 += lnum * (ur[k] - ul[k]);
                lur[k] = lnum * s2;
                lul[k] = -lnum * s2;
            }
            const T ld = -linv * inv * inv;
            lSR += ld;
            lSL -= ld;
            lSL += ls2 * SR;
            lSR += ls2 * SL;
            Flux<T> g;
            g.f0 = lfl[0]; g.f1 = lfl[1]; g.f2 = lfl[2]; g.f3 = lfl[3]; g.f4 = lfl[4]; g.f5 = lfl[5]; g.f6 = lfl[6];
            ideal_flux_vjp(c, L, g, aL);
            g.f0 = lfr[0]; g.f1 = lfr[1]; g.f2 = lfr[2]; g.f3 = lfr[3]; g.f4 = lfr[4]; g.f5 = lfr[5]; g.f6 = lfr[6];
            ideal_flux_vjp(c, R, g, aR);
            aL.r += lul[0] + lul[1] * L.u + lul[2] * L.v + lul[3] * L.w;
            aL.u += lul[1] * L.r; aL.v += lul[2] * L.r; aL.w += lul[3] * L.r;
            lEL += lul[4]; aL.by += lul[5]; aL.bz += lul[6];
            aR.r += lur[0] + lur[1] * R.u + lur[2] * R.v + lur[3] * R.w;
            aR.u += lur[1] * R.r; aR.v += lur[2] * R.r; aR.w += lur[3] * R.r;
            lER += lur[4]; aR.by += lur[5]; aR.bz += lur[6];
        } else {
            // ---- forward recompute of the star construction (M2:470-529) ----
            const T den = L.r * (SL - L.u) - R.r * (SR - R.u);
            const bool sm_ok = fabs(den) > T(1e-14);
            T SM = T(0.0);
            if (sm_ok) SM = (ptR - ptL + L.r * L.u * (SL - L.u) - R.r * R.u * (SR - R.u)) / den;
            const T rLs = L.r * (SL - L.u) / (SL - SM);
            const T rRs = R.r * (SR - R.u) / (SR - SM);
            const T pts = ptL + L.r * (SL - L.u) * (SM - L.u);
            const T sL = SL - L.u, sR = SR - R.u;
            const T bn2 = Bn * Bn;
            const T dL = L.r * sL * (SL - SM) - bn2;
            const T dR = R.r * sR * (SR - SM) - bn2;
            const bool starL = fabs(dL) > T(1e-14), starR = fabs(dR) > T(1e-14);
            T ByLs = L.by, BzLs = L.bz, ByRs = R.by, BzRs = R.bz;
            T vLs = L.v, wLs = L.w, vRs = R.v, wRs = R.w;
            T numL = T(0), ddL = T(1), numR = T(0), ddR = T(1);
            if (starL) {
                numL = L.r * sL * (SL - L.u) - bn2;
                ByLs = L.by * numL / dL;
                BzLs = L.bz * numL / dL;
                ddL = L.r * (SL - L.u) * (SL - SM);
                vLs = L.v - Bn * (ByLs - L.by) / ddL;
                wLs = L.w - Bn * (BzLs - L.bz) / ddL;
            }
            if (starR) {
                numR = R.r * sR * (SR - R.u) - bn2;
                ByRs = R.by * numR / dR;
                BzRs = R.bz * numR / dR;
                ddR = R.r * (SR - R.u) * (SR - SM);
                vRs = R.v - Bn * (ByRs - R.by) / ddR;
                wRs = R.w - Bn * (BzRs - R.bz) / ddR;
            }
            const T sqL = sqrt(vmax(rLs, tiny_pos<T>()));
            const T sqR = sqrt(vmax(rRs, tiny_pos<T>()));
            const T SLL = SM - fabs(Bn) / sqL;
            const T SRR = SM + fabs(Bn) / sqR;
            const bool left = (T(0.0) < SM);
            const bool outer = left ? (T(0.0) < SLL) : !(T(0.0) < SRR);
            // the upwind side by value; its adjoint is folded into aL or aR after the last use
            const Prim<T> W = prim_select(left, L, R);
            Prim<T> aW = prim_zero<T>();
            const T S = left ? SL : SR;
            const T EW = left ? EL : ER;
            const T ptW = left ? ptL : ptR;
            const T rs = left ? rLs : rRs;
            const T sgn = (Bn >= T(0.0)) ? T(1.0) : T(-1.0);
            const T d2 = sqL + sqR;
            T vs, ws, Bys, Bzs;
            if (outer) {
                vs = left ? vLs : vRs; ws = left ? wLs : wRs;
                Bys = left ? ByLs : ByRs; Bzs = left ? BzLs : BzRs;
            } else {
                vs = (sqL * vLs + sqR * vRs + (ByRs - ByLs) * sgn) / d2;
                ws = (sqL * wLs + sqR * wRs + (BzRs - BzLs) * sgn) / d2;
                Bys = (sqL * ByRs + sqR * ByLs + sqL * sqR * (vRs - vLs) * sgn) / d2;
                Bzs = (sqL * BzRs + sqR * BzLs + sqL * sqR * (wRs - wLs) * sgn) / d2;
            }
            const T vBs = SM * Bn + vs * Bys + ws * Bzs;
            const T vBw = W.u * W.bx + W.v * W.by + W.w * W.bz;
            const T numE = (S - W.u) * EW - (ptW * W.u - Bn * vBw) + (pts * SM - Bn * vBs);
            const T dE = S - SM;
            const T Es = numE / dE;

            // ---- reverse (reciprocals of the recurring denominators computed once) ----
            const T i_d2 = T(1) / d2, i_dE = T(1) / dE;
            const T i_ddL = T(1) / ddL, i_ddR = T(1) / ddR;
            const T i_dL = starL ? T(1) / dL : T(0), i_dR = starR ? T(1) / dR : T(0);
            const T i_sLm = T(1) / (SL - SM), i_sRm = T(1) / (SR - SM);
            ideal_flux_vjp(c, W, lF, aW);
            T lS = lF.f0 * (rs - W.r) + lF.f1 * (rs * SM - W.r * W.u) + lF.f2 * (rs * vs - W.r * W.v) +
                   lF.f3 * (rs * ws - W.r * W.w) + lF.f4 * (Es - EW) + lF.f5 * (Bys - W.by) + lF.f6 * (Bzs - W.bz);
            const T lrs = S * (lF.f0 + lF.f1 * SM + lF.f2 * vs + lF.f3 * ws);
            T lSM = S * lF.f1 * rs;
            T lvs = S * lF.f2 * rs, lws = S * lF.f3 * rs;
            const T lEs = S * lF.f4;
            T lEW = -S * lF.f4;
            T lBys = S * lF.f5, lBzs = S * lF.f6;
            aW.r -= S * (lF.f0 + lF.f1 * W.u + lF.f2 * W.v + lF.f3 * W.w);
            aW.u -= S * lF.f1 * W.r;
            aW.v -= S * lF.f2 * W.r;
            aW.w -= S * lF.f3 * W.r;
            aW.by -= S * lF.f5;
            aW.bz -= S * lF.f6;
            // Es = numE / dE
            const T lnumE = lEs * i_dE;
            const T ldE = -lEs * Es * i_dE;
            lS += ldE;
            lSM -= ldE;
            lS += lnumE * EW;
            aW.u -= lnumE * EW;
            lEW += lnumE * (S - W.u);
            T lptW = -lnumE * W.u;
            aW.u -= lnumE * ptW;
            aBn += lnumE * vBw;
            const T lvBw = lnumE * Bn;
            T lpts = lnumE * SM;
            lSM += lnumE * pts;
            aBn -= lnumE * vBs;
            const T lvBs = -lnumE * Bn;
            // vBw = W.u W.bx + W.v W.by + W.w W.bz   (W.bx = Bn)
            aW.u += lvBw * W.bx; aW.bx += lvBw * W.u;
            aW.v += lvBw * W.by; aW.by += lvBw * W.v;
            aW.w += lvBw * W.bz; aW.bz += lvBw * W.w;
            if (left) prim_acc(aL, aW); else prim_acc(aR, aW);
            // vBs = SM Bn + vs Bys + ws Bzs
            lSM += lvBs * Bn; aBn += lvBs * SM;
            lvs += lvBs * Bys; lBys += lvBs * vs;
            lws += lvBs * Bzs; lBzs += lvBs * ws;
            // side quantities
            if (left) { lEL += lEW; lptL += lptW; lSL += lS; } else { lER += lEW; lptR += lptW; lSR += lS; }
            T lrLs = left ? lrs : T(0), lrRs = left ? T(0) : lrs;
            T lvLs = T(0), lwLs = T(0), lByLs = T(0), lBzLs = T(0), lvRs = T(0), lwRs = T(0), lByRs = T(0), lBzRs = T(0);
            T lsqL = T(0), lsqR = T(0);
            if (outer) {
                if (left) { lvLs += lvs; lwLs += lws; lByLs += lBys; lBzLs += lBzs; }
                else { lvRs += lvs; lwRs += lws; lByRs += lBys; lBzRs += lBzs; }
            } else {
                T ld2 = T(0);
                const T lnv = lvs * i_d2;
                ld2 -= lvs * vs * i_d2;
                lsqL += lnv * vLs; lvLs += lnv * sqL; lsqR += lnv * vRs; lvRs += lnv * sqR;
                lByRs += lnv * sgn; lByLs -= lnv * sgn;
                const T lnw = lws * i_d2;
                ld2 -= lws * ws * i_d2;
                lsqL += lnw * wLs; lwLs += lnw * sqL; lsqR += lnw * wRs; lwRs += lnw * sqR;
                lBzRs += lnw * sgn; lBzLs -= lnw * sgn;
                const T lnby = lBys * i_d2;
                ld2 -= lBys * Bys * i_d2;
                lsqL += lnby * (ByRs + sqR * (vRs - vLs) * sgn);
                lByRs += lnby * sqL;
                lsqR += lnby * (ByLs + sqL * (vRs - vLs) * sgn);
                lByLs += lnby * sqR;
                lvRs += lnby * sqL * sqR * sgn;
                lvLs -= lnby * sqL * sqR * sgn;
                const T lnbz = lBzs * i_d2;
                ld2 -= lBzs * Bzs * i_d2;
                lsqL += lnbz * (BzRs + sqR * (wRs - wLs) * sgn);
                lBzRs += lnbz * sqL;
                lsqR += lnbz * (BzLs + sqL * (wRs - wLs) * sgn);
                lBzLs += lnbz * sqR;
                lwRs += lnbz * sqL * sqR * sgn;
                lwLs -= lnbz * sqL * sqR * sgn;
                lsqL += ld2;
                lsqR += ld2;
            }
            if (!(rLs < tiny_pos<T>()) && sqL > T(0)) lrLs += lsqL / (T(2) * sqL);
            if (!(rRs < tiny_pos<T>()) && sqR > T(0)) lrRs += lsqR / (T(2) * sqR);
            // star states of each side (M2:424-442)
            T ldL = T(0), ldR = T(0), lbn2 = T(0), lsL = T(0), lsR = T(0);
            if (starL) {
                const T tB = (ByLs - L.by), tZ = (BzLs - L.bz);
                aL.v += lvLs;
                aBn -= lvLs * tB * i_ddL;
                lByLs -= lvLs * Bn * i_ddL;
                aL.by += lvLs * Bn * i_ddL;
                T lddL = lvLs * Bn * tB * i_ddL * i_ddL;
                aL.w += lwLs;
                aBn -= lwLs * tZ * i_ddL;
                lBzLs -= lwLs * Bn * i_ddL;
                aL.bz += lwLs * Bn * i_ddL;
                lddL += lwLs * Bn * tZ * i_ddL * i_ddL;
                // ddL = L.r (SL - L.u)(SL - SM)
                aL.r += lddL * sL * (SL - SM);
                lsL += lddL * L.r * (SL - SM);
                lSL += lddL * L.r * sL;
                lSM -= lddL * L.r * sL;
                // ByLs = L.by numL / dL, BzLs = L.bz numL / dL
                const T lnumL = (lByLs * L.by + lBzLs * L.bz) * i_dL;
                aL.by += lByLs * numL * i_dL;
                aL.bz += lBzLs * numL * i_dL;
                ldL -= (lByLs * ByLs + lBzLs * BzLs) * i_dL;
                // numL = L.r sL (SL - L.u) - bn2
                aL.r += lnumL * sL * sL;
                lsL += T(2) * lnumL * L.r * sL;
                lbn2 -= lnumL;
            } else {
                aL.by += lByLs; aL.bz += lBzLs; aL.v += lvLs; aL.w += lwLs;
            }
            if (starR) {
                const T tB = (ByRs - R.by), tZ = (BzRs - R.bz);
                aR.v += lvRs;
                aBn -= lvRs * tB * i_ddR;
                lByRs -= lvRs * Bn * i_ddR;
                aR.by += lvRs * Bn * i_ddR;
                T lddR = lvRs * Bn * tB * i_ddR * i_ddR;
                aR.w += lwRs;
                aBn -= lwRs * tZ * i_ddR;
                lBzRs -= lwRs * Bn * i_ddR;
                aR.bz += lwRs * Bn * i_ddR;
                lddR += lwRs * Bn * tZ * i_ddR * i_ddR;
                aR.r += lddR * sR * (SR - SM);
                lsR += lddR * R.r * (SR - SM);
                lSR += lddR * R.r * sR;
                lSM -= lddR * R.r * sR;
                const T lnumR = (lByRs * R.by + lBzRs * R.bz) * i_dR;
                aR.by += lByRs * numR * i_dR;
                aR.bz += lBzRs * numR * i_dR;
                ldR -= (lByRs * ByRs + lBzRs * BzRs) * i_dR;
                aR.r += lnumR * sR * sR;
                lsR += T(2) * lnumR * R.r * sR;
                lbn2 -= lnumR;
            } else {
                aR.by += lByRs; aR.bz += lBzRs; aR.v += lvRs; aR.w += lwRs;
            }
            // dL = L.r sL (SL - SM) - bn2 (only differentiated where it was used)
            if (starL) {
                aL.r += ldL * sL * (SL - SM);
                lsL += ldL * L.r * (SL - SM);
                lSL += ldL * L.r * sL;
                lSM -= ldL * L.r * sL;
                lbn2 -= ldL;
            }
            if (starR) {
                aR.r += ldR * sR * (SR - SM);
                lsR += ldR * R.r * (SR - SM);
                lSR += ldR * R.r * sR;
                lSM -= ldR * R.r * sR;
                lbn2 -= ldR;
            }
            aBn += T(2) * Bn * lbn2;
            // pts = ptL + L.r (SL - L.u)(SM - L.u)
            lptL += lpts;
            aL.r += lpts * sL * (SM - L.u);
            lSL += lpts * L.r * (SM - L.u);
            lSM += lpts * L.r * sL;
            aL.u -= lpts * L.r * ((SM - L.u) + sL);
            // rLs = L.r (SL - L.u) / (SL - SM), rRs likewise
            {
                const T lq = lrLs * i_sLm;
                const T lden = -lrLs * rLs * i_sLm;
                lSL += lden; lSM -= lden;
                aL.r += lq * sL; lSL += lq * L.r; aL.u -= lq * L.r;
            }
            {
                const T lq = lrRs * i_sRm;
                const T lden = -lrRs * rRs * i_sRm;
                lSR += lden; lSM -= lden;
                aR.r += lq * sR; lSR += lq * R.r; aR.u -= lq * R.r;
            }
            // sL = SL - L.u, sR = SR - R.u
            lSL += lsL; aL.u -= lsL;
            lSR += lsR; aR.u -= lsR;
            // SM = numSM / den
            if (sm_ok) {
                const T i_den = T(1) / den;
                const T lnum = lSM * i_den;
                const T lden = -lSM * SM * i_den;
                lptR += lnum;
                lptL -= lnum;
                aL.r += lnum * L.u * sL;
                aL.u += lnum * L.r * (sL - L.u);
                lSL += lnum * L.r * L.u;
                aR.r -= lnum * R.u * sR;
                aR.u -= lnum * R.r * (sR - R.u);
                lSR -= lnum * R.r * R.u;
                aL.r += lden * sL; lSL += lden * L.r; aL.u -= lden * L.r;
                aR.r -= lden * sR; lSR -= lden * R.r; aR.u += lden * R.r;
            }
        }
        energy_vjp(c, L, lEL, aL);
        energy_vjp(c, R, lER, aR);
        aL.P += lptL; aL.bx += lptL * L.bx; aL.by += lptL * L.by; aL.bz += lptL * L.bz;
        aR.P += lptR; aR.bx += lptR * R.bx; aR.by += lptR * R.by; aR.bz += lptR * R.bz;
    } while (false);
    T lcfL = T(0), lcfR = T(0);
    if (uRm < uLm) { aR.u += lSL; lcfR -= lSL; } else { aL.u += lSL; lcfL -= lSL; }
    if (uLp < uRp) { aR.u += lSR; lcfR += lSR; } else { aL.u += lSR; lcfL += lSR; }
    fast_speed_vjp(c, L, Bn, lcfL, aL, aBn);
    fast_speed_vjp(c, R, Bn, lcfR, aR, aBn);
    aBn += aL.bx + aR.bx;
    lL.r += aL.r; lL.u += aL.u; lL.v += aL.v; lL.w += aL.w; lL.P += aL.P; lL.by += aL.by; lL.bz += aL.bz;
    lR.r += aR.r; lR.u += aR.u; lR.v += aR.v; lR.w += aR.w; lR.P += aR.P; lR.by += aR.by; lR.bz += aR.bz;
    lBn += aBn;
}

// y-normal HLLD through the (u,v)/(Bx,By) swap (M2:540-561), reverse
template <class T>
CC_HD void hlld_y_vjp(const M2Const<T>& c, const Prim<T>& L, const Prim<T>& R, const T Bn, const Flux<T>& lF,
                      Prim<T>& lL, Prim<T>& lR, T& lBn) {
    Prim<T> aL, aR;
    aL.r = L.r; aL.u = L.v; aL.v = L.u; aL.w = L.w; aL.P = L.P; aL.bx = Bn; aL.by = L.bx; aL.bz = L.bz;
    aR.r = R.r; aR.u = R.v; aR.v = R.u; aR.w = R.w; aR.P = R.P; aR.bx = Bn; aR.by = R.bx; aR.bz = R.bz;
    Flux<T> g = lF;
    g.f1 = lF.f2;
    g.f2 = lF.f1;
    Prim<T> laL = prim_zero<T>(), laR = prim_zero<T>();
    hlld_x_vjp(c, aL, aR, Bn, g, laL, laR, lBn);
    lL.r += laL.r; lL.v += laL.u; lL.u += laL.v; lL.w += laL.w; lL.P += laL.P; lL.bx += laL.by; lL.bz += laL.bz;
    lR.r += laR.r; lR.v += laR.u; lR.u += laR.v; lR.w += laR.w; lR.P += laR.P; lR.bx += laR.by; lR.bz += laR.bz;
}

// MC slope (M2:106-112, 295), reverse
template <class T>
CC_HD void mc_slope_vjp(T wm, T wc, T wp, T ls, T& lm, T& lc, T& lp) {
    const T dm = wc - wm, dp = wp - wc;
    const T a = T(0.5) * (dm + dp);
    const T x = T(2.0) * dm, y = T(2.0) * dp;
    int bsel;
    T b;
    if (x * y <= T(0.0)) { b = T(0.0); bsel = 0; }
    else if (fabs(x) < fabs(y)) { b = x; bsel = 1; }
    else { b = y; bsel = 2; }
    T la = T(0), lb = T(0);
    if (!(a * b <= T(0.0))) {
        if (fabs(a) < fabs(b)) la = ls;
        else lb = ls;
    }
    T ldm = T(0.5) * la, ldp = T(0.5) * la;
    if (bsel == 1) ldm += T(2.0) * lb;
    else if (bsel == 2) ldp += T(2.0) * lb;
    lc += ldm - ldp;
    lm -= ldm;
    lp += ldp;
}

// cons_to_prim (M2:126-135), reverse: lW -> (lrho, lmx, lmy, lmz, lE, lBx, lBy, lBz)
template <class T>
CC_HD void to_prim_vjp(const M2Const<T>& c, T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz, const Prim<T>& lW,
                       T& lrho, T& lmx, T& lmy, T& lmz, T& lE, T& lBx, T& lBy, T& lBz) {
    const T rf = vmax(rho, c.floor_rho);
    const T u = mx / rf, v = my / rf, w = mz / rf;
    const T kin = T(0.5) * rf * (u * u + v * v + w * w);
    const T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    const T P0 = c.gm1 * (E - kin - mag);
    const T lP0 = (P0 < c.floor_P) ? T(0) : lW.P;
    lE += c.gm1 * lP0;
    const T lkin = -c.gm1 * lP0, lmag = -c.gm1 * lP0;
    lBx += lmag * Bx + lW.bx;
    lBy += lmag * By + lW.by;
    lBz += lmag * Bz + lW.bz;
    T lrf = lkin * T(0.5) * (u * u + v * v + w * w) + lW.r;
    const T lu = lkin * rf * u + lW.u, lv = lkin * rf * v + lW.v, lw = lkin * rf * w + lW.w;
    lmx += lu / rf; lmy += lv / rf; lmz += lw / rf;
    lrf -= (lu * u + lv * v + lw * w) / rf;
    if (!(rho < c.floor_rho)) lrho += lrf;
}

// enforce_floors (M2:114-124), reverse, in place: on entry l* are the
// adjoints of the floored outputs (rho, E changed; the rest pass through),
// on exit the adjoints of the inputs.
template <class T>
CC_HD void floors_vjp(const M2Const<T>& c, T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz, T& lrho, T& lmx,
                      T& lmy, T& lmz, T& lE, T& lBx, T& lBy, T& lBz) {
    const T rf = vmax(rho, c.floor_rho);
    const T u = mx / rf, v = my / rf, w = mz / rf;
    const T kin = T(0.5) * rf * (u * u + v * v + w * w);
    const T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    const T P = c.gm1 * (E - kin - mag);
    T lrf = lrho;
    if (P < c.floor_P) {
        const T lkin = lE, lmag = lE;
        lE = T(0);
        lBx += lmag * Bx; lBy += lmag * By; lBz += lmag * Bz;
        lrf += lkin * T(0.5) * (u * u + v * v + w * w);
        const T lu = lkin * rf * u, lv = lkin * rf * v, lw = lkin * rf * w;
        lmx += lu / rf; lmy += lv / rf; lmz += lw / rf;
        lrf -= (lu * u + lv * v + lw * w) / rf;
    }
    lrho = (rho < c.floor_rho) ? T(0) : lrf;
}

// Joule heating, Bz diffusion and floors of one cell (M2:631-686), reverse.
// Forward inputs: own (rho..Bz) and cell-centred (Bx, By) of the stored
// state s, neighbour Bz (E W N S) and the face values used by Jz (byE =
// by(j, iE), byC = by(j, i), bxN = bx(jN, i), bxC = bx(j, i)).  joule_vjp
// turns the adjoints of the outputs (l[6] = rho mx my mz E Bz, in place) into
// those of the own values, and adds those of the neighbour Bz, the face
// values, the cell-centred Bx, By and eta.
template <class T>
struct JouleIn {
    T rho, mx, my, mz, E, Bz, Bx, By;
    T bzE, bzW, bzN, bzS;
    T byE, byC, bxN, bxC;
};
template <class T>
struct JouleAdj {
    T l[6];
    T bzE, bzW, bzN, bzS, byE, byC, bxN, bxC, Bx, By, eta;
};

template <class T>
CC_HD void joule_vjp(const M2Const<T>& c, T dt, const JouleIn<T>& in, JouleAdj<T>& a) {
    const T dBzdy = (in.bzN - in.bzS) / c.two_dy;
    const T dBzdx = (in.bzE - in.bzW) / c.two_dx;
    const T dBydx = (in.byE - in.byC) / c.dx;
    const T dBxdy = (in.bxN - in.bxC) / c.dy;
    const T Jx = dBzdy, Jy = -dBzdx, Jz = dBydx - dBxdy;
    const T J2 = Jx * Jx + Jy * Jy + Jz * Jz;
    const T E1 = in.E + dt * c.eta * J2;
    const T lap = (in.bzE - T(2) * in.Bz + in.bzW) * c.idx2 + (in.bzN - T(2) * in.Bz + in.bzS) * c.idy2;
    const T Bz1 = in.Bz + dt * c.eta * lap;
    T lrho = a.l[0], lmx = a.l[1], lmy = a.l[2], lmz = a.l[3], lE1 = a.l[4], lBz1 = a.l[5];
    T lBx = T(0), lBy = T(0);
    floors_vjp(c, in.rho, in.mx, in.my, in.mz, E1, in.Bx, in.By, Bz1, lrho, lmx, lmy, lmz, lE1, lBx, lBy, lBz1);
    a.Bx += lBx;
    a.By += lBy;
    // Bz1 = Bz + dt eta lap
    const T llap = dt * c.eta * lBz1;
    a.eta += dt * lap * lBz1;
    T lBz = lBz1;
    a.bzE += c.idx2 * llap;
    a.bzW += c.idx2 * llap;
    lBz -= T(2) * (c.idx2 + c.idy2) * llap;
    a.bzN += c.idy2 * llap;
    a.bzS += c.idy2 * llap;
    // E1 = E + dt eta J2
    const T lJ2 = dt * c.eta * lE1;
    a.eta += dt * J2 * lE1;
    const T lJx = T(2) * Jx * lJ2, lJy = T(2) * Jy * lJ2, lJz = T(2) * Jz * lJ2;
    a.bzN += lJx / c.two_dy;
    a.bzS -= lJx / c.two_dy;
    a.bzE -= lJy / c.two_dx;
    a.bzW += lJy / c.two_dx;
    a.byE += lJz / c.dx;
    a.byC -= lJz / c.dx;
    a.bxN -= lJz / c.dy;
    a.bxC += lJz / c.dy;
    a.l[0] = lrho; a.l[1] = lmx; a.l[2] = lmy; a.l[3] = lmz; a.l[4] = lE1; a.l[5] = lBz;
}

}  // namespace ccb
