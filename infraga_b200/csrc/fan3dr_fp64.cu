// FP64 ray-fan kernel: 3D Cartesian geometry, range-dependent atmosphere
// (hybrid 3D splines over an x/y node grid in km), flat ground or terrain.
//
// Same execution scheme and table layouts as the spherical range-dependent
// kernel (fansphr_fp64.cu).  Physics: the reference's 3D range-dependent
// equation set (src/geoac/geoac.eqset.3d.rngdep.cpp) with
// atmo_state.3d.rngdep.cpp (no boundary-layer vertical wind), the RK4 driver
// (src/util/rk4solver.cpp:14-85) and run_prop
// (src/main.infraga.3d.rngdep.cpp:204-535).  Two reference details carried
// over: without terrain topo::z is 0 (not z_grnd, atmo_state.3d.rngdep.cpp:45-51),
// and the azimuth variation of v is added into dv[3] (eqset.3d.rngdep.cpp:288).
//
// ST instantiations run infraga-3d's stratified profile over terrain
// (topo_file=): c, u, v, rho from the 1D knot table at the clamped altitude
// (atmo_state.3d.strat.cpp:148-233, calc_uvw :462-734) with the same terrain,
// boundary-layer scaling, reflection and bounce loop (geoac.eqset.3d.strat.cpp
// and run_prop, main.infraga.3d.cpp:199-357, have the same forms).  Their
// differences from the range-dependent solver are kept: the Hessian-times-
// Jacobian sums of update_refs run over m >= n only (eqset.3d.strat.cpp:305-310)
// and the turning height starts from topo::z0, the profile's first altitude
// (main.infraga.3d.cpp:427).
#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fan3d_common.cuh"
#include "rngdep_eval.cuh"

namespace iga {

namespace {

#ifndef IGA_3DR_THREADS
#define IGA_3DR_THREADS 128
#endif
#ifndef IGA_3DR_MINB
#define IGA_3DR_MINB 1
#endif
constexpr int kThreads = IGA_3DR_THREADS;

template <bool AMP> struct Dim3r { static constexpr int n = AMP ? 18 : 6; };

struct Cells {
    int hx, hy, hz, tx, ty;
};

struct Views {
    HybView hyb;
    TopoView topo;
    bool has_topo;
};

// hybrid index (0 = z, 1 = x, 2 = y) of Cartesian component i (0 = x, 1 = y, 2 = z)
__device__ __forceinline__ int hix(int i) { return i == 2 ? 0 : i + 1; }

// topo::z (atmo_state.3d.rngdep.cpp:45-51): terrain height, or 0 without terrain
__device__ __forceinline__ double topo_z(const Views& v, Cells& cl, double x, double y) {
    if (!v.has_topo) return 0.0;
    TopoVal t;
    topo_eval(v.topo, x, y, 0, t, cl.tx, cl.ty);
    return t.z;
}

// sum_{k >= i} X[k] H[k], accumulated from k = i like the reference's loop
__device__ __forceinline__ double hsum_from(int i, const double* X, const double* H) {
    return i == 0 ? X[0] * H[0] + X[1] * H[1] + X[2] * H[2] : (i == 1 ? X[1] * H[1] + X[2] * H[2] : X[2] * H[2]);
}

struct AtmFull {
    double c, dc[3], ddc[3][3];
    double u, du[3], ddu[3][3];
    double v, dv[3], ddv[3][3];
};

// Stratified profile row at z clamped to the knot range (interp::in_interval);
// cl.hz caches the segment.
__device__ __forceinline__ const double* strat_at(const Fan3DArgs& a, Cells& cl, double z, Cubic& q) {
    const double ze = fmin(fmax(z, a.z_lo), a.z_hi);
    cl.hz = seg_walk(a.knots, a.n_knots, ze, cl.hz);
    const double* r0 = a.knots + cl.hz * kStride;
    q = cubic_at(r0, ze);
    return r0;
}

// update_refs' atmosphere (atmo::c/dc/ddc and calc_uvw, atmo_state.3d.rngdep.cpp:148-170, 400-700;
// ST: atmo_state.3d.strat.cpp:148-233, 462-734)
template <bool AMP, bool ST>
__device__ __forceinline__ void atm_full(const Fan3DArgs& a, const Views& vw, Cells& cl, double x, double y, double z,
                                         AtmFull& m) {
    HybF2 c2 = {}, u2 = {}, v2 = {};   // hybrid index order: d[0] is d/dz
    if (ST) {
        Cubic q;
        const double* r0 = strat_at(a, cl, z, q);
        if (AMP) {
            cubic_f2(r0, q, 2, c2.f, c2.d[0], c2.dd[0][0]);
            cubic_f2(r0, q, 4, u2.f, u2.d[0], u2.dd[0][0]);
            cubic_f2(r0, q, 6, v2.f, v2.d[0], v2.dd[0][0]);
        } else {
            cubic_f1(r0, q, 2, c2.f, c2.d[0]);
            cubic_f1(r0, q, 4, u2.f, u2.d[0]);
            cubic_f1(r0, q, 6, v2.f, v2.d[0]);
        }
    } else {
    HybLoc L;
    hyb_locate(vw.hyb, x, y, z, L, cl.hx, cl.hy, cl.hz);
    L.zq_raw = L.zq;   // the Cartesian calls pass the clamped z to every block
    if (AMP) {
        hyb_f2(vw.hyb, L, 0, c2);
        hyb_f2(vw.hyb, L, 1, u2);
        hyb_f2(vw.hyb, L, 2, v2);
    } else {
        HybF1 t;
        hyb_f1(vw.hyb, L, 0, t); c2.f = t.f; c2.d[0] = t.d[0]; c2.d[1] = t.d[1]; c2.d[2] = t.d[2];
        hyb_f1(vw.hyb, L, 1, t); u2.f = t.f; u2.d[0] = t.d[0]; u2.d[1] = t.d[1]; u2.d[2] = t.d[2];
        hyb_f1(vw.hyb, L, 2, t); v2.f = t.f; v2.d[0] = t.d[0]; v2.d[1] = t.d[1]; v2.d[2] = t.d[2];
    }
    }
    double zg = 0.0, dzg[2] = {0.0, 0.0}, ddzg[3] = {0.0, 0.0, 0.0};
    double X = 0.0;
    if (z < a.x_cut) {
        if (vw.has_topo) {
            TopoVal t;
            const bool in_bl = z < a.z_bl;
            topo_eval(vw.topo, x, y, in_bl ? (AMP ? 2 : 1) : 0, t, cl.tx, cl.ty);
            zg = t.z;
            if (in_bl) {
                dzg[0] = t.d[0]; dzg[1] = t.d[1];
                if (AMP) { ddzg[0] = t.dd[0]; ddzg[1] = t.dd[1]; ddzg[2] = t.dd[2]; }
            }
        }
        X = exp(-(z - zg) * a.inv_bl);
    }
    const double ib = a.inv_bl, ib2 = ib * ib;
    const double dX[3] = {X * ib * dzg[0], X * ib * dzg[1], -X * ib};
    const double iop = 1.0 / (1.0 + X), iop2 = iop * iop, iop3 = iop2 * iop;
    const double sc0 = (1.0 - X) * iop;
    double dsc[3];
#pragma unroll
    for (int n = 0; n < 3; n++) dsc[n] = -2.0 * dX[n] * iop2;
    m.c = c2.f; m.u = u2.f * sc0; m.v = v2.f * sc0;
#pragma unroll
    for (int n = 0; n < 3; n++) {
        const int h = hix(n);
        m.dc[n] = c2.d[h];
        m.du[n] = u2.d[h] * sc0 + u2.f * dsc[n];
        m.dv[n] = v2.d[h] * sc0 + v2.f * dsc[n];
    }
    if (AMP) {
        double ddX[3][3];
        ddX[0][0] = X * ib * (ddzg[0] + dzg[0] * dzg[0] * ib);
        ddX[0][1] = ddX[1][0] = X * ib * (ddzg[1] + dzg[0] * dzg[1] * ib);
        ddX[1][1] = X * ib * (ddzg[2] + dzg[1] * dzg[1] * ib);
        ddX[0][2] = ddX[2][0] = -X * ib2 * dzg[0];
        ddX[1][2] = ddX[2][1] = -X * ib2 * dzg[1];
        ddX[2][2] = X * ib2;
#pragma unroll
        for (int n = 0; n < 3; n++) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int hn = hix(n), hk = hix(k);
                const double dds = -2.0 * (ddX[n][k] * iop2 - 2.0 * dX[n] * dX[k] * iop3);
                m.ddc[n][k] = c2.dd[hn][hk];
                m.ddu[n][k] = u2.dd[hn][hk] * sc0 + u2.d[hn] * dsc[k] + u2.d[hk] * dsc[n] + u2.f * dds;
                m.ddv[n][k] = v2.dd[hn][hk] * sc0 + v2.d[hn] * dsc[k] + v2.d[hk] * dsc[n] + v2.f * dds;
            }
        }
    }
}

// update_refs + eval_src_eq (geoac.eqset.3d.rngdep.cpp:226-388; ST: eqset.3d.strat.cpp:225-389), w = 0
template <bool AMP, bool ST>
__device__ __forceinline__ void rhs_3dr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y, double* f) {
    AtmFull m;
    atm_full<AMP, ST>(a, vw, cl, y[0], y[1], y[2], m);
    const double n0 = y[3], n1 = y[4], n2 = y[5];
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double inum = 1.0 / num;
    const double cg[3] = {m.c * n0 * inum + m.u, m.c * n1 * inum + m.v, m.c * n2 * inum};
    const double cgm = sqrt(cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2]);
    const double icg = 1.0 / cgm;
    double K[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        K[i] = num * m.dc[i] + n0 * m.du[i] + n1 * m.dv[i];
        f[i] = cg[i] * icg;
        f[3 + i] = -icg * K[i];
    }
    if (AMP) {
        const double icg2 = icg * icg;
        const double cin = m.c * inum, cin2 = cin * inum;
        const double* Xt = y + 6;
        const double* Xp = y + 12;
        // dv[3] collects both variations, dv[4] stays 0 (eqset.3d.rngdep.cpp:288)
        double dv_t = 0.0;
#pragma unroll
        for (int n = 0; n < 3; n++) { dv_t += Xt[n] * m.dv[n]; dv_t += Xp[n] * m.dv[n]; }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const double* Xv = y + 6 + 6 * j;
            const double* mu = y + 9 + 6 * j;
            const double dc = Xv[0] * m.dc[0] + Xv[1] * m.dc[1] + Xv[2] * m.dc[2];
            const double du = Xv[0] * m.du[0] + Xv[1] * m.du[1] + Xv[2] * m.du[2];
            const double dv = j == 0 ? dv_t : 0.0;
            const double dnu = (n0 * mu[0] + n1 * mu[1] + n2 * mu[2]) * inum;
            const double g[3] = {n0 * inum * dc + cin * mu[0] - cin2 * n0 * dnu + du,
                                 n1 * inum * dc + cin * mu[1] - cin2 * n1 * dnu + dv,
                                 n2 * inum * dc + cin * mu[2] - cin2 * n2 * dnu};
            const double dm = (cg[0] * g[0] + cg[1] * g[1] + cg[2] * g[2]) * icg;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                // ST: the stratified update_refs sums m = i..2 only (eqset.3d.strat.cpp:305-310)
                const double ddc = ST ? hsum_from(i, Xv, m.ddc[i]) : Xv[0] * m.ddc[i][0] + Xv[1] * m.ddc[i][1] + Xv[2] * m.ddc[i][2];
                const double ddu = ST ? hsum_from(i, Xv, m.ddu[i]) : Xv[0] * m.ddu[i][0] + Xv[1] * m.ddu[i][1] + Xv[2] * m.ddu[i][2];
                const double ddv = ST ? hsum_from(i, Xv, m.ddv[i]) : Xv[0] * m.ddv[i][0] + Xv[1] * m.ddv[i][1] + Xv[2] * m.ddv[i][2];
                f[6 + 6 * j + i] = g[i] * icg - cg[i] * icg2 * dm;
                f[9 + 6 * j + i] = icg2 * dm * K[i] -
                                   icg * (dnu * m.dc[i] + num * ddc + mu[0] * m.du[i] + mu[1] * m.dv[i] + n0 * ddu + n1 * ddv);
            }
        }
    }
}

// atmo::c/u/v/rho at a point (u, v scaled by bndlyr_sc below z_bndlyr)
struct AtmPt {
    double c, u, v, rho;
};
template <bool ST>
__device__ __forceinline__ void atm_point(const Fan3DArgs& a, const Views& vw, Cells& cl, double x, double y, double z,
                                          AtmPt& o) {
    double sc = 1.0;
    if (z < a.z_bl) {
        const double X = exp(-(z - topo_z(vw, cl, x, y)) * a.inv_bl);
        sc = (1.0 - X) / (1.0 + X);
    }
    if (ST) {
        Cubic q;
        const double* r0 = strat_at(a, cl, z, q);
        o.c = cubic_f(r0, q, 2);
        o.u = cubic_f(r0, q, 4) * sc;
        o.v = cubic_f(r0, q, 6) * sc;
        o.rho = cubic_f(r0, q, 8);
        return;
    }
    HybLoc L;
    hyb_locate(vw.hyb, x, y, z, L, cl.hx, cl.hy, cl.hz);
    o.c = hyb_f(vw.hyb, L, 0);
    o.u = hyb_f(vw.hyb, L, 1) * sc;
    o.v = hyb_f(vw.hyb, L, 2) * sc;
    o.rho = hyb_f(vw.hyb, L, 3);
}

// travel_time / atten of one segment at its midpoint (eqset.3d.rngdep.cpp:487-514, 689-702)
template <bool ST>
__device__ __forceinline__ void seg_increment_3dr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y0,
                                                  const double* y1, double& dt_out, double& da_out) {
    const double dx = y1[0] - y0[0], dy = y1[1] - y0[1], dz = y1[2] - y0[2];
    const double xm = y0[0] + dx * 0.5, ym = y0[1] + dy * 0.5, zm = y0[2] + dz * 0.5;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double n0 = y0[3] + (y1[3] - y0[3]) * 0.5;
    const double n1 = y0[4] + (y1[4] - y0[4]) * 0.5;
    const double n2 = y0[5] + (y1[5] - y0[5]) * 0.5;
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    AtmPt m;
    atm_point<ST>(a, vw, cl, xm, ym, zm, m);
    const double inum = 1.0 / num;
    const double c0 = m.c * n0 * inum + m.u, c1 = m.c * n1 * inum + m.v, c2 = m.c * n2 * inum;
    dt_out = ds / sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    da_out = sb_alpha_cart(m.c, m.rho, zm, a.freq, a.tweak_abs, a.sb) * ds;
}

// travel_time_var of one segment (geoac.eqset.3d.rngdep.cpp:595-660, the
// (tt, .., k1, k2) form run_back_proj calls): the inclination / azimuth
// variations of the travel time at the segment midpoint, with atmo::c, dc, u,
// du, v, dv as atmo_state.3d.rngdep.cpp:148-230 return them (the
// boundary-layer scaling only below z_bndlyr, topo::bndlyr_sc / bndlyr_dsc
// :83-103), w = 0.  Kept with the reference's sign (the sums are decremented)
// and its product in the dot product (dcg[1] * cg[1] * dcg[2] * cg[2]).
template <bool ST>
__device__ __forceinline__ void seg_time_var_3dr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y0,
                                                 const double* y1, double& dvar_t, double& dvar_p) {
    const double dx = y1[0] - y0[0], dy = y1[1] - y0[1], dz = y1[2] - y0[2];
    const double xm = y0[0] + dx / 2.0, ym = y0[1] + dy / 2.0, zm = y0[2] + dz / 2.0;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    double nu[3];
#pragma unroll
    for (int i = 0; i < 3; i++) nu[i] = y0[3 + i] + (y1[3 + i] - y0[3 + i]) / 2.0;
    const double num = sqrt(nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2]);
    // c, u, v and their x, y, z derivatives before the boundary-layer scaling
    double c, dc[3], u, du[3], v, dv[3];
    if (ST) {
        Cubic q;
        const double* r0 = strat_at(a, cl, zm, q);
        cubic_f1(r0, q, 2, c, dc[2]);
        cubic_f1(r0, q, 4, u, du[2]);
        cubic_f1(r0, q, 6, v, dv[2]);
        dc[0] = dc[1] = du[0] = du[1] = dv[0] = dv[1] = 0.0;
    } else {
        HybLoc L;
        hyb_locate(vw.hyb, xm, ym, zm, L, cl.hx, cl.hy, cl.hz);
        L.zq_raw = L.zq;
        HybF1 t;
        hyb_f1(vw.hyb, L, 0, t); c = t.f;
#pragma unroll
        for (int n = 0; n < 3; n++) dc[n] = t.d[hix(n)];
        hyb_f1(vw.hyb, L, 1, t); u = t.f;
#pragma unroll
        for (int n = 0; n < 3; n++) du[n] = t.d[hix(n)];
        hyb_f1(vw.hyb, L, 2, t); v = t.f;
#pragma unroll
        for (int n = 0; n < 3; n++) dv[n] = t.d[hix(n)];
    }
    double sc = 1.0, dsc[3] = {0.0, 0.0, 0.0};
    if (zm < a.z_bl) {
        double zg = 0.0, dzg[2] = {0.0, 0.0};
        if (vw.has_topo) {
            TopoVal tv;
            topo_eval(vw.topo, xm, ym, 1, tv, cl.tx, cl.ty);
            zg = tv.z; dzg[0] = tv.d[0]; dzg[1] = tv.d[1];
        }
        const double X = exp(-(zm - zg) * a.inv_bl);
        sc = (1.0 - X) / (1.0 + X);
        const double dX[3] = {X * a.inv_bl * dzg[0], X * a.inv_bl * dzg[1], -X * a.inv_bl};
#pragma unroll
        for (int n = 0; n < 3; n++) dsc[n] = -2.0 * dX[n] / ((1.0 + X) * (1.0 + X));
    }
#pragma unroll
    for (int n = 0; n < 3; n++) {
        du[n] = du[n] * sc + u * dsc[n];
        dv[n] = dv[n] * sc + v * dsc[n];
    }
    const double cg[3] = {c * nu[0] / num + u * sc, c * nu[1] / num + v * sc, c * nu[2] / num};
    const double cgm = sqrt(cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2]);
    const double den = cgm * cgm * cgm;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int o = 6 * j;   // X at 6..8 / 12..14, mu at 9..11 / 15..17
        double X[3], mu[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            X[i] = y0[6 + o + i] + (y1[6 + o + i] - y0[6 + o + i]) / 2.0;
            mu[i] = y0[9 + o + i] + (y1[9 + o + i] - y0[9 + o + i]) / 2.0;
        }
        double s = X[0] * dc[0];
        s += X[1] * dc[1];
        s += X[2] * dc[2];
        s -= c / (num * num) * (mu[0] * nu[0] + mu[1] * nu[1] + mu[2] * nu[2]);
        double dcg[3];
#pragma unroll
        for (int i = 0; i < 3; i++) dcg[i] = nu[i] / num * s + c / num * mu[i];
        dcg[0] += X[0] * du[0] + X[1] * du[1] + X[2] * du[2];
        dcg[1] += X[0] * dv[0] + X[1] * dv[1] + X[2] * dv[2];
        const double var = -((dcg[0] * cg[0] + dcg[1] * cg[1] * dcg[2] * cg[2]) / den * ds);
        if (j == 0) dvar_t = var; else dvar_p = var;
    }
}

// geoac::amp with geoac::jacobian at the below-ground row (eqset.3d.rngdep.cpp:704-748)
template <bool ST>
__device__ __noinline__ double amp_db_3dr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y, double theta,
                                          double phi, double* jac_out) {
    AtmPt m;
    atm_point<ST>(a, vw, cl, y[0], y[1], y[2], m);
    const double num = sqrt(y[3] * y[3] + y[4] * y[4] + y[5] * y[5]);
    const double num0 = 1.0 - (y[3] * a.u0s + y[4] * a.v0s + y[5] * 0.0) / a.c0;
    const double cp[3] = {m.c * y[3] / num + m.u, m.c * y[4] / num + m.v, m.c * y[5] / num};
    const double ct = cos(theta), st = sin(theta);
    const double g0 = a.c0 * ct * cos(phi) + a.u0s, g1 = a.c0 * ct * sin(phi) + a.v0s, g2 = a.c0 * st;
    const double cpm = sqrt(cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2]);
    const double cpm0 = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
    const double ex = cp[0] / cpm, ey = cp[1] / cpm, ez = cp[2] / cpm;
    const double* Xt = y + 6;
    const double* Xp = y + 12;
    const double jac = ex * (Xt[1] * Xp[2] - Xp[1] * Xt[2]) - Xt[0] * (ey * Xp[2] - ez * Xp[1]) + Xp[0] * (ey * Xt[2] - ez * Xt[1]);
    const double numr = m.rho * num * (m.c * m.c * m.c) * cpm0 * ct;
    const double den = a.rho0 * num0 * (a.c0 * a.c0 * a.c0) * cpm * jac;
    if (jac_out) *jac_out = jac;
    return 20.0 * log10(sqrt(fabs(numr / den)));
}

// approx_intercept + set_refl (eqset.3d.rngdep.cpp:111-209), general terrain
template <int N, bool AMP, bool ST>
__device__ __noinline__ void reflect_3dr(const Fan3DArgs& a, const Views& vw, Cells& cl, double* y, const double* prev) {
    double zy = 0.0, dzy[2] = {0.0, 0.0};
    if (vw.has_topo) {
        TopoVal t;
        topo_eval(vw.topo, y[0], y[1], 1, t, cl.tx, cl.ty);
        zy = t.z; dzy[0] = t.d[0]; dzy[1] = t.d[1];
    }
    const double dz_grnd = zy - y[2];
    const double dz_k = (y[2] - prev[2 * blockDim.x]) - (y[0] - prev[0]) * dzy[0] - (y[1] - prev[1 * blockDim.x]) * dzy[1];
    double p[N];
#pragma unroll
    for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * blockDim.x]) / dz_k * dz_grnd;

    double zg = 0.0, A = 0.0, B = 0.0, zxx = 0.0, zxy = 0.0, zyy = 0.0;
    if (vw.has_topo) {
        TopoVal t;
        topo_eval(vw.topo, p[0], p[1], AMP ? 2 : 1, t, cl.tx, cl.ty);
        zg = t.z; A = t.d[0]; B = t.d[1];
        if (AMP) { zxx = t.dd[0]; zxy = t.dd[1]; zyy = t.dd[2]; }
    }
    const double norm1 = 1.0 + A * A + B * B;
    const double C1x = (1.0 - A * A + B * B) / norm1, C2x = 2.0 * A / norm1;
    const double C1y = (1.0 + A * A - B * B) / norm1, C2y = 2.0 * B / norm1;
    const double C1z = (1.0 - A * A - B * B) / norm1;
    double q[N];
    q[0] = p[0]; q[1] = p[1]; q[2] = zg;
    q[3] = C1x * p[3] + C2x * (p[5] - p[4] * B);
    q[4] = C1y * p[4] + C2y * (p[5] - p[3] * A);
    q[5] = -C1z * p[5] + p[3] * C2x + p[4] * C2y;
    if (AMP) {
        HybF1 cc = {}, uu = {}, vv = {};
        if (ST) {   // atmo::c, dc, du, dv at the ground point (atmo_state.3d.strat.cpp:153-218)
            Cubic qz;
            const double* r0 = strat_at(a, cl, zg, qz);
            cubic_f1(r0, qz, 2, cc.f, cc.d[0]);
            cubic_f1(r0, qz, 4, uu.f, uu.d[0]);
            cubic_f1(r0, qz, 6, vv.f, vv.d[0]);
        } else {
            HybLoc L;
            hyb_locate(vw.hyb, p[0], p[1], zg, L, cl.hx, cl.hy, cl.hz);
            L.zq_raw = L.zq;
            hyb_f1(vw.hyb, L, 0, cc);
            hyb_f1(vw.hyb, L, 1, uu);
            hyb_f1(vw.hyb, L, 2, vv);
        }
        const double c_grnd = cc.f;
        // atmo::du/dv at the ground point: the scaling there has X = exp(-(zg - zg)/bl) = 1
        const double Xg = exp(-(zg - zg) * a.inv_bl);
        const double scg = (1.0 - Xg) / (1.0 + Xg);
        const double dXg[3] = {Xg * a.inv_bl * A, Xg * a.inv_bl * B, -Xg * a.inv_bl};
        double dcg[3], dug[3], dvg[3];
#pragma unroll
        for (int n = 0; n < 3; n++) {
            const double dscg = -2.0 * dXg[n] / ((1.0 + Xg) * (1.0 + Xg));
            const int h = hix(n);
            dcg[n] = cc.d[h];
            dug[n] = uu.d[h] * scg + uu.f * dscg;
            dvg[n] = vv.d[h] * scg + vv.f * dscg;
        }
        const double norm2 = p[5] - A * p[3] - B * p[4];
        const double n1sq = norm1 * norm1;
        auto dAB = [&](int o, double zz0, double zz1) {
            return (p[6 + o] * (p[5] - B * p[4]) - p[3] * (p[8 + o] - B * p[7 + o])) / norm2 * zz0 +
                   (p[7 + o] * (p[5] - A * p[3]) - p[4] * (p[8 + o] - A * p[6 + o])) / norm2 * zz1;
        };
        const double da_t = dAB(0, zxx, zxy), db_t = dAB(0, zxy, zyy);
        const double da_p = dAB(6, zxx, zxy), db_p = dAB(6, zxy, zyy);
        const double dC1x_t = -4.0 * A / n1sq * ((1.0 + B * B) * da_t - A * B * db_t);
        const double dC1x_p = -4.0 * A / n1sq * ((1.0 + B * B) * da_p - A * B * db_p);
        const double dC1y_t = -4.0 * B / n1sq * ((1.0 + A * A) * db_t - A * B * da_t);
        const double dC1y_p = -4.0 * B / n1sq * ((1.0 + A * A) * db_p - A * B * da_p);
        const double dC1z_t = -4.0 / n1sq * (A * da_t + B * db_t), dC1z_p = -4.0 / n1sq * (A * da_p + B * db_p);
        const double dC2x_t = 2.0 / n1sq * ((1.0 - A * A + B * B) * da_t - 2.0 * A * B * db_t);
        const double dC2x_p = 2.0 / n1sq * ((1.0 - A * A + B * B) * da_p - 2.0 * A * B * db_p);
        const double dC2y_t = 2.0 / n1sq * ((1.0 + A * A - B * B) * db_t - 2.0 * A * B * da_t);
        const double dC2y_p = 2.0 / n1sq * ((1.0 + A * A - B * B) * db_p - 2.0 * A * B * da_p);
        const double ds0_t = -a.c0 / c_grnd * (p[8] - A * p[6] - B * p[7]) / norm2;
        const double ds0_p = -a.c0 / c_grnd * (p[14] - A * p[12] - B * p[13]) / norm2;
        const double cr = a.c0 / c_grnd;
        const double dnux = -1.0 / c_grnd * (cr * dcg[0] + p[3] * dug[0] + p[4] * dvg[0]);
        const double dnuy = -1.0 / c_grnd * (cr * dcg[1] + p[3] * dug[1] + p[4] * dvg[1]);
        const double dnuz = -1.0 / c_grnd * (cr * dcg[2] + p[3] * dug[2] + p[4] * dvg[2]);
#pragma unroll
        for (int o = 0; o <= 6; o += 6) {
            q[6 + o] = C1x * p[6 + o] + C2x * (p[8 + o] - p[7 + o] * B);
            q[7 + o] = C1y * p[7 + o] + C2y * (p[8 + o] - p[6 + o] * A);
            q[8 + o] = -C1z * p[8 + o] + p[6 + o] * C2x + p[7 + o] * C2y;
        }
        q[9] = C1x * p[9] + C2x * (p[11] - B * p[10] - p[4] * db_t) + dC1x_t * p[3] + dC2x_t * (p[5] - B * p[4]) +
               ((C1x - 1.0) * dnux + C2x * (dnuz - B * dnuy)) * ds0_t;
        q[10] = C1y * p[10] + C2y * (p[11] - A * p[9] - p[3] * da_t) + dC1y_t * p[4] + dC2y_t * (p[5] - A * p[3]) +
                ((C1y - 1.0) * dnuy + C2y * (dnuz - A * dnux)) * ds0_t;
        q[11] = -C1z * p[11] + C2x * p[9] + C2y * p[10] - dC1z_t * p[5] + dC2x_t * p[3] + dC2y_t * p[4] +
                (-(C1z + 1.0) * dnuz + C2x * dnux + C2y * dnuy) * ds0_t;
        q[15] = C1x * p[15] + C2x * (p[17] - B * p[16] - p[4] * db_p) + dC1x_p * p[3] + dC2x_p * (p[5] - B * p[4]) +
                ((C1x - 1.0) * dnux + C2x * (dnuz - B * dnuy)) * ds0_p;
        q[16] = C1y * p[16] + C2y * (p[17] - A * p[15] - p[3] * da_p) + dC1y_p * p[4] + dC2y_p * (p[5] - A * p[3]) +
                ((C1y - 1.0) * dnuy + C2y * (dnuz - A * dnux)) * ds0_p;
        q[17] = -C1z * p[17] + C2x * p[15] + C2y * p[16] - dC1z_p * p[5] + dC2x_p * p[3] + dC2y_p * p[4] +
                (-(C1z + 1.0) * dnuz + C2x * dnux + C2y * dnuy) * ds0_p;
    }
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = q[i];
}

// Launch state: set_initial (eqset.3d.rngdep.cpp:59-108)
template <bool AMP>
__device__ __forceinline__ void ray_init_3dr(const Fan3DArgs& a, double theta, double phi, double* y) {
    const double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
    const double mx = a.u0s / a.c0, my = a.v0s / a.c0, mz = 0.0 / a.c0;
    const double n0 = ct * cp, n1 = ct * sp, n2 = st;
    const double ms = 1.0 + (n0 * mx + n1 * my + n2 * mz);
    y[0] = a.src_x; y[1] = a.src_y; y[2] = a.src_z;
    y[3] = n0 / ms; y[4] = n1 / ms; y[5] = n2 / ms;
    if (AMP) {
        const double ms2 = ms * ms;
        const double t0 = -st * cp, t1 = -st * sp, t2 = ct;
        const double p0 = -ct * sp, p1 = ct * cp, p2 = 0.0;
        const double tm = t0 * mx + t1 * my + t2 * mz, pm = p0 * mx + p1 * my + p2 * mz;
        y[6] = y[7] = y[8] = 0.0;
        y[9] = t0 / ms - n0 / ms2 * tm; y[10] = t1 / ms - n1 / ms2 * tm; y[11] = t2 / ms - n2 / ms2 * tm;
        y[12] = y[13] = y[14] = 0.0;
        y[15] = p0 / ms - n0 / ms2 * pm; y[16] = p1 / ms - n1 / ms2 * pm; y[17] = p2 / ms - n2 / ms2 * pm;
    }
}

// PATHS: also write the sampled per-step rows and caustic points of
// run_prop's write_rays / write_topo / write_caustics output
// (main.infraga.3d.rngdep.cpp:440-488); the fan results are unchanged.
template <bool AMP, bool PATHS, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_3DR_MINB) fan3dr_fp64_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = Dim3r<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    double* s_hz = s_mem + N * blockDim.x;
    double* s_hx = s_hz + a.hyb_nz;
    double* s_hy = s_hx + a.hyb_nx;
    double* s_tx = s_hy + a.hyb_ny;
    double* s_ty = s_tx + a.topo_nx;
    for (int i = threadIdx.x; i < a.hyb_nz; i += blockDim.x) s_hz[i] = a.hyb_z[i];
    for (int i = threadIdx.x; i < a.hyb_nx; i += blockDim.x) s_hx[i] = a.hyb_x[i];
    for (int i = threadIdx.x; i < a.hyb_ny; i += blockDim.x) s_hy[i] = a.hyb_y[i];
    for (int i = threadIdx.x; i < a.topo_nx; i += blockDim.x) s_tx[i] = a.topo_x[i];
    for (int i = threadIdx.x; i < a.topo_ny; i += blockDim.x) s_ty[i] = a.topo_y[i];
    __syncthreads();
    Views vw;
    vw.hyb = HybView{a.hyb_tab, s_hx, s_hy, s_hz, a.hyb_nx, a.hyb_ny, a.hyb_nz};
    vw.topo = TopoView{a.topo_tab, s_tx, s_ty, a.topo_nx, a.topo_ny};
    vw.has_topo = a.topo_tab != nullptr;
    double* prev = s_prev + threadIdx.x;

    const int nb = a.bounces + 1;
    const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    double y[N];
    Cells cl{0, 0, 0, 0, 0};
    int bnc, kb, na, caustics;
    double D_prev = 0.0;
    long long steps;
    double s, tt, att, pt, pa, zmax;
    long long p_base = 0, p_cap = 0, p_n = 0;   // PATHS: this ray's row range and rows produced
    // PATHS, back projection: travel-time variations (sums and pending increments as tt / pt)
    double tvt = 0.0, tvp = 0.0, ptvt = 0.0, ptvp = 0.0;
    const bool proj = PATHS && AMP && a.path_rows && a.path_mode == kPathProj;

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * kPi / 180.0;
        const double phi = kPi / 2.0 - a.phi_deg[r] * kPi / 180.0;
        ray_init_3dr<AMP>(a, theta, phi, y);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        tvt = tvp = ptvt = ptvp = 0.0;
        zmax = ST ? a.z0 : 0.0;   // run_prop's z_max = topo::z0 (0 in the range-dependent main)
        if (PATHS && a.path_rows) { p_base = a.path_off[r]; p_cap = a.path_off[r + 1] - p_base; p_n = 0; }
    };
    start_ray(ray);

    while (true) {
        zmax = fmax(zmax, y[2]);
        double ds = a.ds_max;   // set_ds (eqset.3d.rngdep.cpp:215-221)
        if (y[2] < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[2] - topo_z(vw, cl, y[0], y[1])) / 0.2);
        s += ds;
        double acc[N], stg[N], f[N];
        rhs_3dr<AMP, ST>(a, vw, cl, y, f);
        if (AMP && (a.aux || (PATHS && a.caus_rows)) && kb >= 1) {   // caustics between rows 1..k-1 of the bounce
            const double* Xt = y + 6;
            const double* Xp = y + 12;
            const double D = f[0] * (Xt[1] * Xp[2] - Xp[1] * Xt[2]) - Xt[0] * (f[1] * Xp[2] - f[2] * Xp[1]) +
                             Xp[0] * (f[1] * Xt[2] - f[2] * Xt[1]);
            if (kb >= 2 && D * D_prev < 0.0) {
                caustics++;
                if (PATHS && a.caus_rows) {   // row kb (raw altitude); time through segment (kb-1, kb)
                    const unsigned long long w = atomicAdd(a.caus_count, 1ull);
                    if ((long long)w < a.caus_cap) {
                        double* o = a.caus_rows + w * kCausCols;
                        o[0] = y[0]; o[1] = y[1]; o[2] = y[2]; o[3] = tt + pt;
                        o[4] = (double)bnc; o[5] = (double)ray; o[6] = (double)(steps + kb);
                    }
                }
            }
            D_prev = D;
        }
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
        // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
        for (int st = 0; st < 3; st++) {
            rhs_3dr<AMP, ST>(a, vw, cl, stg, f);
            const double w = st < 2 ? c_third : c_sixth;
            const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
            for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
        }
        kb++;

        // s_max, break_check (eqset.3d.rngdep.cpp:434-442), ground_check (:444-451)
        const double rx = acc[0] - a.src_x, ry = acc[1] - a.src_y;
        bool esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) || (acc[0] > a.x_max) || (acc[0] < a.x_min) ||
                   (acc[1] > a.y_max) || (acc[1] < a.y_min) || (acc[2] > a.alt_max);
        const bool gnd = !esc && (acc[2] <= a.topo_zmax) && (acc[2] < topo_z(vw, cl, acc[0], acc[1]));

        double dt, da;
        seg_increment_3dr<ST>(a, vw, cl, y, acc, dt, da);
        if (a.write_rays) { tt += pt; att += pa; pt = dt; pa = da; }
        else { pt += dt; pa += da; }
        if (proj) {   // run_back_proj sums travel_time_var per segment the same way (main.infraga.3d.rngdep.cpp:684-686)
            double vt, vp;
            seg_time_var_3dr<ST>(a, vw, cl, y, acc, vt, vp);
            tvt += ptvt; tvp += ptvp; ptvt = vt; ptvp = vp;
        }

        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(acc[2]) || !isfinite(acc[5])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
            if (proj && path_sampled(a.path_mode, kb)) {
                // projection row (main.infraga.3d.rngdep.cpp:688-714): position with the
                // altitude held at the terrain, derivatives per degree, group velocity
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kProjCols;
                    Cells c2 = cl;
                    const double d2r = kPi / 180.0;
                    o[0] = y[0]; o[1] = y[1]; o[2] = fmax(y[2], topo_z(vw, c2, y[0], y[1])); o[3] = tt + pt;
                    o[4] = y[6] * d2r; o[5] = y[7] * d2r; o[6] = y[8] * d2r; o[7] = (tvt + ptvt) * d2r;
                    o[8] = y[12] * d2r; o[9] = y[13] * d2r; o[10] = y[14] * d2r; o[11] = (tvp + ptvp) * d2r;
                    const double num = sqrt(y[3] * y[3] + y[4] * y[4] + y[5] * y[5]);
                    AtmPt mp;
                    atm_point<ST>(a, vw, c2, y[0], y[1], y[2], mp);
                    o[12] = mp.c * y[3] / num + mp.u;
                    o[13] = mp.c * y[4] / num + mp.v;
                    o[14] = mp.c * y[5] / num;
                }
                p_n++;
            } else if (PATHS && a.path_rows && path_sampled(a.path_mode, kb)) {
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kPathCols;
                    Cells c2 = cl;
                    const double zg = topo_z(vw, c2, y[0], y[1]);
                    o[0] = y[0]; o[1] = y[1];
                    o[2] = a.path_mode == kPathRays ? fmax(y[2], zg) : zg;
                    o[3] = (AMP && a.path_mode == kPathRays)
                               ? amp_db_3dr<ST>(a, vw, c2, y, a.theta_deg[ray] * kPi / 180.0,
                                            kPi / 2.0 - a.phi_deg[ray] * kPi / 180.0, nullptr)
                               : 0.0;
                    o[4] = -2.0 * (att + pa); o[5] = tt + pt; o[6] = (double)bnc;
                }
                p_n++;
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.3d.rngdep.cpp:485-531) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        ptvt = 0.0; ptvp = 0.0;
        int status = -1;
        if (a.topo_tab == nullptr && zmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        if (status < 0) {
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            const double zgk = topo_z(vw, cl, acc[0], acc[1]);
            AtmPt mg;
            atm_point<ST>(a, vw, cl, acc[0], acc[1], zgk, mg);
            const double incl = -asin(mg.c / a.c0 * acc[5]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[3]) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = acc[0];
            out[4] = acc[1];
            out[5] = tt;
            out[6] = sqrt(rx * rx + ry * ry) / tt;
            out[7] = zmax;
            out[8] = incl;
            out[9] = baz;
            double jac = 0.0;
            out[10] = AMP ? amp_db_3dr<ST>(a, vw, cl, acc, th_deg * kPi / 180.0, kPi / 2.0 - ph_deg * kPi / 180.0, &jac) : 0.0;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) {
                    // find_eigenray's derivatives with the terrain slope (geoac.eigenray.3d.cpp:334-347)
                    double A = 0.0, B = 0.0;
                    if (vw.has_topo) {
                        TopoVal t;
                        topo_eval(vw.topo, acc[0], acc[1], 1, t, cl.tx, cl.ty);
                        A = t.d[0]; B = t.d[1];
                    }
                    const double den = acc[5] - A * acc[3] - B * acc[4];
                    const double ds_dth = -a.c0 / mg.c * (acc[8] - A * acc[6] - B * acc[7]) / den;
                    const double ds_dph = -a.c0 / mg.c * (acc[14] - A * acc[12] - B * acc[13]) / den;
                    const double dx_t = acc[6] + acc[3] * ds_dth, dy_t = acc[7] + acc[4] * ds_dth;
                    const double dx_p = acc[12] + acc[3] * ds_dph, dy_p = acc[13] + acc[4] * ds_dph;
                    ax[0] = sqrt(dx_t * dx_t + dy_t * dy_t);
                    ax[1] = sqrt(dx_p * dx_p + dy_p * dy_p);
                    ax[2] = jac;
                    ax[3] = (double)caustics;
                } else {
                    ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
                }
            }
            na++;
            reflect_3dr<N, AMP, ST>(a, vw, cl, y, prev);
            bnc++;
            if (bnc > a.bounces) status = 0;
        }
        if (status < 0) {
            s = 0.0; kb = 0;
            continue;
        }
        a.n_arr[ray] = na;
        a.ray_steps[ray] = steps;
        if (a.ray_status) a.ray_status[ray] = status;
        if (PATHS && a.path_rows) a.path_n[ray] = p_n;
        ray = (int)atomicAdd(a.queue, 1u);
        if (ray >= a.n_rays) break;
        start_ray(ray);
    }
}

template <bool AMP, bool PATHS, bool ST>
cudaError_t launch_impl(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    // threads per block: the caller's choice (a multiple of 32 up to kThreads) or kThreads
    const int threads = a.block > 0 ? a.block : kThreads;
    auto kern = fan3dr_fp64_kernel<AMP, PATHS, ST>;
    const size_t smem = ((size_t)Dim3r<AMP>::n * threads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
                        sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, n_sm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long want = ((long long)a.n_rays + threads - 1) / threads;
    long long grid = (long long)n_sm * per_sm;
    if (want < grid) grid = want;
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    if (grid < 1) grid = 1;
    if (grid_used) *grid_used = (int)grid;
    kern<<<(unsigned)grid, threads, smem, stream>>>(a);
    return cudaGetLastError();
}

// One eigenray-search trace per thread (find_eigenray / est_eigenray on this
// solver, geoac.eigenray.3d.cpp:34-371): n_seg prop_rk4 segments from the
// launch source with terrain reflections between them.  Record mode sums
// time and absorption per step and the turning height over rows 1..k-1 from
// 0 (:229-262) and forms the arrival columns (:265-275); an amplitude trace
// also returns what the Newton derivatives read under the last row
// (:334-342): c at the source and on the ground, the ground height and its
// gradient.  Same block size as the fan kernel (reflect_3dr reads row k-2
// from shared memory with that stride).
template <bool AMP, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_3DR_MINB) trace3dr_fp64_kernel(const __grid_constant__ Fan3DArgs a,
                                                                            const TraceReq* __restrict__ reqs,
                                                                            TraceRes18* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                            SegRes* __restrict__ seg_out,
                                                                            int seg_stride) {
    constexpr int N = Dim3r<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    double* s_hz = s_mem + N * blockDim.x;
    double* s_hx = s_hz + a.hyb_nz;
    double* s_hy = s_hx + a.hyb_nx;
    double* s_tx = s_hy + a.hyb_ny;
    double* s_ty = s_tx + a.topo_nx;
    for (int i = threadIdx.x; i < a.hyb_nz; i += blockDim.x) s_hz[i] = a.hyb_z[i];
    for (int i = threadIdx.x; i < a.hyb_nx; i += blockDim.x) s_hx[i] = a.hyb_x[i];
    for (int i = threadIdx.x; i < a.hyb_ny; i += blockDim.x) s_hy[i] = a.hyb_y[i];
    for (int i = threadIdx.x; i < a.topo_nx; i += blockDim.x) s_tx[i] = a.topo_x[i];
    for (int i = threadIdx.x; i < a.topo_ny; i += blockDim.x) s_ty[i] = a.topo_y[i];
    __syncthreads();
    // persistent: each thread takes the next request when its trace ends, so
    // lanes whose trace finished early do not idle until the warp's longest one
    for (int r = (int)atomicAdd(queue, 1u); r < n; r = (int)atomicAdd(queue, 1u)) {
        Views vw;
        vw.hyb = HybView{a.hyb_tab, s_hx, s_hy, s_hz, a.hyb_nx, a.hyb_ny, a.hyb_nz};
        vw.topo = TopoView{a.topo_tab, s_tx, s_ty, a.topo_nx, a.topo_ny};
        vw.has_topo = a.topo_tab != nullptr;
        double* prev = s_prev + threadIdx.x;
        const TraceReq q = reqs[r];
        const bool record = (q.flags & kRecord) != 0, stop = (q.flags & kStopOnEscape) != 0;
        const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;

        double y[N];
        Cells cl{0, 0, 0, 0, 0};
        ray_init_3dr<AMP>(a, q.theta, q.phi, y);
        double tt = 0.0, att = 0.0, zmax = 0.0;
        long long steps = 0;
        double acc[N];
        bool esc = false;
        for (int sg = 0; sg < q.n_seg; sg++) {
            double s = 0.0, pt = 0.0, pa = 0.0;
            int kb = 0;
            bool capped = false;
#pragma unroll
            for (int i = 0; i < N; i++) prev[i * blockDim.x] = y[i];
            while (true) {
                if (record && kb >= 1) zmax = fmax(zmax, y[2]);
                double ds = a.ds_max;
                if (y[2] < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[2] - topo_z(vw, cl, y[0], y[1])) / 0.2);
                s += ds;
                double stg[N], f[N];
                rhs_3dr<AMP, ST>(a, vw, cl, y, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
                // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
                for (int st = 0; st < 3; st++) {
                    rhs_3dr<AMP, ST>(a, vw, cl, stg, f);
                    const double w = st < 2 ? c_third : c_sixth;
                    const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
                    for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
                }
                kb++;
                const double rx = acc[0] - a.src_x, ry = acc[1] - a.src_y;
                esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) || (acc[0] > a.x_max) || (acc[0] < a.x_min) ||
                      (acc[1] > a.y_max) || (acc[1] < a.y_min) || (acc[2] > a.alt_max);
                const bool gnd = !esc && (acc[2] <= a.topo_zmax) && (acc[2] < topo_z(vw, cl, acc[0], acc[1]));
                if (record) {
                    double dt, da;
                    seg_increment_3dr<ST>(a, vw, cl, y, acc, dt, da);
                    tt += pt; att += pa; pt = dt; pa = da;
                }
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(acc[2]) || !isfinite(acc[5])) esc = true;
                }
                if (!esc && !gnd) {
#pragma unroll
                    for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
                    continue;
                }
                break;
            }
            steps += capped ? a.length : kb;
            if (seg_out) {
                SegRes& g = seg_out[(size_t)r * seg_stride + sg];
                g.x = acc[0]; g.y = acc[1]; g.steps = steps; g.escaped = esc ? 1 : 0;
            }
            if (sg == q.n_seg - 1 || (esc && stop)) break;
            reflect_3dr<N, AMP, ST>(a, vw, cl, y, prev);
        }
        TraceRes18& o = out[r];
#pragma unroll
        for (int i = 0; i < 18; i++) o.y[i] = i < N ? acc[i] : 0.0;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        o.tt = o.att = o.zmax = o.amp_db = o.incl = o.baz = 0.0;
        o.c_src = a.c0; o.c_grnd = 0.0; o.z_grnd = 0.0; o.dzg[0] = 0.0; o.dzg[1] = 0.0;
        if (AMP && !record) {   // ground under the last row: topo::z (0 without terrain), topo::dz, atmo::c there
            double zg = 0.0;
            if (vw.has_topo) {
                TopoVal t;
                topo_eval(vw.topo, acc[0], acc[1], 1, t, cl.tx, cl.ty);
                zg = t.z; o.dzg[0] = t.d[0]; o.dzg[1] = t.d[1];
            }
            AtmPt m;
            atm_point<ST>(a, vw, cl, acc[0], acc[1], zg, m);
            o.z_grnd = zg;
            o.c_grnd = m.c;
        }
        if (record) {
            o.tt = tt; o.att = att; o.zmax = zmax;
            o.amp_db = AMP ? amp_db_3dr<ST>(a, vw, cl, acc, q.theta, q.phi, nullptr) : 0.0;
            AtmPt m;
            atm_point<ST>(a, vw, cl, acc[0], acc[1], acc[2], m);
            o.incl = -asin(m.c / a.c0 * acc[5]) * (180.0 / kPi);
            double baz = 90.0 - atan2(-acc[4], -acc[3]) * (180.0 / kPi);
            while (baz > 180.0) baz -= 360.0;
            while (baz < -180.0) baz += 360.0;
            o.baz = baz;
        }
    }
}

template <bool AMP, bool ST>
cudaError_t launch_trace_impl(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, cudaStream_t st,
                              SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = trace3dr_fp64_kernel<AMP, ST>;
    const size_t smem = ((size_t)Dim3r<AMP>::n * kThreads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
                        sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kThreads, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride);
    return cudaGetLastError();
}

// a.knots set (no hybrid tables): stratified profile over terrain
template <bool ST>
cudaError_t launch_fan(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    if (a.path_rows || a.caus_rows)
        return calc_amp ? launch_impl<true, true, ST>(a, stream, grid_used) : launch_impl<false, true, ST>(a, stream, grid_used);
    return calc_amp ? launch_impl<true, false, ST>(a, stream, grid_used) : launch_impl<false, false, ST>(a, stream, grid_used);
}

}  // namespace

cudaError_t launch_fan3dr_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    return a.knots ? launch_fan<true>(a, calc_amp, stream, grid_used) : launch_fan<false>(a, calc_amp, stream, grid_used);
}

cudaError_t launch_trace_3dr(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                             cudaStream_t st, SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (a.knots)
        return amp ? launch_trace_impl<true, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
                   : launch_trace_impl<false, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
    return amp ? launch_trace_impl<true, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
               : launch_trace_impl<false, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
}

}  // namespace iga
