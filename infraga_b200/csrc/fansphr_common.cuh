// Device helpers of the spherical range-dependent solver (also infraga-sph
// over terrain, the ST forms), shared by the FP64 and FP32-compensated
// kernels: cached cell indices, the atmosphere at a point with its gradient
// and Hessian, the right-hand side, travel time / absorption segments,
// amplitude and the terrain reflection.
#pragma once
#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fansph_common.cuh"
#include "rngdep_eval.cuh"

namespace iga {

namespace {

// per-thread cached cell indices
struct Cells {
    int hx, hy, hz;   // hybrid grid
    int tx, ty;       // terrain grid
};

struct Views {
    HybView hyb;
    TopoView topo;
    bool has_topo;
};

// topo::z (atmo_state.sph.rngdep.cpp:43-52): r_earth + terrain, or the flat ground
__device__ __forceinline__ double topo_r(const Fan3DArgs& a, const Views& v, Cells& cl, double lat, double lon) {
    if (!v.has_topo) return a.r_grnd;
    TopoVal t;
    topo_eval(v.topo, lat, lon, 0, t, cl.tx, cl.ty);
    return a.r_earth + t.z;
}

// atmosphere at a stage state, as update_refs sees it
// (geoac.eqset.sph.rngdep.cpp:238-301; calc_uvw atmo_state.sph.rngdep.cpp:584-888):
// index 0 = r, 1 = lat, 2 = lon.
struct AtmFull {
    double c, dc[3], ddc[3][3];
    double u, du[3], ddu[3][3];
    double v, dv[3], ddv[3][3];
};

// Stratified profile row at the altitude r - r_earth clamped to the knot
// range (interp::in_interval); cl.hz caches the segment.
__device__ __forceinline__ const double* strat_at(const Fan3DArgs& a, Cells& cl, double r, Cubic& q) {
    const double ze = fmin(fmax(r - a.r_earth, a.z_lo), a.z_hi);
    cl.hz = seg_walk(a.knots, a.n_knots, ze, cl.hz);
    const double* r0 = a.knots + cl.hz * kStride;
    q = cubic_at(r0, ze);
    return r0;
}

template <bool AMP, bool ST>
__device__ __forceinline__ void atm_full(const Fan3DArgs& a, const Views& vw, Cells& cl, double r, double lat, double lon,
                                         AtmFull& m) {
    HybF2 c2 = {}, u2 = {}, v2 = {};
    if (ST) {   // derivatives in r only
        Cubic q;
        const double* r0 = strat_at(a, cl, r, q);
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
    hyb_locate(vw.hyb, lat, lon, r - a.r_earth, L, cl.hx, cl.hy, cl.hz);
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
    // boundary-layer scaling over the terrain (or flat ground)
    const double zr = r - a.r_earth;
    double zg = a.r_grnd, dzg[2] = {0.0, 0.0}, ddzg[3] = {0.0, 0.0, 0.0};
    double X = 0.0;
    if (zr < a.x_cut) {
        if (vw.has_topo) {
            TopoVal t;
            const bool in_bl = zr < a.z_bl;
            topo_eval(vw.topo, lat, lon, in_bl ? (AMP ? 2 : 1) : 0, t, cl.tx, cl.ty);
            zg = a.r_earth + t.z;
            if (in_bl) {
                dzg[0] = t.d[0]; dzg[1] = t.d[1];
                if (AMP) { ddzg[0] = t.dd[0]; ddzg[1] = t.dd[1]; ddzg[2] = t.dd[2]; }
            }
        }
        X = exp(-(r - zg) * a.inv_bl);
    }
    const double ib = a.inv_bl, ib2 = ib * ib;
    const double dX[3] = {-X * ib, X * ib * dzg[0], X * ib * dzg[1]};
    const double iop = 1.0 / (1.0 + X), iop2 = iop * iop, iop3 = iop2 * iop;
    const double sc0 = (1.0 - X) * iop;
    double dsc[3];
#pragma unroll
    for (int n = 0; n < 3; n++) dsc[n] = -2.0 * dX[n] * iop2;
    m.c = c2.f; m.u = u2.f * sc0; m.v = v2.f * sc0;
#pragma unroll
    for (int n = 0; n < 3; n++) {
        m.dc[n] = c2.d[n];
        m.du[n] = u2.d[n] * sc0 + u2.f * dsc[n];
        m.dv[n] = v2.d[n] * sc0 + v2.f * dsc[n];
    }
    if (AMP) {
        // ddX (calc_uvw, atmo_state.sph.rngdep.cpp:744-770) with ddzg = (xx, xy, yy)
        double ddX[3][3];
        ddX[0][0] = X * ib2;
        ddX[0][1] = ddX[1][0] = -X * ib2 * dzg[0];
        ddX[0][2] = ddX[2][0] = -X * ib2 * dzg[1];
        ddX[1][1] = (ddzg[0] + dzg[0] * dzg[0] * ib) * (X * ib);
        ddX[1][2] = ddX[2][1] = (ddzg[1] + dzg[0] * dzg[1] * ib) * (X * ib);
        ddX[2][2] = (ddzg[2] + dzg[1] * dzg[1] * ib) * (X * ib);
#pragma unroll
        for (int n = 0; n < 3; n++) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double dds = -2.0 * (ddX[n][k] * iop2 - 2.0 * dX[n] * dX[k] * iop3);
                m.ddc[n][k] = c2.dd[n][k];
                m.ddu[n][k] = u2.dd[n][k] * sc0 + u2.d[n] * dsc[k] + u2.d[k] * dsc[n] + u2.f * dds;
                m.ddv[n][k] = v2.dd[n][k] * sc0 + v2.d[n] * dsc[k] + v2.d[k] * dsc[n] + v2.f * dds;
            }
        }
    }
}

// RHS with full gradients: update_refs + eval_src_eq
// (geoac.eqset.sph.rngdep.cpp:238-437), w = 0.
template <bool AMP, bool ST>
__device__ __forceinline__ void rhs_sphr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y, double* f) {
    AtmFull m;
    atm_full<AMP, ST>(a, vw, cl, y[0], y[1], y[2], m);
    const double r = y[0];
    double st, ct;
    sincos(y[1], &st, &ct);
    const double ir = 1.0 / r, ict = 1.0 / ct, tnt = st * ict;
    const double n0 = y[3], n1 = y[4], n2 = y[5];
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double inum = 1.0 / num;
    const double cg0 = m.c * n0 * inum, cg1 = m.c * n1 * inum + m.v, cg2 = m.c * n2 * inum + m.u;
    const double cgm = sqrt(cg0 * cg0 + cg1 * cg1 + cg2 * cg2);
    const double icg = 1.0 / cgm;
    const double G[3] = {1.0, ir, ir * ict};
    const double T[3] = {-ir * (n1 * cg1 + n2 * cg2), n0 * m.v + n0 * cg1 + n2 * cg2 * tnt,
                         n0 * m.u * ct + (n1 * m.u - n2 * m.v) * st + cg2 * (n0 * ct - n1 * st)};
    const double cg[3] = {cg0, cg1, cg2};
    double K[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        K[i] = num * m.dc[i] + n1 * m.dv[i] + n2 * m.du[i];
        f[i] = G[i] * cg[i] * icg;
        f[3 + i] = -G[i] * icg * (K[i] + T[i]);
    }
    if (AMP) {
        const double icg2 = icg * icg, ir2 = ir * ir;
        const double cin = m.c * inum, cin2 = cin * inum;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const double* R = y + 6 + 6 * j;
            const double* mu = y + 9 + 6 * j;
            const double dc = R[0] * m.dc[0] + R[1] * m.dc[1] + R[2] * m.dc[2];
            const double du = R[0] * m.du[0] + R[1] * m.du[1] + R[2] * m.du[2];
            const double dv = R[0] * m.dv[0] + R[1] * m.dv[1] + R[2] * m.dv[2];
            const double dnu = (n0 * mu[0] + n1 * mu[1] + n2 * mu[2]) * inum;
            const double g0 = n0 * inum * dc + cin * mu[0] - cin2 * n0 * dnu;
            const double g1 = n1 * inum * dc + cin * mu[1] - cin2 * n1 * dnu + dv;
            const double g2 = n2 * inum * dc + cin * mu[2] - cin2 * n2 * dnu + du;
            const double gg[3] = {g0, g1, g2};
            const double dm = (cg0 * g0 + cg1 * g1 + cg2 * g2) * icg;
            const double dG[3] = {0.0, -R[0] * ir2, -R[0] * ir2 * ict + st * ir * ict * ict * R[1]};
            const double dT[3] = {
                R[0] * ir2 * (n1 * cg1 + n2 * cg2) - ir * (mu[1] * cg1 + n1 * g1 + mu[2] * cg2 + n2 * g2),
                (mu[0] * m.v + n0 * dv) + mu[0] * cg1 + n0 * g1 + (mu[2] * cg2 + n2 * g2) * tnt + n2 * cg2 * R[1] * ict * ict,
                (mu[0] * m.u + n0 * du) * ct - (n0 * m.u) * R[1] * st + (mu[1] * m.u + n1 * du - mu[2] * m.v - n2 * dv) * st +
                    (n1 * m.u - n2 * m.v) * R[1] * ct + g2 * (n0 * ct - n1 * st) +
                    cg2 * ((mu[0] - n1 * R[1]) * ct - (mu[1] + n0 * R[1]) * st)};
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const double ddc = R[0] * m.ddc[i][0] + R[1] * m.ddc[i][1] + R[2] * m.ddc[i][2];
                const double ddu = R[0] * m.ddu[i][0] + R[1] * m.ddu[i][1] + R[2] * m.ddu[i][2];
                const double ddv = R[0] * m.ddv[i][0] + R[1] * m.ddv[i][1] + R[2] * m.ddv[i][2];
                f[6 + 6 * j + i] = dG[i] * cg[i] * icg + G[i] * gg[i] * icg - G[i] * cg[i] * icg2 * dm;
                f[9 + 6 * j + i] = -dG[i] * icg * (K[i] + T[i]) + G[i] * icg2 * dm * K[i] -
                                   G[i] * icg * (dnu * m.dc[i] + num * ddc + mu[1] * m.dv[i] + mu[2] * m.du[i] +
                                                 n1 * ddv + n2 * ddu + dT[i]);
            }
        }
    }
}

// atmo::u/v scaling (bndlyr_sc, atmo_state.sph.rngdep.cpp:97-104)
__device__ __forceinline__ double bl_sc(const Fan3DArgs& a, const Views& vw, Cells& cl, double r, double lat, double lon) {
    if (r - a.r_earth < a.z_bl) {
        const double X = exp(-(r - topo_r(a, vw, cl, lat, lon)) * a.inv_bl);
        return (1.0 - X) / (1.0 + X);
    }
    return 1.0;
}

// c, u, v, rho as atmo::c/u/v/rho return them at (r, lat, lon)
struct AtmPt {
    double c, u, v, rho;
};
template <bool ST>
__device__ __forceinline__ void atm_point(const Fan3DArgs& a, const Views& vw, Cells& cl, double r, double lat, double lon,
                                          AtmPt& o) {
    if (ST) {
        const double sc = bl_sc(a, vw, cl, r, lat, lon);
        Cubic q;
        const double* r0 = strat_at(a, cl, r, q);
        o.c = cubic_f(r0, q, 2);
        o.u = cubic_f(r0, q, 4) * sc;
        o.v = cubic_f(r0, q, 6) * sc;
        o.rho = cubic_f(r0, q, 8);
        return;
    }
    HybLoc L;
    hyb_locate(vw.hyb, lat, lon, r - a.r_earth, L, cl.hx, cl.hy, cl.hz);
    const double sc = bl_sc(a, vw, cl, r, lat, lon);
    o.c = hyb_f(vw.hyb, L, 0);
    o.u = hyb_f(vw.hyb, L, 1) * sc;
    o.v = hyb_f(vw.hyb, L, 2) * sc;
    o.rho = hyb_f(vw.hyb, L, 3);
}

// atmo::c alone at (r, lat, lon)
template <bool ST>
__device__ __forceinline__ double c_at(const Fan3DArgs& a, const Views& vw, Cells& cl, double r, double lat, double lon) {
    if (ST) {
        Cubic q;
        const double* r0 = strat_at(a, cl, r, q);
        return cubic_f(r0, q, 2);
    }
    HybLoc L;
    hyb_locate(vw.hyb, lat, lon, r - a.r_earth, L, cl.hx, cl.hy, cl.hz);
    return hyb_f(vw.hyb, L, 0);
}

// travel_time / atten segment (geoac.eqset.sph.rngdep.cpp:547-579, 775-796):
// the atmosphere is read at (r, lat, lon) of the segment midpoint with the
// longitude midpoint taken before the +-2 pi wrap of dp.
template <bool ST>
__device__ __forceinline__ void seg_increment_sphr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y0,
                                                   const double* y1, double& dt_out, double& da_out) {
    const double dr = y1[0] - y0[0], rm = y0[0] + dr * 0.5;
    const double dth = y1[1] - y0[1], tm = y0[1] + dth * 0.5;
    double dp = y1[2] - y0[2];
    const double pm = y0[2] + dp * 0.5;
    if (dp > kPi) dp -= 2.0 * kPi;
    else if (dp < -kPi) dp += 2.0 * kPi;
    const double a1 = rm * dth, a2 = rm * cos(tm) * dp;
    const double ds = sqrt(dr * dr + a1 * a1 + a2 * a2);
    const double n0 = y0[3] + (y1[3] - y0[3]) * 0.5;
    const double n1 = y0[4] + (y1[4] - y0[4]) * 0.5;
    const double n2 = y0[5] + (y1[5] - y0[5]) * 0.5;
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    AtmPt m;
    atm_point<ST>(a, vw, cl, rm, tm, pm, m);
    const double inum = 1.0 / num;
    const double cp0 = m.c * n0 * inum, cp1 = m.c * n1 * inum + m.v, cp2 = m.c * n2 * inum + m.u;
    dt_out = ds / sqrt(cp0 * cp0 + cp1 * cp1 + cp2 * cp2);
    da_out = sb_alpha<true>(m.c, m.rho, rm - a.r_earth, a.freq, a.tweak_abs, a.sb) * ds;
}

// geoac::amp / jacobian at the below-ground row (geoac.eqset.sph.rngdep.cpp:798-850)
template <bool ST>
__device__ __noinline__ double amp_db_sphr(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* y, double theta,
                                           double phi, double* jac_out) {
    AtmPt m;
    atm_point<ST>(a, vw, cl, y[0], y[1], y[2], m);
    const double r = y[0], n0 = y[3], n1 = y[4], n2 = y[5];
    double st, ct, sp, cp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    const double ms = 1.0 + (st * 0.0 + ct * sp * (a.v0s / a.c0) + ct * cp * (a.u0s / a.c0));
    const double nu0 = 1.0 / ms;
    const double e0 = nu0 * st, e1 = nu0 * ct * sp, e2 = nu0 * ct * cp;
    const double g0 = a.c0 * e0 / nu0, g1 = a.c0 * e1 / nu0 + a.v0s, g2 = a.c0 * e2 / nu0 + a.u0s;
    const double cgm0 = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
    const double numag = (a.c0 - n1 * m.v - n2 * m.u) / m.c;
    const double p0 = m.c * n0 / numag, p1 = m.c * n1 / numag + m.v, p2 = m.c * n2 / numag + m.u;
    const double cpm = sqrt(p0 * p0 + p1 * p1 + p2 * p2);
    const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double j0 = m.c * n0 / nm, j1 = m.c * n1 / nm + m.v, j2 = m.c * n2 / nm + m.u;
    const double jm = sqrt(j0 * j0 + j1 * j1 + j2 * j2);
    const double cl1 = cos(y[1]);
    const double dr_ds = j0 / jm, dt_ds = 1.0 / r * j1 / jm, dp_ds = 1.0 / (r * cl1) * j2 / jm;
    const double* Rt = y + 6;
    const double* Rp = y + 12;
    const double jac = r * r * cl1 *
                       (dr_ds * (Rt[1] * Rp[2] - Rp[1] * Rt[2]) - Rt[0] * (dt_ds * Rp[2] - dp_ds * Rp[1]) +
                        Rp[0] * (dt_ds * Rt[2] - dp_ds * Rt[1]));
    const double numr = m.rho * numag * (m.c * m.c * m.c) * cgm0 * ct;
    const double den = a.rho0 * nu0 * (a.c0 * a.c0 * a.c0) * cpm * jac;
    if (jac_out) *jac_out = jac;
    return 20.0 * log10(sqrt(fabs(numr / den)));
}

// approx_intercept + set_refl (geoac.eqset.sph.rngdep.cpp:117-224), general
// terrain; p = row k-2 on entry (element i at prev[i * stride]), y = row k-1
// (in/out).
template <int N, bool AMP, bool ST>
__device__ __noinline__ void reflect_sphr(const Fan3DArgs& a, const Views& vw, Cells& cl, double* y, const double* prev,
                                        int stride) {
    // approx_intercept with the terrain slope at row k-1
    double zy = a.r_grnd, dzy[2] = {0.0, 0.0};
    if (vw.has_topo) {
        TopoVal t;
        topo_eval(vw.topo, y[1], y[2], 1, t, cl.tx, cl.ty);
        zy = a.r_earth + t.z; dzy[0] = t.d[0]; dzy[1] = t.d[1];
    }
    const double dr_grnd = zy - y[0];
    const double dr_k = (y[0] - prev[0]) - (y[1] - prev[1 * stride]) * 1.0 / y[0] * dzy[0] -
                        (y[2] - prev[2 * stride]) * 1.0 / (y[0] * cos(y[1])) * dzy[1];
    double p[N];
#pragma unroll
    for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * stride]) / dr_k * dr_grnd;

    double rg = a.r_grnd, dz0 = 0.0, dz1 = 0.0, zxx = 0.0, zxy = 0.0, zyy = 0.0;
    if (vw.has_topo) {
        TopoVal t;
        topo_eval(vw.topo, p[1], p[2], AMP ? 2 : 1, t, cl.tx, cl.ty);
        rg = a.r_earth + t.z; dz0 = t.d[0]; dz1 = t.d[1];
        if (AMP) { zxx = t.dd[0]; zxy = t.dd[1]; zyy = t.dd[2]; }
    }
    const double cl1 = cos(p[1]);
    const double A = 1.0 / rg * dz0;
    const double B = 1.0 / (rg * cl1) * dz1;
    const double norm1 = 1.0 + A * A + B * B;
    const double C1r = (1.0 - A * A - B * B) / norm1;
    const double C1th = (1.0 - A * A + B * B) / norm1, C2th = 2.0 * A / norm1;
    const double C1ph = (1.0 + A * A - B * B) / norm1, C2ph = 2.0 * B / norm1;

    double q[N];
    q[0] = rg; q[1] = p[1]; q[2] = p[2];
    q[3] = -C1r * p[3] + C2th * p[4] + C2ph * p[5];
    q[4] = C1th * p[4] + C2th * (p[3] - B * p[5]);
    q[5] = C1ph * p[5] + C2ph * (p[3] - A * p[4]);
    if (AMP) {
        // atmosphere at the intercept: c and its gradient (atmo::c/dc), and
        // du, dv = df * sc + f * dsc with the scaling at the ground itself
        // (X = 1: sc = 0, dsc = (1/bl)/2 * (1, -dz_lat, -dz_lon))
        HybF1 cc = {}, uu = {}, vv = {};
        if (ST) {   // atmo::c, dc, du, dv at the ground point (atmo_state.sph.strat.cpp:172-234)
            Cubic qz;
            const double* r0 = strat_at(a, cl, rg, qz);
            cubic_f1(r0, qz, 2, cc.f, cc.d[0]);
            cubic_f1(r0, qz, 4, uu.f, uu.d[0]);
            cubic_f1(r0, qz, 6, vv.f, vv.d[0]);
        } else {
            HybLoc L;
            hyb_locate(vw.hyb, p[1], p[2], rg - a.r_earth, L, cl.hx, cl.hy, cl.hz);
            hyb_f1(vw.hyb, L, 0, cc);
            hyb_f1(vw.hyb, L, 1, uu);
            hyb_f1(vw.hyb, L, 2, vv);
        }
        const double c_grnd = cc.f;
        const double Xg = exp(-(rg - rg) * a.inv_bl);
        const double scg = (1.0 - Xg) / (1.0 + Xg);
        const double dXg[3] = {-Xg * a.inv_bl, Xg * a.inv_bl * dz0, Xg * a.inv_bl * dz1};
        double dcg[3], dug[3], dvg[3];
#pragma unroll
        for (int n = 0; n < 3; n++) {
            const double dscg = -2.0 * dXg[n] / ((1.0 + Xg) * (1.0 + Xg));
            dcg[n] = cc.d[n];
            dug[n] = uu.d[n] * scg + uu.f * dscg;
            dvg[n] = vv.d[n] * scg + vv.f * dscg;
        }
        const double norm2 = p[3] - A * p[4] - B * p[5];
        const double n1sq = norm1 * norm1;
        auto da = [&](int o) {   // o = 0: inclination (6..8), 6: azimuth (12..14)
            return -p[6 + o] / rg * A + 1.0 / rg * ((p[7 + o] * (p[3] - B * p[5]) - p[4] * (p[6 + o] / rg - cl1 * B * p[8 + o])) / norm2 * zxx +
                                                    (p[8 + o] * (p[3] - A * p[4]) - p[5] * (p[6 + o] / (rg * cl1) - A / cl1 * p[7 + o])) / norm2 * zxy);
        };
        auto db = [&](int o) {   // tan(prev[4]) as in the reference (geoac.eqset.sph.rngdep.cpp:161)
            return -(p[6 + o] / rg - tan(p[4]) * p[7 + o]) * B +
                   1.0 / (rg * cl1) * ((p[7 + o] * (p[3] - B * p[5]) - p[4] * (p[6 + o] / rg - cl1 * B * p[8 + o])) / norm2 * zxy +
                                       (p[8 + o] * (p[3] - A * p[4]) - p[5] * (p[6 + o] / (rg * cl1) - A / cl1 * p[7 + o])) / norm2 * zyy);
        };
        const double da_t = da(0), da_p = da(6), db_t = db(0), db_p = db(6);
        const double dC1r_t = -4.0 / n1sq * (A * da_t + B * db_t), dC1r_p = -4.0 / n1sq * (A * da_p + B * db_p);
        const double dC1th_t = -4.0 * A / n1sq * ((1.0 + B * B) * da_t - A * B * db_t);
        const double dC1th_p = -4.0 * A / n1sq * ((1.0 + B * B) * da_p - A * B * db_p);
        const double dC1ph_t = -4.0 * B / n1sq * ((1.0 + A * A) * db_t - A * B * da_t);
        const double dC1ph_p = -4.0 * B / n1sq * ((1.0 + A * A) * db_p - A * B * da_p);
        const double dC2th_t = 2.0 / n1sq * ((1.0 - A * A + B * B) * da_t - 2.0 * A * B * db_t);
        const double dC2th_p = 2.0 / n1sq * ((1.0 - A * A + B * B) * da_p - 2.0 * A * B * db_p);
        // dC2ph/dlth uses db_dlth in both places (geoac.eqset.sph.rngdep.cpp:171)
        const double dC2ph_t = 2.0 / n1sq * ((1.0 + A * A - B * B) * db_t - 2.0 * A * B * db_t);
        const double dC2ph_p = 2.0 / n1sq * ((1.0 + A * A - B * B) * db_p - 2.0 * A * B * da_p);
        const double ds0_t = -a.c0 / c_grnd * (p[6] - rg * A * p[7] - rg * cl1 * B * p[8]) / norm2;
        const double ds0_p = -a.c0 / c_grnd * (p[12] - rg * A * p[13] - rg * cl1 * B * p[14]) / norm2;
        const double cr = a.c0 / c_grnd, cg2c0 = c_grnd * c_grnd / a.c0;
        double dnu_r = cr * dcg[0] + p[4] * dvg[0] + p[5] * dug[0];
        double dnu_t = cr * dcg[1] + p[4] * dvg[1] + p[5] * dug[1];
        double dnu_p = cr * dcg[2] + p[4] * dvg[2] + p[5] * dug[2];
        dnu_r += cg2c0 * 1.0 / rg * (p[4] * p[4] + p[5] * p[5]);
        dnu_t -= cg2c0 * (p[3] * p[4] + tan(p[1]) * p[5] * p[5]);
        dnu_p -= cg2c0 * p[5] * (p[3] * cl1 + p[4] * sin(p[1]));
        dnu_r *= -1.0 / c_grnd;
        dnu_t *= -1.0 / (c_grnd * rg);
        dnu_p *= -1.0 / (c_grnd * rg * cl1);
#pragma unroll
        for (int o = 0; o <= 6; o += 6) {
            q[6 + o] = -C1r * p[6 + o] + rg * C2th * p[7 + o] + rg * cl1 * C2ph * p[8 + o];
            q[7 + o] = C1th * p[7 + o] + C2th * (p[6 + o] / rg - B * cl1 * p[8 + o]);
            q[8 + o] = C1ph * p[8 + o] + C2ph * (p[6 + o] / (rg * cl1) - A / cl1 * p[7 + o]);
        }
        q[9] = -C1r * p[9] + C2th * p[10] + C2ph * p[11] - dC1r_t * p[3] + dC2th_t * p[4] + dC2ph_t * p[5] +
               (-(C1r + 1.0) * dnu_r + C2th * dnu_t + C2ph * dnu_p) * ds0_t;
        q[10] = C1th * p[10] + C2th * (p[9] - B * p[11] - db_t * p[5]) + dC1th_t * p[4] + dC2th_t * (p[3] - B * p[5]) +
                ((C1th - 1.0) * dnu_t + C2th * (dnu_r - B * dnu_p)) * ds0_t;
        q[11] = C1ph * p[11] + C2ph * (p[9] - A * p[10] - da_t * p[4]) + dC1ph_t * p[5] + dC2ph_t * (p[3] - A * p[4]) +
                ((C1ph - 1.0) * dnu_p + C2ph * (dnu_r - A * dnu_t)) * ds0_t;
        q[15] = -C1r * p[15] + C2th * p[16] + C2ph * p[17] - dC1r_p * p[3] + dC2th_p * p[4] + dC2ph_p * p[5] +
                (-(C1r + 1.0) * dnu_r + C2th * dnu_t + C2ph * dnu_p) * ds0_p;
        q[16] = C1th * p[16] + C2th * (p[15] - B * p[17] - db_p * p[5]) + dC1th_p * p[4] + dC2th_p * (p[3] - B * p[5]) +
                ((C1th - 1.0) * dnu_t + C2th * (dnu_r - B * dnu_p)) * ds0_p;
        q[17] = C1ph * p[17] + C2ph * (p[15] - A * p[16] - da_p * p[4]) + dC1ph_p * p[5] + dC2ph_p * (p[3] - A * p[4]) +
                ((C1ph - 1.0) * dnu_p + C2ph * (dnu_r - A * dnu_t)) * ds0_p;
    }
#pragma unroll
    for (int i = 0; i < N; i++) y[i] = q[i];
}

}  // namespace

}  // namespace iga
