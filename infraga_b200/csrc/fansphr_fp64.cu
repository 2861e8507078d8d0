// FP64 ray-fan kernel: spherical (global) geometry, range-dependent
// atmosphere (hybrid 3D splines), flat ground or terrain.
//
// Execution scheme as in the other fan kernels (one thread per ray,
// persistent grid on a device ray queue, one RK4 step per loop iteration,
// ground hits / arrivals / reflections in the loop, row k-1 in shared
// memory).  The atmosphere tables (atmo_rngdep.h) are read through the
// read-only cache: a ray reads the 4 corner records of its cell (2 x 512 B
// each, two z knots) per evaluation and stays in the same cell for many
// steps, so the working set is L1/L2-resident; the node coordinate arrays
// are staged in shared memory.
//
// Physics: the reference's spherical range-dependent equation set
// (src/geoac/geoac.eqset.sph.rngdep.cpp) with atmo_state.sph.rngdep.cpp
// (no boundary-layer vertical wind: topo_use_BLw=false, the default), its RK4
// driver (src/util/rk4solver.cpp:14-85) and run_prop
// (src/main.infraga.sph.rngdep.cpp:412-545).
//
// ST instantiations run infraga-sph's stratified profile over terrain
// (topo_file=): c, u, v, rho from the 1D knot table at the clamped altitude
// (atmo_state.sph.strat.cpp:166-245, calc_uvw :498-800) with the same terrain,
// boundary-layer scaling, equations (geoac.eqset.sph.strat.cpp differs from
// the range-dependent set only in where the atmosphere comes from) and bounce
// loop; run_prop of infraga-sph records the arrival inclination as -asin(...)
// (main.infraga.sph.cpp:523) where the range-dependent one has +asin.
#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fansph_common.cuh"
#include "rngdep_eval.cuh"

namespace iga {

namespace {

#ifndef IGA_SPHR_THREADS
#define IGA_SPHR_THREADS 128
#endif
#ifndef IGA_SPHR_MINB
#define IGA_SPHR_MINB 1
#endif
constexpr int kThreads = IGA_SPHR_THREADS;

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
// terrain; p = row k-2 on entry (the shared-memory copy), y = row k-1 (in/out).
template <int N, bool AMP, bool ST>
__device__ __noinline__ void reflect_sphr(const Fan3DArgs& a, const Views& vw, Cells& cl, double* y, const double* prev) {
    // approx_intercept with the terrain slope at row k-1
    double zy = a.r_grnd, dzy[2] = {0.0, 0.0};
    if (vw.has_topo) {
        TopoVal t;
        topo_eval(vw.topo, y[1], y[2], 1, t, cl.tx, cl.ty);
        zy = a.r_earth + t.z; dzy[0] = t.d[0]; dzy[1] = t.d[1];
    }
    const double dr_grnd = zy - y[0];
    const double dr_k = (y[0] - prev[0]) - (y[1] - prev[1 * blockDim.x]) * 1.0 / y[0] * dzy[0] -
                        (y[2] - prev[2 * blockDim.x]) * 1.0 / (y[0] * cos(y[1])) * dzy[1];
    double p[N];
#pragma unroll
    for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * blockDim.x]) / dr_k * dr_grnd;

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

// PATHS: also write the sampled per-step rows and caustic points of
// run_prop's write_rays / write_topo / write_caustics output
// (main.infraga.sph.rngdep.cpp:450-503); the fan results are unchanged.
template <bool AMP, bool PATHS, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_SPHR_MINB) fansphr_fp64_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = DimSph<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    // node coordinates in shared memory
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
    double* prev = s_prev + threadIdx.x;   // element i at prev[i * blockDim.x]

    const int nb = a.bounces + 1;
    const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    double y[N];
    Cells cl{0, 0, 0, 0, 0};
    int bnc, kb, na, caustics;
    double D_prev = 0.0;
    long long steps;
    double s, tt, att, pt, pa, rmax;
    long long p_base = 0, p_cap = 0, p_n = 0;   // PATHS: this ray's row range and rows produced
    const double rad2deg = 180.0 / kPi;

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * (kPi / 180.0);
        const double phi = kPi / 2.0 - a.phi_deg[r] * (kPi / 180.0);
        ray_init_sph<AMP>(a, theta, phi, y);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        rmax = 0.0;
        if (PATHS && a.path_rows) { p_base = a.path_off[r]; p_cap = a.path_off[r + 1] - p_base; p_n = 0; }
    };
    start_ray(ray);

    while (true) {
        rmax = fmax(rmax, y[0] - a.r_earth);
        double ds = a.ds_max;   // set_ds (geoac.eqset.sph.rngdep.cpp:227-233)
        if (y[0] - a.r_earth < a.z_bl)
            ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - topo_r(a, vw, cl, y[1], y[2])) / 0.2);
        s += ds;
        double acc[N], stg[N], f[N];
        rhs_sphr<AMP, ST>(a, vw, cl, y, f);
        if (AMP && (a.aux || (PATHS && a.caus_rows)) && kb >= 1) {
            const double D = ray_det_sph(f, y);
            if (kb >= 2 && D * D_prev < 0.0) {
                caustics++;
                if (PATHS && a.caus_rows) {   // row kb; time through segment (kb-1, kb)
                    const unsigned long long w = atomicAdd(a.caus_count, 1ull);
                    if ((long long)w < a.caus_cap) {
                        double* o = a.caus_rows + w * kCausCols;
                        o[0] = y[1] * rad2deg; o[1] = y[2] * rad2deg; o[2] = y[0] - a.r_earth; o[3] = tt + pt;
                        o[4] = (double)bnc; o[5] = (double)ray; o[6] = (double)(steps + kb);
                    }
                }
            }
            D_prev = D;
        }
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
        rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_third; stg[i] = y[i] + t * 0.5; }
        rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_third; stg[i] = y[i] + t; }
        rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_sixth; }
        kb++;

        bool esc = s > a.s_max;
        if (!esc) {
            if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
            else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
            esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                  beyond_range(a, acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                  (acc[2] < a.lon_min || acc[2] > a.lon_max);
        }
        // ground_check (geoac.eqset.sph.rngdep.cpp:496-503)
        const bool gnd = !esc && (acc[0] - a.r_earth <= a.topo_zmax) && (acc[0] < topo_r(a, vw, cl, acc[1], acc[2]));

        double dt, da;
        seg_increment_sphr<ST>(a, vw, cl, y, acc, dt, da);
        if (a.write_rays) { tt += pt; att += pa; pt = dt; pa = da; }
        else { pt += dt; pa += da; }

        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(acc[0]) || !isfinite(acc[1]) || !isfinite(acc[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
            if (PATHS && a.path_rows && path_sampled(a.path_mode, kb)) {
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kPathCols;
                    Cells c2 = cl;
                    o[0] = y[1] * rad2deg; o[1] = y[2] * rad2deg;
                    o[2] = a.path_mode == kPathRays ? y[0] - a.r_earth : topo_r(a, vw, c2, y[1], y[2]) - a.r_earth;
                    o[3] = (AMP && a.path_mode == kPathRays)
                               ? amp_db_sphr<ST>(a, vw, c2, y, a.theta_deg[ray] * (kPi / 180.0),
                                             kPi / 2.0 - a.phi_deg[ray] * (kPi / 180.0), nullptr)
                               : 0.0;
                    o[4] = -2.0 * (att + pa); o[5] = tt + pt; o[6] = (double)bnc;
                }
                p_n++;
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.sph.rngdep.cpp:499-541) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        int status = -1;
        if (a.topo_tab == nullptr && rmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        else if (tt / 3600.0 > a.time_max_h) status = 6;
        if (status < 0) {
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            AtmPt mk;
            atm_point<ST>(a, vw, cl, acc[0], acc[1], acc[2], mk);
            // the range-dependent run_prop records +asin(...) (main.infraga.sph.rngdep.cpp:514),
            // infraga-sph -asin(...) (main.infraga.sph.cpp:523)
            const double incl = (ST ? -1.0 : 1.0) * asin(mk.c / a.c0 * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = acc[1] * (180.0 / kPi);
            out[4] = acc[2] * (180.0 / kPi);
            out[5] = tt;
            out[6] = gc_dist(a.r_earth, acc[1], acc[2], a.src_x, a.src_y, a.cos_lat_src) / tt;
            out[7] = rmax;
            out[8] = incl;
            out[9] = baz;
            double jac = 0.0;
            out[10] = AMP ? amp_db_sphr<ST>(a, vw, cl, acc, th_deg * (kPi / 180.0), kPi / 2.0 - ph_deg * (kPi / 180.0), &jac) : 0.0;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux_sph(ax, a, acc, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            reflect_sphr<N, AMP, ST>(a, vw, cl, y, prev);
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
    auto kern = fansphr_fp64_kernel<AMP, PATHS, ST>;
    const size_t smem = ((size_t)DimSph<AMP>::n * threads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
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
// solver, geoac.eigenray.sph.cpp:42-380): n_seg prop_rk4 segments from the
// launch source with terrain reflections between them.  Record mode sums
// time and absorption per step and the turning height over rows 1..k-1 from
// 0 (:230-268) and forms the arrival columns (:283-296), with the arrival
// inclination's c taken at a radius equal to the source ALTITUDE (clamped to
// the lowest knot under the source, :284); an amplitude trace also returns
// what the Newton derivatives read under the last row (:335-345): c at the
// source and on the ground, the ground radius and the terrain gradient.
// Same block size as the fan kernel (reflect_sphr reads row k-2 from shared
// memory with that stride).
template <bool AMP, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_SPHR_MINB) tracesphr_fp64_kernel(const __grid_constant__ Fan3DArgs a,
                                                                              const TraceReq* __restrict__ reqs,
                                                                              TraceRes18* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                              SegRes* __restrict__ seg_out,
                                                                              int seg_stride) {
    constexpr int N = DimSph<AMP>::n;
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
        ray_init_sph<AMP>(a, q.theta, q.phi, y);
        double tt = 0.0, att = 0.0, rmax = 0.0;
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
                if (record && kb >= 1) rmax = fmax(rmax, y[0] - a.r_earth);
                double ds = a.ds_max;
                if (y[0] - a.r_earth < a.z_bl)
                    ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - topo_r(a, vw, cl, y[1], y[2])) / 0.2);
                s += ds;
                double stg[N], f[N];
                rhs_sphr<AMP, ST>(a, vw, cl, y, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
                rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_third; stg[i] = y[i] + t * 0.5; }
                rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_third; stg[i] = y[i] + t; }
                rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * c_sixth; }
                kb++;
                esc = s > a.s_max;
                if (!esc) {
                    if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
                    else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
                    esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                          beyond_range(a, acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                          (acc[2] < a.lon_min || acc[2] > a.lon_max);
                }
                const bool gnd = !esc && (acc[0] - a.r_earth <= a.topo_zmax) && (acc[0] < topo_r(a, vw, cl, acc[1], acc[2]));
                if (record) {
                    double dt, da;
                    seg_increment_sphr<ST>(a, vw, cl, y, acc, dt, da);
                    tt += pt; att += pa; pt = dt; pa = da;
                }
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(acc[0]) || !isfinite(acc[1]) || !isfinite(acc[3])) esc = true;
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
                g.x = acc[1]; g.y = acc[2]; g.steps = steps; g.escaped = esc ? 1 : 0;
            }
            if (sg == q.n_seg - 1 || (esc && stop)) break;
            reflect_sphr<N, AMP, ST>(a, vw, cl, y, prev);
        }
        TraceRes18& o = out[r];
#pragma unroll
        for (int i = 0; i < 18; i++) o.y[i] = i < N ? acc[i] : 0.0;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        o.tt = o.att = o.zmax = o.amp_db = o.incl = o.baz = 0.0;
        o.c_src = a.c0; o.c_grnd = 0.0; o.z_grnd = 0.0; o.dzg[0] = 0.0; o.dzg[1] = 0.0;
        if (AMP && !record) {   // topo::z (a radius), topo::dz and atmo::c on the ground under the last row
            double rg = a.r_grnd;
            if (vw.has_topo) {
                TopoVal t;
                topo_eval(vw.topo, acc[1], acc[2], 1, t, cl.tx, cl.ty);
                rg = a.r_earth + t.z; o.dzg[0] = t.d[0]; o.dzg[1] = t.d[1];
            }
            o.z_grnd = rg;
            o.c_grnd = c_at<ST>(a, vw, cl, rg, acc[1], acc[2]);
        }
        if (record) {
            o.tt = tt; o.att = att; o.zmax = rmax;
            o.amp_db = AMP ? amp_db_sphr<ST>(a, vw, cl, acc, q.theta, q.phi, nullptr) : 0.0;
            const double c_k = c_at<ST>(a, vw, cl, acc[0], acc[1], acc[2]);
            const double c_s = c_at<ST>(a, vw, cl, a.src_z, a.src_x, a.src_y);   // r = the source altitude
            o.incl = -asin(c_k / c_s * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * (180.0 / kPi);
            while (baz < -180.0) baz += 360.0;
            while (baz > 180.0) baz -= 360.0;
            o.baz = baz;
        }
    }
}

template <bool AMP, bool ST>
cudaError_t launch_trace_impl(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, cudaStream_t st,
                              SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = tracesphr_fp64_kernel<AMP, ST>;
    const size_t smem = ((size_t)DimSph<AMP>::n * kThreads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
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

cudaError_t launch_fansphr_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    return a.knots ? launch_fan<true>(a, calc_amp, stream, grid_used) : launch_fan<false>(a, calc_amp, stream, grid_used);
}

cudaError_t launch_trace_sphr(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                              cudaStream_t st, SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (a.knots)
        return amp ? launch_trace_impl<true, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
                   : launch_trace_impl<false, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
    return amp ? launch_trace_impl<true, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
               : launch_trace_impl<false, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
}

}  // namespace iga
