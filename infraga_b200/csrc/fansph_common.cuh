// Device helpers of the spherical (global) stratified fan: flat ground at
// radius r_grnd = r_earth + z0 over a 1D profile.
//
// State layout, the reference's own (geoac.eqset.sph.strat.cpp:59-106):
//   0 r, 1 latitude, 2 longitude, 3-5 nu (r, lat, lon components),
//   6-8 d(r,lat,lon)/d(incl), 9-11 d(nu)/d(incl),
//   12-14 d(r,lat,lon)/d(az), 15-17 d(nu)/d(az).
// Without terrain nothing in this set is constant along a ray (the geometry
// terms T move nu_lat and nu_lon), so all 18 (6 without amplitude) are
// integrated.  The atmosphere depends on r only: the latitude/longitude
// derivatives of c, u, v and the vertical wind w are identically zero
// (atmo_state.sph.strat.cpp:498-612 with is_topo = false), so the reference's
// sums over those terms reduce to their r-parts exactly.
#pragma once
#include "fan3d.cuh"

namespace iga {

template <bool AMP> struct DimSph { static constexpr int n = AMP ? 18 : 6; };

// Above this height over the ground X = exp(-(r - r_grnd)/0.1) < 1e-173.
constexpr double kBlCutoffKmSph = 40.0;

// c, u, v (and their r-derivatives) at radius r, as update_refs sees them:
// spline values at z = r - r_earth clamped to the profile, winds scaled by the
// no-slip factor S = (1-X)/(1+X), X = exp(-(r - r_grnd)/bl), evaluated at
// every altitude like atmo::calc_uvw (atmo_state.sph.strat.cpp:498-560).
// More than 40 km above the ground X < 1e-173 and drops out of every sum it
// enters, so it is taken as 0 there (same doubles, no exp).
struct SphAtm {
    double c, cr, crr;
    double u, ur, urr;
    double v, vr, vrr;
};

template <bool D2>
static __device__ __forceinline__ void sph_atm(const double* __restrict__ tab, const Fan3DArgs& a, int& seg, double r,
                                               SphAtm& m) {
    const double ze = fmin(fmax(r - a.r_earth, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    double u0, u0z, u0zz = 0.0, v0, v0z, v0zz = 0.0;
    m.crr = 0.0;
    if (D2) {
        cubic_f2(r0, q, 2, m.c, m.cr, m.crr);
        cubic_f2(r0, q, 4, u0, u0z, u0zz);
        cubic_f2(r0, q, 6, v0, v0z, v0zz);
    } else {
        cubic_f1(r0, q, 2, m.c, m.cr);
        cubic_f1(r0, q, 4, u0, u0z);
        cubic_f1(r0, q, 6, v0, v0z);
    }
    const double hz = r - a.r_grnd;
    const double Xb = hz < kBlCutoffKmSph ? exp(-hz * a.inv_bl) : 0.0;
    const double iop = 1.0 / (1.0 + Xb);
    const double sc0 = (1.0 - Xb) * iop;
    const double dX = -Xb * a.inv_bl;
    const double dsc = -2.0 * dX * (iop * iop);
    m.u = u0 * sc0;
    m.v = v0 * sc0;
    m.ur = u0z * sc0 + u0 * dsc;
    m.vr = v0z * sc0 + v0 * dsc;
    m.urr = m.vrr = 0.0;
    if (D2) {
        const double ddX = Xb * (a.inv_bl * a.inv_bl);
        const double ddsc = -2.0 * (ddX * (iop * iop) - 2.0 * dX * dX * (iop * iop * iop));
        m.urr = u0zz * sc0 + 2.0 * u0z * dsc + u0 * ddsc;
        m.vrr = v0zz * sc0 + 2.0 * v0z * dsc + v0 * ddsc;
    }
}

// Right-hand side at state y: update_refs (geoac.eqset.sph.strat.cpp:227-371)
// followed by eval_src_eq (:375-433), with the zero lat/lon derivatives and
// w = 0 of a stratified atmosphere dropped.
template <bool AMP>
static __device__ __forceinline__ void rhs_sph(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                               const double* y, double* f) {
    SphAtm m;
    sph_atm<AMP>(tab, a, seg, y[0], m);
    const double r = y[0];
    double st, ct;
    sincos(y[1], &st, &ct);
    const double ir = 1.0 / r;
    const double ict = 1.0 / ct;
    const double tnt = st * ict;
    const double n0 = y[3], n1 = y[4], n2 = y[5];
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double inum = 1.0 / num;
    const double cg0 = m.c * n0 * inum;
    const double cg1 = m.c * n1 * inum + m.v;
    const double cg2 = m.c * n2 * inum + m.u;
    const double cgm = sqrt(cg0 * cg0 + cg1 * cg1 + cg2 * cg2);
    const double icg = 1.0 / cgm;
    const double G1 = ir, G2 = ir * ict;
    const double T0 = -ir * (n1 * cg1 + n2 * cg2);
    const double T1 = n0 * m.v + n0 * cg1 + n2 * cg2 * tnt;
    const double T2 = n0 * m.u * ct + (n1 * m.u - n2 * m.v) * st + cg2 * (n0 * ct - n1 * st);
    const double K0 = num * m.cr + n1 * m.vr + n2 * m.ur;
    f[0] = cg0 * icg;
    f[1] = G1 * cg1 * icg;
    f[2] = G2 * cg2 * icg;
    f[3] = -icg * (K0 + T0);
    f[4] = -G1 * icg * T1;
    f[5] = -G2 * icg * T2;
    if (AMP) {
        const double icg2 = icg * icg;
        const double ir2 = ir * ir;
        const double cin = m.c * inum, cin2 = cin * inum;
#pragma unroll
        for (int j = 0; j < 2; j++) {   // j = 0: inclination, 1: azimuth
            const double* R = y + 6 + 6 * j;
            const double* mu = y + 9 + 6 * j;
            const double dc = R[0] * m.cr, du = R[0] * m.ur, dv = R[0] * m.vr;
            const double dnu = (n0 * mu[0] + n1 * mu[1] + n2 * mu[2]) * inum;
            const double g0 = n0 * inum * dc + cin * mu[0] - cin2 * n0 * dnu;
            const double g1 = n1 * inum * dc + cin * mu[1] - cin2 * n1 * dnu + dv;
            const double g2 = n2 * inum * dc + cin * mu[2] - cin2 * n2 * dnu + du;
            const double dm = (cg0 * g0 + cg1 * g1 + cg2 * g2) * icg;
            const double dG1 = -R[0] * ir2;
            const double dG2 = -R[0] * ir2 * ict + st * ir * ict * ict * R[1];
            const double dT0 = R[0] * ir2 * (n1 * cg1 + n2 * cg2) - ir * (mu[1] * cg1 + n1 * g1 + mu[2] * cg2 + n2 * g2);
            const double dT1 = (mu[0] * m.v + n0 * dv) + mu[0] * cg1 + n0 * g1 + (mu[2] * cg2 + n2 * g2) * tnt +
                               n2 * cg2 * R[1] * ict * ict;
            const double dT2 = (mu[0] * m.u + n0 * du) * ct - (n0 * m.u) * R[1] * st +
                               (mu[1] * m.u + n1 * du - mu[2] * m.v - n2 * dv) * st + (n1 * m.u - n2 * m.v) * R[1] * ct +
                               g2 * (n0 * ct - n1 * st) + cg2 * ((mu[0] - n1 * R[1]) * ct - (mu[1] + n0 * R[1]) * st);
            double* fR = f + 6 + 6 * j;
            double* fm = f + 9 + 6 * j;
            fR[0] = g0 * icg - cg0 * icg2 * dm;
            fR[1] = dG1 * cg1 * icg + G1 * g1 * icg - G1 * cg1 * icg2 * dm;
            fR[2] = dG2 * cg2 * icg + G2 * g2 * icg - G2 * cg2 * icg2 * dm;
            fm[0] = icg2 * dm * K0 -
                    icg * (dnu * m.cr + num * (R[0] * m.crr) + mu[1] * m.vr + mu[2] * m.ur + n1 * (R[0] * m.vrr) +
                           n2 * (R[0] * m.urr) + dT0);
            fm[1] = -dG1 * icg * T1 - G1 * icg * dT1;
            fm[2] = -dG2 * icg * T2 - G2 * icg * dT2;
        }
    }
}

// Winds as atmo::u/v return them (bndlyr_sc applied only below z_bndlyr,
// atmo_state.sph.strat.cpp:100-108): used by travel_time, jacobian and amp.
static __device__ __forceinline__ double bl_scale_sph(const Fan3DArgs& a, double r) {
    if (r - a.r_earth < a.z_bl) {
        const double X = exp(-(r - a.r_grnd) * a.inv_bl);
        return (1.0 - X) / (1.0 + X);
    }
    return 1.0;
}

// Great-circle distance (globe::gc_dist, util/globe.cpp:23-28).
static __device__ __forceinline__ double gc_dist(double r_earth, double lat1, double lon1, double lat2, double lon2,
                                                 double cos_lat2) {
    const double s1 = sin((lat2 - lat1) * 0.5), s2 = sin((lon2 - lon1) * 0.5);
    return 2.0 * r_earth * asin(sqrt(s1 * s1 + cos(lat1) * cos_lat2 * (s2 * s2)));
}

// Range test of break_check: gc_dist > rng_max.  asin(sqrt(h)) is increasing,
// so away from the threshold the haversine h decides it; within 1e-9 of the
// threshold the distance itself is formed and compared.
static __device__ __forceinline__ bool beyond_range(const Fan3DArgs& a, double lat, double lon) {
    const double s1 = sin((a.src_x - lat) * 0.5), s2 = sin((a.src_y - lon) * 0.5);
    const double h = s1 * s1 + cos(lat) * a.cos_lat_src * (s2 * s2);
    if (!a.rng_exact_only && fabs(h - a.hav_rng) > 1e-9 * a.hav_rng) return h > a.hav_rng;
    return 2.0 * a.r_earth * asin(sqrt(h)) > a.rng_max;
}

// Travel-time and absorption increments of the segment y0 -> y1 at its
// midpoint (travel_time :549-581, atten :777-797, SB_alpha sph).
static __device__ __forceinline__ void seg_increment_sph(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                                         const double* y0, const double* y1, double& dt_out,
                                                         double& da_out) {
    const double dr = y1[0] - y0[0];
    const double rm = y0[0] + dr * 0.5;
    const double dth = y1[1] - y0[1];
    const double tm = y0[1] + dth * 0.5;
    double dp = y1[2] - y0[2];
    if (dp > kPi) dp -= 2.0 * kPi;
    else if (dp < -kPi) dp += 2.0 * kPi;
    const double a1 = rm * dth, a2 = rm * cos(tm) * dp;
    const double ds = sqrt(dr * dr + a1 * a1 + a2 * a2);
    const double n0 = y0[3] + (y1[3] - y0[3]) * 0.5;
    const double n1 = y0[4] + (y1[4] - y0[4]) * 0.5;
    const double n2 = y0[5] + (y1[5] - y0[5]) * 0.5;
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double zm = rm - a.r_earth;
    const double ze = fmin(fmax(zm, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale_sph(a, rm);
    const double u = cubic_f(r0, q, 4) * sc;
    const double v = cubic_f(r0, q, 6) * sc;
    const double rho = cubic_f(r0, q, 8);
    const double inum = 1.0 / num;
    const double cp0 = c * n0 * inum, cp1 = c * n1 * inum + v, cp2 = c * n2 * inum + u;
    dt_out = ds / sqrt(cp0 * cp0 + cp1 * cp1 + cp2 * cp2);
    da_out = sb_alpha<true>(c, rho, zm, a.freq, a.tweak_abs, a.sb) * ds;
}

// Launch state: geoac::set_initial (geoac.eqset.sph.strat.cpp:59-106).
// theta/phi in radians (phi measured from east, as geoac::phi).
template <bool AMP>
static __device__ __forceinline__ void ray_init_sph(const Fan3DArgs& a, double theta, double phi, double* y) {
    double st, ct, sp, cp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    const double mt = a.v0s / a.c0, mp = a.u0s / a.c0;   // (w, v, u) / c0 with w = 0
    const double n0 = st, n1 = ct * sp, n2 = ct * cp;
    const double ms = 1.0 + (n0 * 0.0 + n1 * mt + n2 * mp);
    y[0] = a.r_earth + a.src_z;
    y[1] = a.src_x;
    y[2] = a.src_y;
    // once per ray: divide as the reference does
    y[3] = n0 / ms; y[4] = n1 / ms; y[5] = n2 / ms;
    if (AMP) {
        const double ms2 = ms * ms;
        const double l0 = ct, l1 = -st * sp, l2 = -st * cp;   // d(nu0)/d(incl)
        const double p0 = 0.0, p1 = ct * cp, p2 = -ct * sp;   // d(nu0)/d(az)
        const double lm = l0 * 0.0 + l1 * mt + l2 * mp;
        const double pm = p0 * 0.0 + p1 * mt + p2 * mp;
        y[6] = y[7] = y[8] = 0.0;
        y[9] = l0 / ms - n0 / ms2 * lm;
        y[10] = l1 / ms - n1 / ms2 * lm;
        y[11] = l2 / ms - n2 / ms2 * lm;
        y[12] = y[13] = y[14] = 0.0;
        y[15] = p0 / ms - n0 / ms2 * pm;
        y[16] = p1 / ms - n1 / ms2 * pm;
        y[17] = p2 / ms - n2 / ms2 * pm;
    }
}

// geoac::amp with geoac::jacobian at the below-ground row y
// (geoac.eqset.sph.strat.cpp:800-852); returns 20 log10(amp).
static __device__ __noinline__ double amp_db_sph(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                                 const double* y, double theta, double phi, double* jac_out) {
    const double r = y[0];
    const double ze = fmin(fmax(r - a.r_earth, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale_sph(a, r);
    const double u = cubic_f(r0, q, 4) * sc, v = cubic_f(r0, q, 6) * sc;
    const double rho = cubic_f(r0, q, 8);
    const double n0 = y[3], n1 = y[4], n2 = y[5];
    // source side
    double st, ct, sp, cp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    const double ms = 1.0 + (st * 0.0 + ct * sp * (a.v0s / a.c0) + ct * cp * (a.u0s / a.c0));
    const double nu0 = 1.0 / ms;
    const double e0 = nu0 * st, e1 = nu0 * ct * sp, e2 = nu0 * ct * cp;
    const double g0 = a.c0 * e0 / nu0, g1 = a.c0 * e1 / nu0 + a.v0s, g2 = a.c0 * e2 / nu0 + a.u0s;
    const double cgm0 = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
    // receiver side (nu_mag from the eikonal with the source's c0)
    const double numag = (a.c0 - n1 * v - n2 * u) / c;
    const double p0 = c * n0 / numag, p1 = c * n1 / numag + v, p2 = c * n2 / numag + u;
    const double cpm = sqrt(p0 * p0 + p1 * p1 + p2 * p2);
    // jacobian(solution, k)
    const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double j0 = c * n0 / nm, j1 = c * n1 / nm + v, j2 = c * n2 / nm + u;
    const double jm = sqrt(j0 * j0 + j1 * j1 + j2 * j2);
    const double cl = cos(y[1]);
    const double dr_ds = j0 / jm, dt_ds = 1.0 / r * j1 / jm, dp_ds = 1.0 / (r * cl) * j2 / jm;
    const double* Rt = y + 6;
    const double* Rp = y + 12;
    const double jac = r * r * cl *
                       (dr_ds * (Rt[1] * Rp[2] - Rp[1] * Rt[2]) - Rt[0] * (dt_ds * Rp[2] - dp_ds * Rp[1]) +
                        Rp[0] * (dt_ds * Rt[2] - dp_ds * Rt[1]));
    const double numr = rho * numag * (c * c * c) * cgm0 * ct;
    const double den = a.rho0 * nu0 * (a.c0 * a.c0 * a.c0) * cpm * jac;
    if (jac_out) *jac_out = jac;
    return 20.0 * log10(sqrt(fabs(numr / den)));
}

// geoac::jacobian (geoac.eqset.sph.strat.cpp:800-822) at state y (18-state
// layout): the unit group-velocity direction in (r, lat, lon) rates and the
// position derivatives, scaled by r^2 cos(lat) (the determinant amp_db_sph
// also takes).
static __device__ __noinline__ double row_jacobian_sph(const double* __restrict__ tab, const Fan3DArgs& a, int seg,
                                                       const double* y) {
    const double r = y[0];
    const double ze = fmin(fmax(r - a.r_earth, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale_sph(a, r);
    const double u = cubic_f(r0, q, 4) * sc, v = cubic_f(r0, q, 6) * sc;
    const double n0 = y[3], n1 = y[4], n2 = y[5];
    const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double j0 = c * n0 / nm, j1 = c * n1 / nm + v, j2 = c * n2 / nm + u;
    const double jm = sqrt(j0 * j0 + j1 * j1 + j2 * j2);
    const double cl = cos(y[1]);
    const double dr_ds = j0 / jm, dt_ds = 1.0 / r * j1 / jm, dp_ds = 1.0 / (r * cl) * j2 / jm;
    const double* Rt = y + 6;
    const double* Rp = y + 12;
    return r * r * cl *
           (dr_ds * (Rt[1] * Rp[2] - Rp[1] * Rt[2]) - Rt[0] * (dt_ds * Rp[2] - dp_ds * Rp[1]) +
            Rp[0] * (dt_ds * Rt[2] - dp_ds * Rt[1]));
}

// Per-arrival diagnostics (18-state layout): launch-angle derivatives of the
// ground intercept as the spherical find_eigenray forms them
// (geoac.eigenray.sph.cpp:351-359, flat ground), as ground distance per
// radian [km/rad]; the Jacobian D and the caustic count.
__device__ __forceinline__ void write_aux_sph(double* ax, const Fan3DArgs& a, const double* y, double jac,
                                              int caustics) {
    const double ds_dth = a.refl_mcr * y[6] / y[3];
    const double ds_dph = a.refl_mcr * y[12] / y[3];
    const double cl = cos(y[1]);
    const double rgc = a.r_grnd * cl;
    const double dlat_dth = y[7] + y[4] / a.r_grnd * ds_dth, dlon_dth = y[8] + y[5] / rgc * ds_dth;
    const double dlat_dph = y[13] + y[4] / a.r_grnd * ds_dph, dlon_dph = y[14] + y[5] / rgc * ds_dph;
    const double x0 = a.r_grnd * dlat_dth, x1 = rgc * dlon_dth;
    const double x2 = a.r_grnd * dlat_dph, x3 = rgc * dlon_dph;
    ax[0] = sqrt(x0 * x0 + x1 * x1);
    ax[1] = sqrt(x2 * x2 + x3 * x3);
    ax[2] = jac;
    ax[3] = (double)caustics;
}

// Sign-carrying Jacobian determinant from the stage-1 RHS direction f[0..2]
// = (dr/ds, dlat/ds, dlon/ds) and the auxiliaries (caustic counting; the
// positive factor r^2 cos(lat) is left out).
__device__ __forceinline__ double ray_det_sph(const double* f, const double* y) {
    const double* Rt = y + 6;
    const double* Rp = y + 12;
    return f[0] * (Rt[1] * Rp[2] - Rp[1] * Rt[2]) - Rt[0] * (f[1] * Rp[2] - f[2] * Rp[1]) +
           Rp[0] * (f[1] * Rt[2] - f[2] * Rt[1]);
}

}  // namespace iga
