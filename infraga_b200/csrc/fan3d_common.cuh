// Device helpers shared by the FP64 and FP32-compensated 3D stratified fan
// kernels (flat ground).
#pragma once
#include "fan3d.cuh"

namespace iga {

// Per-ray constants on flat ground: d(nu_x)/ds = d(nu_y)/ds = 0 and the x/y
// components of the mu equations vanish (geoac.eqset.3d.strat.cpp:353, 367,
// 382), and the flat-ground reflection keeps them, so they are fixed at launch.
struct RayConst {
    double nx, ny;             // nu_x, nu_y
    double mtx, mty, mpx, mpy; // mu_th_{x,y}, mu_ph_{x,y}
};


// Boundary-layer scaling of atmo::u/v (bndlyr_sc, atmo_state.3d.strat.cpp:85-92).
static __device__ __forceinline__ double bl_scale(const Fan3DArgs& a, double z) {
    if (z < a.z_bl) {
        const double X = exp(-(z - a.z0) * a.inv_bl);
        return (1.0 - X) / (1.0 + X);
    }
    return 1.0;
}

// Evolving state: 0 x, 1 y, 2 z, 3 nu_z, 4-6 X_th, 7 mu_th_z, 8-10 X_ph, 11 mu_ph_z.
template <bool AMP> struct Dim { static constexpr int n = AMP ? 12 : 4; };

// Above this height X = exp(-(z-zg)/0.1) < 1e-173 (see rhs()).
constexpr double kBlCutoffKm = 40.0;

// Right-hand side of the ray (and, with AMP, auxiliary) equations at state y:
// update_refs (geoac.eqset.3d.strat.cpp:225-328) + eval_src_eq (:333-389)
// with atmo::calc_uvw (atmo_state.3d.strat.cpp:462-734) on flat ground.
template <bool AMP>
static __device__ __forceinline__ void rhs(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                    const double* y, const RayConst& rc, double* f) {
    const double z = y[2];
    const double ze = fmin(fmax(z, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    double c, cz, czz = 0.0, u0, u0z, u0zz = 0.0, v0, v0z, v0zz = 0.0;
    if (AMP) {
        cubic_f2(r0, q, 2, c, cz, czz);
        cubic_f2(r0, q, 4, u0, u0z, u0zz);
        cubic_f2(r0, q, 6, v0, v0z, v0zz);
    } else {
        cubic_f1(r0, q, 2, c, cz);
        cubic_f1(r0, q, 4, u0, u0z);
        cubic_f1(r0, q, 6, v0, v0z);
    }
    // No-slip boundary-layer scaling S = (1-X)/(1+X), X = exp(-(z-zg)/bl).
    // The reference evaluates X at every altitude; more than 40 km above the
    // ground X < 1e-173, below half an ulp of every term it is added to
    // (S rounds to 1, the X-terms of S' and S'' vanish against the spline
    // derivatives), so X = 0 there gives the same doubles without the exp.
    const double hz = z - a.z0;
    const double Xb = hz < kBlCutoffKm ? exp(-hz * a.inv_bl) : 0.0;
    const double opX = 1.0 + Xb;
    const double iop = 1.0 / opX;
    const double sc0 = (1.0 - Xb) * iop;
    const double dX2 = -Xb * a.inv_bl;
    const double dsc2 = -2.0 * dX2 * (iop * iop);
    const double u = u0 * sc0, v = v0 * sc0;
    const double uz = u0z * sc0 + u0 * dsc2;
    const double vz = v0z * sc0 + v0 * dsc2;

    const double nz = y[3];
    const double num = sqrt(rc.nx * rc.nx + rc.ny * rc.ny + nz * nz);
    const double inum = 1.0 / num;
    const double cgx = c * rc.nx * inum + u;
    const double cgy = c * rc.ny * inum + v;
    const double cgz = c * nz * inum;
    const double cgm = sqrt(cgx * cgx + cgy * cgy + cgz * cgz);
    const double icg = 1.0 / cgm;
    f[0] = cgx * icg;
    f[1] = cgy * icg;
    f[2] = cgz * icg;
    const double Kz = num * cz + rc.nx * uz + rc.ny * vz;
    f[3] = -icg * Kz;
    if (AMP) {
        const double ddX22 = Xb * (a.inv_bl * a.inv_bl);
        const double ddsc22 = -2.0 * (ddX22 * (iop * iop) - 2.0 * dX2 * dX2 * (iop * iop * iop));
        const double uzz = u0zz * sc0 + 2.0 * u0z * dsc2 + u0 * ddsc22;
        const double vzz = v0zz * sc0 + 2.0 * v0z * dsc2 + v0 * ddsc22;
        const double Xtz = y[6], Xpz = y[10], mtz = y[7], mpz = y[11];
        const double dc3 = Xtz * cz, dc4 = Xpz * cz;
        const double du3 = Xtz * uz, du4 = Xpz * uz;
        // The reference adds the azimuth variation of v into dv[3] and
        // leaves dv[4] at zero (geoac.eqset.3d.strat.cpp:298).
        const double dv3 = Xtz * vz + Xpz * vz;
        const double dnu0 = (rc.nx * rc.mtx + rc.ny * rc.mty + nz * mtz) * inum;
        const double dnu1 = (rc.nx * rc.mpx + rc.ny * rc.mpy + nz * mpz) * inum;
        const double cin = c * inum, cin2 = cin * inum;
        const double g0x = rc.nx * inum * dc3 + cin * rc.mtx - cin2 * rc.nx * dnu0 + du3;
        const double g0y = rc.ny * inum * dc3 + cin * rc.mty - cin2 * rc.ny * dnu0 + dv3;
        const double g0z = nz * inum * dc3 + cin * mtz - cin2 * nz * dnu0;
        const double g1x = rc.nx * inum * dc4 + cin * rc.mpx - cin2 * rc.nx * dnu1 + du4;
        const double g1y = rc.ny * inum * dc4 + cin * rc.mpy - cin2 * rc.ny * dnu1;
        const double g1z = nz * inum * dc4 + cin * mpz - cin2 * nz * dnu1;
        const double dm0 = (cgx * g0x + cgy * g0y + cgz * g0z) * icg;
        const double dm1 = (cgx * g1x + cgy * g1y + cgz * g1z) * icg;
        const double icg2 = icg * icg;
        f[4] = g0x * icg - cgx * icg2 * dm0;
        f[5] = g0y * icg - cgy * icg2 * dm0;
        f[6] = g0z * icg - cgz * icg2 * dm0;
        f[8] = g1x * icg - cgx * icg2 * dm1;
        f[9] = g1y * icg - cgy * icg2 * dm1;
        f[10] = g1z * icg - cgz * icg2 * dm1;
        f[7] = dm0 * icg2 * Kz - icg * (dnu0 * cz + num * (Xtz * czz) + rc.mtx * uz + rc.mty * vz + rc.nx * (Xtz * uzz) + rc.ny * (Xtz * vzz));
        f[11] = dm1 * icg2 * Kz - icg * (dnu1 * cz + num * (Xpz * czz) + rc.mpx * uz + rc.mpy * vz + rc.nx * (Xpz * uzz) + rc.ny * (Xpz * vzz));
    }
}

// Travel-time and absorption increments of the segment y0 -> y1, evaluated at
// the segment midpoint (travel_time :486-511, atten :688-699, SB_alpha).
static __device__ __forceinline__ void seg_increment(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                              const double* y0, const double* y1, const RayConst& rc,
                                              double& dt, double& da) {
    const double dx = y1[0] - y0[0], dy = y1[1] - y0[1], dz = y1[2] - y0[2];
    const double zm = y0[2] + dz * 0.5;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double nzm = y0[3] + (y1[3] - y0[3]) * 0.5;
    const double num = sqrt(rc.nx * rc.nx + rc.ny * rc.ny + nzm * nzm);
    const double ze = fmin(fmax(zm, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale(a, zm);
    const double u = cubic_f(r0, q, 4) * sc;
    const double v = cubic_f(r0, q, 6) * sc;
    const double rho = cubic_f(r0, q, 8);
    const double inum = 1.0 / num;
    const double cgx = c * rc.nx * inum + u, cgy = c * rc.ny * inum + v, cgz = c * nzm * inum;
    dt = ds / sqrt(cgx * cgx + cgy * cgy + cgz * cgz);
    da = sb_alpha_cart(c, rho, zm, a.freq, a.tweak_abs, a.sb) * ds;
}

// geoac::travel_time_var of one segment, the (k1, k2) form run_back_proj
// calls (geoac.eqset.3d.strat.cpp:597-670): the inclination and azimuth
// variations of the travel-time increment from the midpoint state, with that
// form's sign (the sums are decremented, :644 and :668) and its product in
// place of a sum in the last term of d|c_g| (dcg[1] * cg[1] * dcg[2] * cg[2]).
// Flat ground: dc, du, dv have only z components, w = 0.
static __device__ __forceinline__ void seg_time_var(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                                    const double* y0, const double* y1, const RayConst& rc,
                                                    double& dvar_t, double& dvar_p) {
    const double dx = y1[0] - y0[0], dy = y1[1] - y0[1], dz = y1[2] - y0[2];
    const double zm = y0[2] + dz / 2.0;
    const double ds = sqrt(dx * dx + dy * dy + dz * dz);
    const double nu[3] = {rc.nx, rc.ny, y0[3] + (y1[3] - y0[3]) / 2.0};
    const double num = sqrt(nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2]);
    const double ze = fmin(fmax(zm, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    double c, cz, u0, u0z, v0, v0z;
    cubic_f1(r0, q, 2, c, cz);
    cubic_f1(r0, q, 4, u0, u0z);
    cubic_f1(r0, q, 6, v0, v0z);
    double sc = 1.0, dsc = 0.0;   // bndlyr_sc, bndlyr_dsc(n = 2) (atmo_state.3d.strat.cpp:87-112)
    if (zm < a.z_bl) {
        const double X = exp(-(zm - a.z0) * a.inv_bl);
        sc = (1.0 - X) / (1.0 + X);
        dsc = -2.0 * (-X * a.inv_bl) / ((1.0 + X) * (1.0 + X));
    }
    const double cg[3] = {c * nu[0] / num + u0 * sc, c * nu[1] / num + v0 * sc, c * nu[2] / num};
    const double cgm = sqrt(cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2]);
    const double duz = u0 * dsc + u0z * sc, dvz = v0 * dsc + v0z * sc;
    const double den = cgm * cgm * cgm;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int o = 4 * j;   // reduced state: X at 4..6 / 8..10, mu_z at 7 / 11
        const double X2 = y0[6 + o] + (y1[6 + o] - y0[6 + o]) / 2.0;
        const double mu[3] = {j == 0 ? rc.mtx : rc.mpx, j == 0 ? rc.mty : rc.mpy, y0[7 + o] + (y1[7 + o] - y0[7 + o]) / 2.0};
        const double s = X2 * cz - c / (num * num) * (mu[0] * nu[0] + mu[1] * nu[1] + mu[2] * nu[2]);
        double dcg[3];
#pragma unroll
        for (int i = 0; i < 3; i++) dcg[i] = nu[i] / num * s + c / num * mu[i];
        dcg[0] += X2 * duz;
        dcg[1] += X2 * dvz;
        const double v = -((dcg[0] * cg[0] + dcg[1] * cg[1] * dcg[2] * cg[2]) / den * ds);
        if (j == 0) dvar_t = v; else dvar_p = v;
    }
}

// Launch state of a ray: geoac::set_initial (geoac.eqset.3d.strat.cpp:58-105).
template <bool AMP>
static __device__ __forceinline__ void ray_init(const Fan3DArgs& a, double theta, double phi, double* y, RayConst& rc) {
    const double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
    const double mx = a.u0s / a.c0, my = a.v0s / a.c0;
    const double n0x = ct * cp, n0y = ct * sp, n0z = st;
    const double ms = 1.0 + (n0x * mx + n0y * my + n0z * 0.0);
    const double ims = 1.0 / ms, ims2 = ims * ims;
    y[0] = a.src_x; y[1] = a.src_y; y[2] = a.src_z;
    rc.nx = n0x * ims; rc.ny = n0y * ims; y[3] = n0z * ims;
    if (AMP) {
        const double tx = -st * cp, ty = -st * sp, tz = ct;
        const double px = -ct * sp, py = ct * cp, pz = 0.0;
        const double tm = tx * mx + ty * my + tz * 0.0;
        const double pm = px * mx + py * my + pz * 0.0;
        rc.mtx = tx * ims - n0x * ims2 * tm;
        rc.mty = ty * ims - n0y * ims2 * tm;
        y[7] = tz * ims - n0z * ims2 * tm;
        rc.mpx = px * ims - n0x * ims2 * pm;
        rc.mpy = py * ims - n0y * ims2 * pm;
        y[11] = pz * ims - n0z * ims2 * pm;
        y[4] = y[5] = y[6] = 0.0;
        y[8] = y[9] = y[10] = 0.0;
    } else {
        rc.mtx = rc.mty = rc.mpx = rc.mpy = 0.0;
    }
}

// geoac::amp with geoac::jacobian at the below-ground row
// (geoac.eqset.3d.strat.cpp:704-748).
static __device__ __noinline__ double amp_db(const double* __restrict__ tab, const Fan3DArgs& a, int& seg, const double* y,
                         const RayConst& rc, double theta, double phi, double* jac_out) {
    const double zk = y[2];
    const double ze = fmin(fmax(zk, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale(a, zk);
    const double wx = cubic_f(r0, q, 4) * sc, wy = cubic_f(r0, q, 6) * sc;
    const double rho = cubic_f(r0, q, 8);
    const double nz = y[3];
    const double num = sqrt(rc.nx * rc.nx + rc.ny * rc.ny + nz * nz);
    const double num0 = 1.0 - (rc.nx * a.u0s + rc.ny * a.v0s) / a.c0;
    const double cgx = c * rc.nx / num + wx, cgy = c * rc.ny / num + wy, cgz = c * nz / num;
    const double ct = cos(theta), st = sin(theta);
    const double g0x = a.c0 * ct * cos(phi) + a.u0s, g0y = a.c0 * ct * sin(phi) + a.v0s, g0z = a.c0 * st;
    const double cgm = sqrt(cgx * cgx + cgy * cgy + cgz * cgz);
    const double cgm0 = sqrt(g0x * g0x + g0y * g0y + g0z * g0z);
    const double ex = cgx / cgm, ey = cgy / cgm, ez = cgz / cgm;
    const double Xt[3] = {y[4], y[5], y[6]}, Xp[3] = {y[8], y[9], y[10]};
    const double jac = ex * (Xt[1] * Xp[2] - Xp[1] * Xt[2]) - Xt[0] * (ey * Xp[2] - ez * Xp[1]) + Xp[0] * (ey * Xt[2] - ez * Xt[1]);
    const double numr = rho * num * (c * c * c) * cgm0 * ct;
    const double den = a.rho0 * num0 * (a.c0 * a.c0 * a.c0) * cgm * jac;
    if (jac_out) *jac_out = jac;
    return 20.0 * log10(sqrt(fabs(numr / den)));
}

// geoac::jacobian (geoac.eqset.3d.strat.cpp:703-723) at state y: the unit
// group-velocity direction from c, u, v at the row's altitude and the
// position derivatives X_th, X_ph (the determinant amp_db also takes).
static __device__ __noinline__ double row_jacobian(const double* __restrict__ tab, const Fan3DArgs& a, int seg,
                                                   const double* y, const RayConst& rc) {
    const double zk = y[2];
    const double ze = fmin(fmax(zk, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double c = cubic_f(r0, q, 2);
    const double sc = bl_scale(a, zk);
    const double wx = cubic_f(r0, q, 4) * sc, wy = cubic_f(r0, q, 6) * sc;
    const double nz = y[3];
    const double num = sqrt(rc.nx * rc.nx + rc.ny * rc.ny + nz * nz);
    const double cgx = c * rc.nx / num + wx, cgy = c * rc.ny / num + wy, cgz = c * nz / num;
    const double cgm = sqrt(cgx * cgx + cgy * cgy + cgz * cgz);
    const double ex = cgx / cgm, ey = cgy / cgm, ez = cgz / cgm;
    const double Xt[3] = {y[4], y[5], y[6]}, Xp[3] = {y[8], y[9], y[10]};
    return ex * (Xt[1] * Xp[2] - Xp[1] * Xt[2]) - Xt[0] * (ey * Xp[2] - ez * Xp[1]) + Xp[0] * (ey * Xt[2] - ez * Xt[1]);
}

// geoac::eval_eikonal and geoac::eval_eikonal_deriv (geoac.eqset.3d.strat.cpp:
// 393-432) at state y (12-state layout) over flat ground, the print_resid
// diagnostics: eik = |nu| - c0 / c + (u nu_x + v nu_y) / c, and aux = the norm
// of the inclination and azimuth residuals of the auxiliary parameters.  The
// horizontal derivatives of c, u and v vanish over flat ground and w = 0, so
// only the z terms of the reference's sums remain; u, v and their
// z-derivatives carry the boundary-layer scaling as atmo::u / atmo::du do.
template <bool AMP>
__device__ __noinline__ void eikonal_resid(const double* __restrict__ tab, const Fan3DArgs& a, int seg, const double* y,
                                           const RayConst& rc, double& eik, double& aux) {
    const double z = y[2];
    const double ze = fmin(fmax(z, a.z_lo), a.z_hi);
    seg = seg_walk(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStride;
    const Cubic q = cubic_at(r0, ze);
    double c, cz, u0, u0z, v0, v0z;
    cubic_f1(r0, q, 2, c, cz);
    cubic_f1(r0, q, 4, u0, u0z);
    cubic_f1(r0, q, 6, v0, v0z);
    double sc = 1.0, dsc = 0.0;   // bndlyr_sc / bndlyr_dsc(n = 2) (atmo_state.3d.strat.cpp:85-112)
    if (z < a.z_bl) {
        const double X = exp(-(z - a.z0) / a.bl);
        sc = (1.0 - X) / (1.0 + X);
        dsc = -2.0 * (-X / a.bl) / ((1.0 + X) * (1.0 + X));
    }
    const double u = u0 * sc, v = v0 * sc;
    const double nu[3] = {rc.nx, rc.ny, y[3]};
    const double num = sqrt(nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2]);
    eik = num - a.c0 / c + (u * nu[0] + v * nu[1]) / c;
    aux = 0.0;
    if (AMP) {
        const double uz = u0 * dsc + u0z * sc, vz = v0 * dsc + v0z * sc;
        double r[2];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int o = 4 * j;   // X at 4..6 / 8..10, mu_z at 7 / 11
            const double Xz = y[6 + o];
            const double mu[3] = {j == 0 ? rc.mtx : rc.mpx, j == 0 ? rc.mty : rc.mpy, y[7 + o]};
            r[j] = (nu[0] * mu[0] + nu[1] * mu[1] + nu[2] * mu[2]) / num + num / c * (Xz * cz) +
                   1.0 / c * (mu[0] * u + mu[1] * v + nu[0] * (Xz * uz) + nu[1] * (Xz * vz));
        }
        aux = sqrt(r[0] * r[0] + r[1] * r[1]);
    }
}

// Per-arrival diagnostics at the below-ground row y (12-state layout,
// flat ground): launch-angle derivatives of the ground intercept as
// find_eigenray forms them (geoac.eigenray.3d.cpp:334-348), the Jacobian D
// and the caustic count.
__device__ __forceinline__ void write_aux(double* ax, const Fan3DArgs& a, const double* y, const RayConst& rc,
                                          double jac, int caustics) {
    const double ds_dth = -a.c0 / a.c_gnd * y[6] / y[3];
    const double ds_dph = -a.c0 / a.c_gnd * y[10] / y[3];
    const double dx_dth = y[4] + rc.nx * ds_dth, dy_dth = y[5] + rc.ny * ds_dth;
    const double dx_dph = y[8] + rc.nx * ds_dph, dy_dph = y[9] + rc.ny * ds_dph;
    ax[0] = sqrt(dx_dth * dx_dth + dy_dth * dy_dth);
    ax[1] = sqrt(dx_dph * dx_dph + dy_dph * dy_dph);
    ax[2] = jac;
    ax[3] = (double)caustics;
}

// Jacobian D from the ray direction (the stage-1 RHS f[0..2] = c_g/|c_g|) and
// the auxiliaries X_th (y[4..6]), X_ph (y[8..10]) (geoac::jacobian).
template <class T>
__device__ __forceinline__ T ray_jacobian(const T* f, const T* y) {
    return f[0] * (y[5] * y[10] - y[9] * y[6]) - y[4] * (f[1] * y[10] - f[2] * y[9]) + y[8] * (f[1] * y[6] - f[2] * y[5]);
}

}  // namespace iga
