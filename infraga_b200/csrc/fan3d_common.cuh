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
