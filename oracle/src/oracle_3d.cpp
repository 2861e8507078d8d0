// CPU oracle (test infrastructure only; never linked into the product).
//
// Restatement of the reference's 3D Cartesian stratified ray-fan solver on
// flat ground, one function per reference function, same operation order:
//
//   boundary-layer scaling   atmo_state.3d.strat.cpp:85-142 (bndlyr_sc/dsc)
//   atmo::c/u/v/w/rho        atmo_state.3d.strat.cpp:148-456
//   atmo::calc_uvw           atmo_state.3d.strat.cpp:462-734 (9- and 12-arg)
//   atmo::SB_alpha           atmo_state.abs.cart.cpp:12-142
//   geoac::set_initial       geoac.eqset.3d.strat.cpp:58-105
//   geoac::approx_intercept  geoac.eqset.3d.strat.cpp:110-117
//   geoac::set_refl          geoac.eqset.3d.strat.cpp:122-209
//   geoac::set_ds            geoac.eqset.3d.strat.cpp:214-220
//   geoac::update_refs       geoac.eqset.3d.strat.cpp:225-328
//   geoac::eval_src_eq       geoac.eqset.3d.strat.cpp:333-389
//   break/ground_check       geoac.eqset.3d.strat.cpp:438-453
//   travel_time, atten       geoac.eqset.3d.strat.cpp:463-513, 676-699
//   jacobian, amp            geoac.eqset.3d.strat.cpp:704-748
//   geoac::prop_rk4          util/rk4solver.cpp:14-85
//   bounce loop + arrival    main.infraga.3d.cpp:421-540
//
// The reference keeps every RK4 row of a bounce and sums travel time and
// absorption in a post-pass (main.infraga.3d.cpp:451-488); this restatement
// keeps the last three rows and sums each segment as it is produced, in the
// same order, which gives the same sums.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <thread>
#include "oracle_atmo.h"
#include "oracle_api.h"

namespace orc {
namespace d3 {

struct Atmo {
    Profile P;
    double z0 = 0.0, z_max = 0.0, z_bndlyr = 2.0;   // topo::z0, z_max, z_bndlyr (flat ground)
    double bl = 0.1;                                 // topo::bndlyr_param
    double tweak_abs = 1.0;
};

struct Refs {   // geoac::src_refs (geoac.eqset.3d.strat.cpp:31-53)
    double src_loc[3]; double c0;
    double c; double dc[5]; double ddc[3][2];
    double u; double du[5]; double ddu[3][2];
    double v; double dv[5]; double ddv[3][2];
    double w; double dw[5]; double ddw[3][2];
    double nu0; double nu_mag; double dnu_mag[2];
    double cg[3]; double cg_mag; double dcg[3][2]; double dcg_mag[2];
};

struct Ray {
    const Atmo* A;
    const orc_fan_cfg* cfg;
    bool calc_amp;
    int eq_cnt;
    double theta, phi;
    Refs refs;
    int acc_c = 0, acc_u = 0, acc_v = 0, acc_rho = 0;
    double D_prev = 0.0;
};

// ---- topography on flat ground (atmo_state.3d.strat.cpp:51-83) ----
static inline double topo_z(const Ray& r, double, double) { return r.A->z0; }
static inline double topo_dz(const Ray&, double, double, int) { return 0.0; }
static inline double topo_ddz(const Ray&, double, double, int, int) { return 0.0; }

// ---- boundary-layer scaling (atmo_state.3d.strat.cpp:85-142) ----
static double bndlyr_sc(const Ray& r, double x, double y, double z) {
    double X, result = 1.0;
    if (z < r.A->z_bndlyr) {
        X = exp(-(z - topo_z(r, x, y)) / r.A->bl);
        result = (1.0 - X) / (1.0 + X);
    }
    return result;
}
static double bndlyr_dsc(const Ray& r, double x, double y, double z, int n) {
    double X, dX, result = 0.0;
    if (z < r.A->z_bndlyr) {
        X = exp(-(z - topo_z(r, x, y)) / r.A->bl);
        if (n < 2) dX = X / r.A->bl * topo_dz(r, x, y, n);
        else dX = -X / r.A->bl;
        result = -2.0 * dX / pow(1.0 + X, 2);
    }
    return result;
}

// ---- atmosphere (atmo_state.3d.strat.cpp:148-233) ----
static double a_rho(Ray& r, double, double, double z) {
    const Spline1D& s = r.A->P.rho;
    return eval_f(in_interval(z, s.x[0], s.x[s.n - 1]), s, r.acc_rho);
}
static double a_c(Ray& r, double, double, double z) {
    const Spline1D& s = r.A->P.c;
    return eval_f(in_interval(z, s.x[0], s.x[s.n - 1]), s, r.acc_c);
}
static double a_dc(Ray& r, double, double, double z, int n) {
    const Spline1D& s = r.A->P.c;
    double result = 0.0;
    if (n == 2) result = eval_df(in_interval(z, s.x[0], s.x[s.n - 1]), s, r.acc_c);
    return result;
}
static double a_u(Ray& r, double x, double y, double z) {
    const Spline1D& s = r.A->P.u;
    return eval_f(in_interval(z, s.x[0], s.x[s.n - 1]), s, r.acc_u) * bndlyr_sc(r, x, y, z);
}
static double a_du(Ray& r, double x, double y, double z, int n) {
    const Spline1D& s = r.A->P.u;
    double ze = in_interval(z, s.x[0], s.x[s.n - 1]);
    double result = eval_f(ze, s, r.acc_u) * bndlyr_dsc(r, x, y, z, n);
    if (n == 2) result += eval_df(ze, s, r.acc_u) * bndlyr_sc(r, x, y, z);
    return result;
}
static double a_v(Ray& r, double x, double y, double z) {
    const Spline1D& s = r.A->P.v;
    return eval_f(in_interval(z, s.x[0], s.x[s.n - 1]), s, r.acc_v) * bndlyr_sc(r, x, y, z);
}
static double a_dv(Ray& r, double x, double y, double z, int n) {
    const Spline1D& s = r.A->P.v;
    double ze = in_interval(z, s.x[0], s.x[s.n - 1]);
    double result = eval_f(ze, s, r.acc_v) * bndlyr_dsc(r, x, y, z, n);
    if (n == 2) result += eval_df(ze, s, r.acc_v) * bndlyr_sc(r, x, y, z);
    return result;
}
// atmo::w and dw are zero without terrain (atmo_state.3d.strat.cpp:235-456).
static double a_w(Ray&, double, double, double) { return 0.0; }
static double a_dw(Ray&, double, double, double, int) { return 0.0; }

// atmo::calc_uvw, 9-argument form (atmo_state.3d.strat.cpp:462-554), flat ground.
static void calc_uvw9(Ray& r, double x, double y, double z, double& u, double& v, double& w,
                      double du[3], double dv[3], double dw[3]) {
    const Atmo& A = *r.A;
    double zg, dzg[2], u0, v0, du_temp, du0[3], dv0[3], X, dX[3], sc0, dsc0[3];
    double ze = in_interval(z, A.P.u.x[0], A.P.u.x[A.P.u.n - 1]);
    zg = topo_z(r, x, y);
    dzg[0] = dzg[1] = 0.0;
    eval_all(ze, A.P.u, r.acc_u, u0, du_temp);
    du0[0] = du0[1] = 0.0; du0[2] = du_temp;
    eval_all(ze, A.P.v, r.acc_v, v0, du_temp);
    dv0[0] = dv0[1] = 0.0; dv0[2] = du_temp;
    X = exp(-(z - zg) / A.bl);
    for (int n = 0; n < 2; n++) dX[n] = X / A.bl * dzg[n];
    dX[2] = -X / A.bl;
    sc0 = (1.0 - X) / (1.0 + X);
    for (int n = 0; n < 3; n++) dsc0[n] = -2.0 * dX[n] / pow(1.0 + X, 2);
    u = u0 * sc0;
    v = v0 * sc0;
    for (int n = 0; n < 3; n++) {
        du[n] = du0[n] * sc0 + u0 * dsc0[n];
        dv[n] = dv0[n] * sc0 + v0 * dsc0[n];
    }
    w = 0.0;
    for (int n = 0; n < 3; n++) dw[n] = 0.0;
}

// atmo::calc_uvw, 12-argument form (atmo_state.3d.strat.cpp:556-734), flat ground.
static void calc_uvw12(Ray& r, double x, double y, double z, double& u, double& v, double& w,
                       double du[3], double dv[3], double dw[3], double ddu[6], double ddv[6], double ddw[6]) {
    const Atmo& A = *r.A;
    const double bl = A.bl;
    double zg, dzg[2], ddzg[2][2];
    double u0, v0, du0[3], dv0[3], ddu0[3][3], ddv0[3][3], du_temp, ddu_temp;
    double X, dX[3], ddX[3][3], sc0, dsc0[3], ddsc0[3][3];
    double ze = in_interval(z, A.P.u.x[0], A.P.u.x[A.P.u.n - 1]);
    zg = topo_z(r, x, y);
    for (int n = 0; n < 2; n++) { dzg[n] = 0.0; for (int m = 0; m < 2; m++) ddzg[n][m] = 0.0; }
    eval_all(ze, A.P.u, r.acc_u, u0, du_temp, ddu_temp);
    for (int n = 0; n < 3; n++) { du0[n] = 0.0; for (int m = 0; m < 3; m++) ddu0[n][m] = 0.0; }
    du0[2] = du_temp; ddu0[2][2] = ddu_temp;
    eval_all(ze, A.P.v, r.acc_v, v0, du_temp, ddu_temp);
    for (int n = 0; n < 3; n++) { dv0[n] = 0.0; for (int m = 0; m < 3; m++) ddv0[n][m] = 0.0; }
    dv0[2] = du_temp; ddv0[2][2] = ddu_temp;

    X = exp(-(z - zg) / bl);
    for (int n = 0; n < 2; n++) {
        dX[n] = X / bl * dzg[n];
        for (int m = n; m < 3; m++) {
            if (m < 2) ddX[n][m] = X / bl * (ddzg[n][m] + 1.0 / bl * dzg[n] * dzg[m]);
            else ddX[n][m] = -X / pow(bl, 2) * dzg[n];
            ddX[m][n] = ddX[n][m];
        }
    }
    dX[2] = -X / bl;
    ddX[2][2] = X / pow(bl, 2);
    sc0 = (1.0 - X) / (1.0 + X);
    for (int n = 0; n < 3; n++) {
        dsc0[n] = -2.0 * dX[n] / pow(1.0 + X, 2);
        for (int m = n; m < 3; m++) {
            ddsc0[n][m] = -2.0 * (ddX[n][m] / pow(1.0 + X, 2) - 2.0 * dX[n] * dX[m] / pow(1.0 + X, 3));
            ddsc0[m][n] = ddsc0[n][m];
        }
    }
    u = u0 * sc0;
    v = v0 * sc0;
    for (int n = 0; n < 3; n++) {
        du[n] = du0[n] * sc0 + u0 * dsc0[n];
        dv[n] = dv0[n] * sc0 + v0 * dsc0[n];
        ddu[n] = ddu0[n][n] * sc0 + 2.0 * du0[n] * dsc0[n] + u0 * ddsc0[n][n];
        ddv[n] = ddv0[n][n] * sc0 + 2.0 * dv0[n] * dsc0[n] + v0 * ddsc0[n][n];
    }
    ddu[3] = ddu0[0][1] * sc0 + du0[0] * dsc0[1] + du0[1] * dsc0[0] + u0 * ddsc0[0][1];
    ddu[4] = ddu0[0][2] * sc0 + du0[0] * dsc0[2] + du0[2] * dsc0[0] + u0 * ddsc0[0][2];
    ddu[5] = ddu0[1][2] * sc0 + du0[1] * dsc0[2] + du0[2] * dsc0[1] + u0 * ddsc0[1][2];
    ddv[3] = ddv0[0][1] * sc0 + dv0[0] * dsc0[1] + dv0[1] * dsc0[0] + v0 * ddsc0[0][1];
    ddv[4] = ddv0[0][2] * sc0 + dv0[0] * dsc0[2] + dv0[2] * dsc0[0] + v0 * ddsc0[0][2];
    ddv[5] = ddv0[1][2] * sc0 + dv0[1] * dsc0[2] + dv0[2] * dsc0[1] + v0 * ddsc0[1][2];
    w = 0.0;
    for (int n = 0; n < 3; n++) dw[n] = 0.0;
    for (int n = 0; n < 6; n++) ddw[n] = 0.0;
}

// atmo::SB_alpha (atmo_state.abs.cart.cpp:12-142), including the reference's
// pow(z, 2) in the z^4 term of the N profile (line 78).
double sb_alpha_cart(double c_kms, double rho_gcc, double z, double freq, double tweak_abs) {
    int m;
    double T_o, P_o, S;
    double X[7], X_ON, Z_rot[2], Z_rot_;
    double sigma, nn, chi, cchi, mu, nu, mu_o;
    double beta_0, beta_1, beta_2, alpha_1, alpha_2;
    double a_cl, a_rot, a_vib;
    double T_z, P_z, c_snd_z;
    double A1, A2, B, C, D, E, F, G, H, I, J, K, L, ZZ, hu;
    double f_vib[4], Cp_R[4], Cv_R[4], theta[4], C_R, A_max, Tr;
    mu_o = 18.192e-6; T_o = 293.15; P_o = 101325; S = 117.0;
    Cv_R[0] = 5.0 / 2.0; Cv_R[1] = 5.0 / 2.0; Cv_R[2] = 3.0; Cv_R[3] = 3.0;
    Cp_R[0] = 7.0 / 2.0; Cp_R[1] = 7.0 / 2.0; Cp_R[2] = 4.0; Cp_R[3] = 4.0;
    theta[0] = 2239.1; theta[1] = 3352.0; theta[2] = 915.0; theta[3] = 1037.0;

    T_z = pow(c_kms * 1.0e3, 2) / (kR * kGam);
    P_z = rho_gcc * 1.0e3 * pow(c_kms * 1.0e3, 2) / kGam;
    c_snd_z = c_kms * 1.0e3;
    mu = mu_o * sqrt(T_z / T_o) * ((1.0 + S / T_o) / (1.0 + S / T_z));
    nu = (8.0 * kPi * freq * mu) / (3.0 * P_z);

    if (z > 90.0) X[0] = pow(10.0, 49.296 - (1.5524 * z) + (1.8714e-2 * pow(z, 2)) - (1.1069e-4 * pow(z, 3)) + (3.199e-7 * pow(z, 4)) - (3.6211e-10 * pow(z, 5)));
    else X[0] = pow(10.0, -0.67887);
    if (z > 76.0) X[1] = pow(10.0, (1.3972e-1) - (5.6269e-3 * z) + (3.9407e-5 * pow(z, 2)) - (1.0737e-7 * pow(z, 3)));
    else X[1] = pow(10.0, -0.10744);
    X[2] = pow(10.0, -3.3979);
    if (z > 80.0) X[3] = pow(10.0, -4.234 - (3.0975e-2 * z));
    else X[3] = pow(10.0, -19.027 + (1.3093 * z) - (4.6496e-2 * pow(z, 2)) + (7.8543e-4 * pow(z, 3)) - (6.5169e-6 * pow(z, 4)) + (2.1343e-8 * pow(z, 5)));
    if (z > 95.0) X[4] = pow(10.0, -3.2456 + (4.6642e-2 * z) - (2.6894e-4 * pow(z, 2)) + (5.264e-7 * pow(z, 3)));
    else X[4] = pow(10.0, -11.195 + (1.5408e-1 * z) - (1.4348e-3 * pow(z, 2)) + (1.0166e-5 * pow(z, 3)));
    X[5] = pow(10.0, -53.746 + (1.5439 * z) - (1.8824e-2 * pow(z, 2)) + (1.1587e-4 * pow(z, 3)) - (3.5399e-7 * pow(z, 2)) + (4.2609e-10 * pow(z, 5)));
    if (z > 30.0) X[6] = pow(10.0, -4.2563 + (7.6245e-2 * z) - (2.1824e-3 * pow(z, 2)) - (2.3010e-6 * pow(z, 3)) + (2.4265e-7 * pow(z, 4)) - (1.2500e-9 * pow(z, 5)));
    else X[6] = pow(10.0, -1.7491 + (4.4986e-2 * z) - (6.8549e-2 * pow(z, 2)) + (5.4639e-3 * pow(z, 3)) - (1.5539e-4 * pow(z, 4)) + (1.5063e-6 * pow(z, 5)));
    X_ON = (X[0] + X[1]) / 0.9903;

    Z_rot[0] = 54.1 * exp(-17.3 * (pow(T_z, -1.0 / 3.0)));
    Z_rot[1] = 63.3 * exp(-16.7 * (pow(T_z, -1.0 / 3.0)));
    Z_rot_ = 1.0 / ((X[1] / Z_rot[1]) + (X[0] / Z_rot[0]));

    sigma = 5.0 / sqrt(21.0);
    nn = (4.0 / 5.0) * sqrt(3.0 / 7.0) * Z_rot_;
    chi = 3.0 * nn * nu / 4.0;
    cchi = 2.36 * chi;

    beta_0 = 2.0 * kPi * freq / c_snd_z;
    beta_1 = sqrt(0.5 * (sqrt(1.0 + pow(nu, 2)) + 1.0) / (1.0 + pow(nu, 2)));
    beta_2 = sqrt((1.0 + pow(cchi, 2)) / (1.0 + pow((sigma * cchi), 2)));
    alpha_1 = beta_0 * sqrt(0.5 * (sqrt(1.0 + pow(nu, 2)) - 1.0) / (1.0 + pow(nu, 2)));
    alpha_2 = beta_0 * (((sigma / 2.0 - 1.0 / (2.0 * sigma)) * chi) / (sqrt((1.0 + pow(cchi, 2)) * (1.0 + pow(sigma * cchi, 2)))));
    a_cl = alpha_1 * beta_2;
    a_rot = alpha_2 * beta_1 * X_ON;

    Tr = pow(T_z / T_o, -1.0 / 3.0) - 1.0;
    A1 = (X[0] + X[1]) * 24.0 * exp(-9.16 * Tr);
    A2 = (X[4] + X[5]) * 2400.0;
    B = 40400.0 * exp(10.0 * Tr);
    C = 0.02 * exp(-11.2 * Tr);
    D = 0.391 * exp(8.41 * Tr);
    E = 9.0 * exp(-19.9 * Tr);
    F = 60000.0;
    G = 28000.0 * exp(-4.17 * Tr);
    H = 22000.0 * exp(-7.68 * Tr);
    I = 15100.0 * exp(-10.4 * Tr);
    J = 11500.0 * exp(-9.17 * Tr);
    K = (8.48e08) * exp(9.17 * Tr);
    L = exp(-7.72 * Tr);
    ZZ = H * X[2] + I * (X[0] + 0.5 * X[4]) + J * (X[1] + 0.5 * X[5]) + K * (X[6] + X[3]);
    hu = 100.0 * (X[3] + X[6]);
    f_vib[0] = (P_z / P_o) * (mu_o / mu) * (A1 + A2 + B * hu * (C + hu) * (D + hu));
    f_vib[1] = (P_z / P_o) * (mu_o / mu) * (E + F * X[3] + G * X[6]);
    f_vib[2] = (P_z / P_o) * (mu_o / mu) * ZZ;
    f_vib[3] = (P_z / P_o) * (mu_o / mu) * 1.2e5 * L;
    double a_vib_ = 0.0;
    for (m = 0; m < 4; m++) {
        C_R = ((pow(theta[m] / T_z, 2)) * exp(-theta[m] / T_z)) / (pow(1.0 - exp(-theta[m] / T_z), 2));
        A_max = (X[m] * (kPi / 2) * C_R) / (Cp_R[m] * (Cv_R[m] + C_R));
        a_vib_ += (A_max / c_snd_z) * ((2.0 * (pow(freq, 2)) / f_vib[m]) / (1.0 + pow(freq / f_vib[m], 2)));
    }
    a_vib = a_vib_;
    return (a_cl * 1.003 + a_rot + a_vib) * tweak_abs * 8.685889e3;
}

static double SB_alpha(Ray& r, double x, double y, double z, double freq) {
#ifdef ORC_REGION_ABSORPTION
    ORC_REGION_ABSORPTION;   // operation-counting build only (oracle/opcount)
#endif
    double c = a_c(r, x, y, z);
    return sb_alpha_cart(c, a_rho(r, x, y, z), z, freq, r.A->tweak_abs);
}

// ---- equation set (geoac.eqset.3d.strat.cpp) ----
static void set_initial(Ray& r, double* sol0, double x0, double y0, double z0) {
    Refs& refs = r.refs;
    refs.src_loc[0] = x0; refs.src_loc[1] = y0; refs.src_loc[2] = z0;
    refs.c0 = a_c(r, x0, y0, z0);
    double mach[3] = {a_u(r, x0, y0, z0) / refs.c0, a_v(r, x0, y0, z0) / refs.c0, a_w(r, x0, y0, z0) / refs.c0};
    const double th = r.theta, ph = r.phi;
    double nu0[3] = {cos(th) * cos(ph), cos(th) * sin(ph), sin(th)};
    double mu0_th[3] = {-sin(th) * cos(ph), -sin(th) * sin(ph), cos(th)};
    double mu0_ph[3] = {-cos(th) * sin(ph), cos(th) * cos(ph), 0.0};
    double ms = 1.0 + (nu0[0] * mach[0] + nu0[1] * mach[1] + nu0[2] * mach[2]);
    refs.nu0 = 1.0 / ms;
    for (int n = 0; n < r.eq_cnt; n++) {
        switch (n) {
            case 0: sol0[n] = x0; break;
            case 1: sol0[n] = y0; break;
            case 2: sol0[n] = z0; break;
            case 3: case 4: case 5: sol0[n] = nu0[n - 3] / ms; break;
            case 6: case 7: case 8: case 12: case 13: case 14: sol0[n] = 0.0; break;
            case 9: case 10: case 11:
                sol0[n] = mu0_th[n - 9] / ms - nu0[n - 9] / pow(ms, 2) * (mu0_th[0] * mach[0] + mu0_th[1] * mach[1] + mu0_th[2] * mach[2]);
                break;
            case 15: case 16: case 17:
                sol0[n] = mu0_ph[n - 15] / ms - nu0[n - 15] / pow(ms, 2) * (mu0_ph[0] * mach[0] + mu0_ph[1] * mach[1] + mu0_ph[2] * mach[2]);
                break;
        }
    }
}

static void approx_intercept(Ray& r, const double* s2, const double* s1, double* prev) {
    double dz_grnd = topo_z(r, s1[0], s1[1]) - s1[2];
    double dz_k = (s1[2] - s2[2]) - (s1[0] - s2[0]) * topo_dz(r, s1[0], s1[1], 0) - (s1[1] - s2[1]) * topo_dz(r, s1[0], s1[1], 1);
    for (int n = 0; n < r.eq_cnt; n++) prev[n] = s1[n] + (s1[n] - s2[n]) / dz_k * dz_grnd;
}

static void set_refl(Ray& r, const double* s2, const double* s1, double* out) {
    double prev[18];
    approx_intercept(r, s2, s1, prev);
    double zg, c_grnd, a, b, norm1, norm2, C1x, C1y, C1z, C2x, C2y;
    double da_dth = 0, db_dth = 0, da_dph = 0, db_dph = 0;
    double dC1x_dth = 0, dC1y_dth = 0, dC1z_dth = 0, dC2x_dth = 0, dC2y_dth = 0, ds0_dth = 0;
    double dC1x_dph = 0, dC1y_dph = 0, dC1z_dph = 0, dC2x_dph = 0, dC2y_dph = 0, ds0_dph = 0;
    double dnux_ds = 0, dnuy_ds = 0, dnuz_ds = 0;
    const double c0 = r.refs.c0;
    zg = topo_z(r, prev[0], prev[1]);
    c_grnd = a_c(r, prev[0], prev[1], zg);
    a = topo_dz(r, prev[0], prev[1], 0);
    b = topo_dz(r, prev[0], prev[1], 1);
    norm1 = 1.0 + pow(a, 2) + pow(b, 2);
    C1x = (1.0 - pow(a, 2) + pow(b, 2)) / norm1; C2x = 2.0 * a / norm1;
    C1y = (1.0 + pow(a, 2) - pow(b, 2)) / norm1; C2y = 2.0 * b / norm1;
    C1z = (1.0 - pow(a, 2) - pow(b, 2)) / norm1;
    if (r.calc_amp) {
        norm2 = prev[5] - a * prev[3] - b * prev[4];
        double z00 = topo_ddz(r, prev[0], prev[1], 0, 0), z01 = topo_ddz(r, prev[0], prev[1], 0, 1);
        double z10 = topo_ddz(r, prev[0], prev[1], 1, 0), z11 = topo_ddz(r, prev[0], prev[1], 1, 1);
        da_dth = (prev[6] * (prev[5] - b * prev[4]) - prev[3] * (prev[8] - b * prev[7])) / norm2 * z00
               + (prev[7] * (prev[5] - a * prev[3]) - prev[4] * (prev[8] - a * prev[6])) / norm2 * z01;
        db_dth = (prev[6] * (prev[5] - b * prev[4]) - prev[3] * (prev[8] - b * prev[7])) / norm2 * z10
               + (prev[7] * (prev[5] - a * prev[3]) - prev[4] * (prev[8] - a * prev[6])) / norm2 * z11;
        da_dph = (prev[12] * (prev[5] - b * prev[4]) - prev[3] * (prev[14] - b * prev[13])) / norm2 * z00
               + (prev[13] * (prev[5] - a * prev[3]) - prev[4] * (prev[14] - a * prev[12])) / norm2 * z01;
        db_dph = (prev[12] * (prev[5] - b * prev[4]) - prev[3] * (prev[14] - b * prev[13])) / norm2 * z10
               + (prev[13] * (prev[5] - a * prev[3]) - prev[4] * (prev[14] - a * prev[12])) / norm2 * z11;
        dC1x_dth = -4.0 * a / pow(norm1, 2) * ((1.0 + pow(b, 2)) * da_dth - a * b * db_dth);
        dC1x_dph = -4.0 * a / pow(norm1, 2) * ((1.0 + pow(b, 2)) * da_dph - a * b * db_dph);
        dC1y_dth = -4.0 * b / pow(norm1, 2) * ((1.0 + pow(a, 2)) * db_dth - a * b * da_dth);
        dC1y_dph = -4.0 * b / pow(norm1, 2) * ((1.0 + pow(a, 2)) * db_dph - a * b * da_dph);
        dC1z_dth = -4.0 / pow(norm1, 2) * (a * da_dth + b * db_dth);
        dC1z_dph = -4.0 / pow(norm1, 2) * (a * da_dph + b * db_dph);
        dC2x_dth = 2.0 / pow(norm1, 2) * ((1.0 - pow(a, 2) + pow(b, 2)) * da_dth - 2.0 * a * b * db_dth);
        dC2x_dph = 2.0 / pow(norm1, 2) * ((1.0 - pow(a, 2) + pow(b, 2)) * da_dph - 2.0 * a * b * db_dph);
        dC2y_dth = 2.0 / pow(norm1, 2) * ((1.0 + pow(a, 2) - pow(b, 2)) * db_dth - 2.0 * a * b * da_dth);
        dC2y_dph = 2.0 / pow(norm1, 2) * ((1.0 + pow(a, 2) - pow(b, 2)) * db_dph - 2.0 * a * b * da_dph);
        ds0_dth = -c0 / c_grnd * (prev[8] - a * prev[6] - b * prev[7]) / norm2;
        ds0_dph = -c0 / c_grnd * (prev[14] - a * prev[12] - b * prev[13]) / norm2;
        double x = prev[0], y = prev[1];
        dnux_ds = -1.0 / c_grnd * (c0 / c_grnd * a_dc(r, x, y, zg, 0) + prev[3] * a_du(r, x, y, zg, 0) + prev[4] * a_dv(r, x, y, zg, 0) + prev[5] * a_dw(r, x, y, zg, 0));
        dnuy_ds = -1.0 / c_grnd * (c0 / c_grnd * a_dc(r, x, y, zg, 1) + prev[3] * a_du(r, x, y, zg, 1) + prev[4] * a_dv(r, x, y, zg, 1) + prev[5] * a_dw(r, x, y, zg, 1));
        dnuz_ds = -1.0 / c_grnd * (c0 / c_grnd * a_dc(r, x, y, zg, 2) + prev[3] * a_du(r, x, y, zg, 2) + prev[4] * a_dv(r, x, y, zg, 2) + prev[5] * a_dw(r, x, y, zg, 2));
    }
    for (int n = 0; n < r.eq_cnt; n++) {
        switch (n) {
            case 0: case 1: out[n] = prev[n]; break;
            case 2: out[n] = zg; break;
            case 3: case 6: case 12: out[n] = C1x * prev[n] + C2x * (prev[n + 2] - prev[n + 1] * b); break;
            case 4: case 7: case 13: out[n] = C1y * prev[n] + C2y * (prev[n + 1] - prev[n - 1] * a); break;
            case 5: case 8: case 14: out[n] = -C1z * prev[n] + prev[n - 2] * C2x + prev[n - 1] * C2y; break;
            case 9: out[n] = C1x * prev[9] + C2x * (prev[11] - b * prev[10] - prev[4] * db_dth) + dC1x_dth * prev[3] + dC2x_dth * (prev[5] - b * prev[4]) + ((C1x - 1.0) * dnux_ds + C2x * (dnuz_ds - b * dnuy_ds)) * ds0_dth; break;
            case 10: out[n] = C1y * prev[10] + C2y * (prev[11] - a * prev[9] - prev[3] * da_dth) + dC1y_dth * prev[4] + dC2y_dth * (prev[5] - a * prev[3]) + ((C1y - 1.0) * dnuy_ds + C2y * (dnuz_ds - a * dnux_ds)) * ds0_dth; break;
            case 11: out[n] = -C1z * prev[11] + C2x * prev[9] + C2y * prev[10] - dC1z_dth * prev[5] + dC2x_dth * prev[3] + dC2y_dth * prev[4] + (-(C1z + 1.0) * dnuz_ds + C2x * dnux_ds + C2y * dnuy_ds) * ds0_dth; break;
            case 15: out[n] = C1x * prev[15] + C2x * (prev[17] - b * prev[16] - prev[4] * db_dph) + dC1x_dph * prev[3] + dC2x_dph * (prev[5] - b * prev[4]) + ((C1x - 1.0) * dnux_ds + C2x * (dnuz_ds - b * dnuy_ds)) * ds0_dph; break;
            case 16: out[n] = C1y * prev[16] + C2y * (prev[17] - a * prev[15] - prev[3] * da_dph) + dC1y_dph * prev[4] + dC2y_dph * (prev[5] - a * prev[3]) + ((C1y - 1.0) * dnuy_ds + C2y * (dnuz_ds - a * dnux_ds)) * ds0_dph; break;
            case 17: out[n] = -C1z * prev[17] + C2x * prev[15] + C2y * prev[16] - dC1z_dph * prev[5] + dC2x_dph * prev[3] + dC2y_dph * prev[4] + (-(C1z + 1.0) * dnuz_ds + C2x * dnux_ds + C2y * dnuy_ds) * ds0_dph; break;
        }
    }
}

static double set_ds(const Ray& r, const double* cv) {
    double result = r.cfg->ds_max;
    if (cv[2] < r.A->z_bndlyr) result -= (r.cfg->ds_max - r.cfg->ds_min) * exp(-(cv[2] - topo_z(r, cv[0], cv[1])) / 0.2);
    return result;
}

static void update_refs(Ray& r, const double* cv) {
    Refs& refs = r.refs;
    const Atmo& A = *r.A;
    double x = cv[0], y = cv[1], z = cv[2];
    double nu[3] = {cv[3], cv[4], cv[5]};
    double dc_temp, ddc_temp;
    double dd_u_temp[6], dd_v_temp[6], dd_w_temp[6];
    double dd_c[3][3], dd_u[3][3], dd_v[3][3], dd_w[3][3];
    double X_th[3], X_ph[3], mu_th[3], mu_ph[3];
    refs.nu_mag = sqrt(pow(nu[0], 2) + pow(nu[1], 2) + pow(nu[2], 2));
    double z_eval = in_interval(z, A.P.c.x[0], A.P.c.x[A.P.c.n - 1]);
    if (!r.calc_amp) {
        eval_all(z_eval, A.P.c, r.acc_c, refs.c, dc_temp);
        for (int n = 0; n < 2; n++) refs.dc[n] = 0.0;
        refs.dc[2] = dc_temp;
        r.acc_u = r.acc_c; r.acc_v = r.acc_c;
        calc_uvw9(r, x, y, z, refs.u, refs.v, refs.w, refs.du, refs.dv, refs.dw);
        refs.cg[0] = refs.c * nu[0] / refs.nu_mag + refs.u;
        refs.cg[1] = refs.c * nu[1] / refs.nu_mag + refs.v;
        refs.cg[2] = refs.c * nu[2] / refs.nu_mag + refs.w;
        refs.cg_mag = sqrt(pow(refs.cg[0], 2) + pow(refs.cg[1], 2) + pow(refs.cg[2], 2));
        return;
    }
    eval_all(z_eval, A.P.c, r.acc_c, refs.c, dc_temp, ddc_temp);
    for (int n = 0; n < 3; n++) { refs.dc[n] = 0.0; for (int m = 0; m < 3; m++) dd_c[n][m] = 0.0; }
    refs.dc[2] = dc_temp;
    dd_c[2][2] = ddc_temp;
    r.acc_u = r.acc_c; r.acc_v = r.acc_c;
    calc_uvw12(r, x, y, z, refs.u, refs.v, refs.w, refs.du, refs.dv, refs.dw, dd_u_temp, dd_v_temp, dd_w_temp);
    refs.cg[0] = refs.c * nu[0] / refs.nu_mag + refs.u;
    refs.cg[1] = refs.c * nu[1] / refs.nu_mag + refs.v;
    refs.cg[2] = refs.c * nu[2] / refs.nu_mag + refs.w;
    refs.cg_mag = sqrt(pow(refs.cg[0], 2) + pow(refs.cg[1], 2) + pow(refs.cg[2], 2));
    for (int n = 0; n < 3; n++) { dd_u[n][n] = dd_u_temp[n]; dd_v[n][n] = dd_v_temp[n]; dd_w[n][n] = dd_w_temp[n]; }
    dd_u[0][1] = dd_u_temp[3]; dd_u[1][0] = dd_u[0][1];
    dd_u[0][2] = dd_u_temp[4]; dd_u[2][0] = dd_u[0][2];
    dd_u[1][2] = dd_u_temp[5]; dd_u[2][1] = dd_u[1][2];
    dd_v[0][1] = dd_v_temp[3]; dd_v[1][0] = dd_v[0][1];
    dd_v[0][2] = dd_v_temp[4]; dd_v[2][0] = dd_v[0][2];
    dd_v[1][2] = dd_v_temp[5]; dd_v[2][1] = dd_v[1][2];
    dd_w[0][1] = dd_w_temp[3]; dd_w[1][0] = dd_w[0][1];
    dd_w[0][2] = dd_w_temp[4]; dd_w[2][0] = dd_w[0][2];
    dd_w[1][2] = dd_w_temp[5]; dd_w[2][1] = dd_w[1][2];
    for (int n = 0; n < 3; n++) { X_th[n] = cv[6 + n]; mu_th[n] = cv[9 + n]; X_ph[n] = cv[12 + n]; mu_ph[n] = cv[15 + n]; }
    refs.dc[3] = 0.0; refs.du[3] = 0.0; refs.dv[3] = 0.0; refs.dw[3] = 0.0;
    refs.dc[4] = 0.0; refs.du[4] = 0.0; refs.dv[4] = 0.0; refs.dw[4] = 0.0;
    for (int n = 0; n < 3; n++) {
        refs.dc[3] += X_th[n] * refs.dc[n]; refs.du[3] += X_th[n] * refs.du[n]; refs.dv[3] += X_th[n] * refs.dv[n]; refs.dw[3] += X_th[n] * refs.dw[n];
        // The reference accumulates the azimuth variation of v into dv[3]
        // (geoac.eqset.3d.strat.cpp:298); reproduced as is.
        refs.dc[4] += X_ph[n] * refs.dc[n]; refs.du[4] += X_ph[n] * refs.du[n]; refs.dv[3] += X_ph[n] * refs.dv[n]; refs.dw[4] += X_ph[n] * refs.dw[n];
        refs.ddc[n][0] = 0.0; refs.ddc[n][1] = 0.0;
        refs.ddu[n][0] = 0.0; refs.ddu[n][1] = 0.0;
        refs.ddv[n][0] = 0.0; refs.ddv[n][1] = 0.0;
        refs.ddw[n][0] = 0.0; refs.ddw[n][1] = 0.0;
        for (int m = n; m < 3; m++) {
            refs.ddc[n][0] += X_th[m] * dd_c[n][m]; refs.ddc[n][1] += X_ph[m] * dd_c[n][m];
            refs.ddu[n][0] += X_th[m] * dd_u[n][m]; refs.ddu[n][1] += X_ph[m] * dd_u[n][m];
            refs.ddv[n][0] += X_th[m] * dd_v[n][m]; refs.ddv[n][1] += X_ph[m] * dd_v[n][m];
            refs.ddw[n][0] += X_th[m] * dd_w[n][m]; refs.ddw[n][1] += X_ph[m] * dd_w[n][m];
        }
    }
    refs.dnu_mag[0] = (nu[0] * mu_th[0] + nu[1] * mu_th[1] + nu[2] * mu_th[2]) / refs.nu_mag;
    refs.dnu_mag[1] = (nu[0] * mu_ph[0] + nu[1] * mu_ph[1] + nu[2] * mu_ph[2]) / refs.nu_mag;
    for (int n = 0; n < 3; n++) {
        refs.dcg[n][0] = nu[n] / refs.nu_mag * refs.dc[3] + refs.c * mu_th[n] / refs.nu_mag - refs.c * nu[n] / pow(refs.nu_mag, 2) * refs.dnu_mag[0];
        refs.dcg[n][1] = nu[n] / refs.nu_mag * refs.dc[4] + refs.c * mu_ph[n] / refs.nu_mag - refs.c * nu[n] / pow(refs.nu_mag, 2) * refs.dnu_mag[1];
    }
    refs.dcg[0][0] += refs.du[3]; refs.dcg[0][1] += refs.du[4];
    refs.dcg[1][0] += refs.dv[3]; refs.dcg[1][1] += refs.dv[4];
    refs.dcg[2][0] += refs.dw[3]; refs.dcg[2][1] += refs.dw[4];
    refs.dcg_mag[0] = (refs.cg[0] * refs.dcg[0][0] + refs.cg[1] * refs.dcg[1][0] + refs.cg[2] * refs.dcg[2][0]) / refs.cg_mag;
    refs.dcg_mag[1] = (refs.cg[0] * refs.dcg[0][1] + refs.cg[1] * refs.dcg[1][1] + refs.cg[2] * refs.dcg[2][1]) / refs.cg_mag;
}

static double eval_src_eq(const Ray& r, const double* cv, int n_eq) {
    const Refs& refs = r.refs;
    const bool is_topo = false;
    double result = 0.0;
    double nu[3] = {cv[3], cv[4], cv[5]}, mu_th[3] = {0, 0, 0}, mu_ph[3] = {0, 0, 0};
    if (r.calc_amp) {
        mu_th[0] = cv[9]; mu_th[1] = cv[10]; mu_th[2] = cv[11];
        mu_ph[0] = cv[15]; mu_ph[1] = cv[16]; mu_ph[2] = cv[17];
    }
    switch (n_eq) {
        case 0: case 1: case 2:
            result = refs.cg[n_eq] / refs.cg_mag; break;
        case 3: case 4: case 5:
            if (is_topo || n_eq == 5) result = -1.0 / refs.cg_mag * (refs.nu_mag * refs.dc[n_eq - 3] + nu[0] * refs.du[n_eq - 3] + nu[1] * refs.dv[n_eq - 3] + nu[2] * refs.dw[n_eq - 3]);
            break;
        case 6: case 7: case 8:
            result = refs.dcg[n_eq - 6][0] / refs.cg_mag - refs.cg[n_eq - 6] / pow(refs.cg_mag, 2) * refs.dcg_mag[0]; break;
        case 9: case 10: case 11:
            if (is_topo || n_eq == 11) {
                int i = n_eq - 9;
                result = refs.dcg_mag[0] / pow(refs.cg_mag, 2) * (refs.nu_mag * refs.dc[i] + nu[0] * refs.du[i] + nu[1] * refs.dv[i] + nu[2] * refs.dw[i])
                       - 1.0 / refs.cg_mag * (refs.dnu_mag[0] * refs.dc[i] + refs.nu_mag * refs.ddc[i][0] + mu_th[0] * refs.du[i] + mu_th[1] * refs.dv[i] + mu_th[2] * refs.dw[i]
                                              + nu[0] * refs.ddu[i][0] + nu[1] * refs.ddv[i][0] + nu[2] * refs.ddw[i][0]);
            }
            break;
        case 12: case 13: case 14:
            result = refs.dcg[n_eq - 12][1] / refs.cg_mag - refs.cg[n_eq - 12] / pow(refs.cg_mag, 2) * refs.dcg_mag[1]; break;
        case 15: case 16: case 17:
            if (is_topo || n_eq == 17) {
                int i = n_eq - 15;
                result = refs.dcg_mag[1] / pow(refs.cg_mag, 2) * (refs.nu_mag * refs.dc[i] + nu[0] * refs.du[i] + nu[1] * refs.dv[i] + nu[2] * refs.dw[i])
                       - 1.0 / refs.cg_mag * (refs.dnu_mag[1] * refs.dc[i] + refs.nu_mag * refs.ddc[i][1] + mu_ph[0] * refs.du[i] + mu_ph[1] * refs.dv[i] + mu_ph[2] * refs.dw[i]
                                              + nu[0] * refs.ddu[i][1] + nu[1] * refs.ddv[i][1] + nu[2] * refs.ddw[i][1]);
            }
            break;
    }
    return result;
}

static bool break_check(const Ray& r, const double* s) {
    const orc_fan_cfg& P = *r.cfg;
    if (sqrt(pow(s[0] - r.refs.src_loc[0], 2) + pow(s[1] - r.refs.src_loc[1], 2)) > P.rng_max) return true;
    if (s[0] > P.x_max || s[0] < P.x_min) return true;
    if (s[1] > P.y_max || s[1] < P.y_min) return true;
    if (s[2] > P.alt_max) return true;
    return false;
}
static bool ground_check(const Ray& r, const double* s) {
    if (s[2] <= r.A->z_max) {
        if (s[2] < topo_z(r, s[0], s[1])) return true;
    }
    return false;
}

// Midpoint travel-time increment of one segment (geoac.eqset.3d.strat.cpp:486-511).
static double seg_time(Ray& r, const double* a, const double* b) {
    double dx, dy, dz, ds, x, y, z, nu[3], nu_mag, cg[3], cg_mag, c;
    dx = b[0] - a[0]; x = a[0] + dx / 2.0;
    dy = b[1] - a[1]; y = a[1] + dy / 2.0;
    dz = b[2] - a[2]; z = a[2] + dz / 2.0;
    ds = sqrt(dx * dx + dy * dy + dz * dz);
    nu[0] = a[3] + (b[3] - a[3]) / 2.0;
    nu[1] = a[4] + (b[4] - a[4]) / 2.0;
    nu[2] = a[5] + (b[5] - a[5]) / 2.0;
    nu_mag = sqrt(nu[0] * nu[0] + nu[1] * nu[1] + nu[2] * nu[2]);
    c = a_c(r, x, y, z);
    cg[0] = c * nu[0] / nu_mag + a_u(r, x, y, z);
    cg[1] = c * nu[1] / nu_mag + a_v(r, x, y, z);
    cg[2] = c * nu[2] / nu_mag + a_w(r, x, y, z);
    cg_mag = sqrt(pow(cg[0], 2) + pow(cg[1], 2) + pow(cg[2], 2));
    return ds / cg_mag;
}
// Midpoint absorption increment of one segment (geoac.eqset.3d.strat.cpp:688-699).
static double seg_atten(Ray& r, const double* a, const double* b, double freq) {
    double dx, dy, dz, ds, x, y, z;
    dx = b[0] - a[0]; x = a[0] + dx / 2.0;
    dy = b[1] - a[1]; y = a[1] + dy / 2.0;
    dz = b[2] - a[2]; z = a[2] + dz / 2.0;
    ds = sqrt(pow(dx, 2) + pow(dy, 2) + pow(dz, 2));
    return SB_alpha(r, x, y, z, freq) * ds;
}

static double jacobian(Ray& r, const double* s) {
    double c = a_c(r, s[0], s[1], s[2]);
    double nu_mag = sqrt(pow(s[3], 2) + pow(s[4], 2) + pow(s[5], 2));
    double cg[3], cg_mag;
    cg[0] = c * s[3] / nu_mag + a_u(r, s[0], s[1], s[2]);
    cg[1] = c * s[4] / nu_mag + a_v(r, s[0], s[1], s[2]);
    cg[2] = c * s[5] / nu_mag + a_w(r, s[0], s[1], s[2]);
    cg_mag = sqrt(pow(cg[0], 2) + pow(cg[1], 2) + pow(cg[2], 2));
    double dxds = cg[0] / cg_mag, dyds = cg[1] / cg_mag, dzds = cg[2] / cg_mag;
    double dxdth = s[6], dydth = s[7], dzdth = s[8], dxdph = s[12], dydph = s[13], dzdph = s[14];
    return dxds * (dydth * dzdph - dydph * dzdth) - dxdth * (dyds * dzdph - dzds * dydph) + dxdph * (dyds * dzdth - dzds * dydth);
}

static double amp(Ray& r, const double* s) {
    const Refs& refs = r.refs;
    const double* sl = refs.src_loc;
    double c = a_c(r, s[0], s[1], s[2]);
    double winds[3], winds0[3], cg[3], cg0[3];
    winds[0] = a_u(r, s[0], s[1], s[2]); winds0[0] = a_u(r, sl[0], sl[1], sl[2]);
    winds[1] = a_v(r, s[0], s[1], s[2]); winds0[1] = a_v(r, sl[0], sl[1], sl[2]);
    winds[2] = a_w(r, s[0], s[1], s[2]); winds0[2] = a_w(r, sl[0], sl[1], sl[2]);
    double nu_mag = sqrt(pow(s[3], 2) + pow(s[4], 2) + pow(s[5], 2));
    double nu_mag0 = 1.0 - (s[3] * winds0[0] + s[4] * winds0[1] + s[5] * winds0[2]) / refs.c0;
    for (int n = 0; n < 3; n++) cg[n] = c * s[3 + n] / nu_mag + winds[n];
    cg0[0] = refs.c0 * cos(r.theta) * cos(r.phi) + winds0[0];
    cg0[1] = refs.c0 * cos(r.theta) * sin(r.phi) + winds0[1];
    cg0[2] = refs.c0 * sin(r.theta) + winds0[2];
    double cg_mag = sqrt(pow(cg[0], 2) + pow(cg[1], 2) + pow(cg[2], 2));
    double cg_mag0 = sqrt(pow(cg0[0], 2) + pow(cg0[1], 2) + pow(cg0[2], 2));
    double num = a_rho(r, s[0], s[1], s[2]) * nu_mag * pow(c, 3) * cg_mag0 * cos(r.theta);
    double den = a_rho(r, sl[0], sl[1], sl[2]) * nu_mag0 * pow(refs.c0, 3) * cg_mag * jacobian(r, s);
    return sqrt(fabs(num / den));
}

// One prop_rk4 call (rk4solver.cpp:14-85) on a three-row window.
// On entry rows[1] is the starting row; on return rows[0..2] hold rows
// k-2, k-1 and k (k = returned step count), which is all that set_refl and
// the arrival record read.  tt/att are the ray's running sums: in per-step
// mode (write_rays, main.infraga.3d.cpp:451-453) each segment but the last is
// added to them directly; otherwise the bounce's sum is formed first and
// then added (main.infraga.3d.cpp:486-487), as the reference does.
struct SegOut { int k; bool check; double zmax; };

static SegOut prop_rk4(Ray& r, double rows[3][18], double zmax_in, double freq, bool per_step,
                       double& tt, double& att, int* caustics) {
    const int eq = r.eq_cnt;
    const int length = int(r.cfg->s_max / r.cfg->ds_min);
    double s = 0.0, ds;
    double t0[18], t1[18], t2[18], t3[18], t4[18], p1[18], p2[18], p3[18];
    double buf[3][18];
    double* pm1 = buf[0];   // row k-1
    double* cur = buf[1];   // row k (step base)
    double* nxt = buf[2];   // row k+1
    memcpy(cur, rows[1], sizeof(double) * 18);
    memset(pm1, 0, sizeof(double) * 18);
    SegOut o{0, false, zmax_in};
    double seg_tt = 0.0, seg_att = 0.0;
    double pend_t = 0.0, pend_a = 0.0;
    bool have_pend = false;
    int k;
    for (k = 0; k < length - 1; k++) {
        o.zmax = std::max(o.zmax, cur[2]);
        // Caustics as the write_caustics path counts them: sign changes of
        // the Jacobian between consecutive rows 1..k-1 of a bounce
        // (main.infraga.3d.cpp:448-480).
        if (caustics && r.calc_amp && k >= 1) {
            const double D = jacobian(r, cur);
            if (k >= 2 && D * r.D_prev < 0.0) (*caustics)++;
            r.D_prev = D;
        }
        for (int i = 0; i < eq; i++) t0[i] = cur[i];
        update_refs(r, t0);
        ds = set_ds(r, t0);
        s += ds;
        for (int i = 0; i < eq; i++) { t1[i] = ds * eval_src_eq(r, t0, i); p1[i] = cur[i] + t1[i] / 2.0; }
        update_refs(r, p1);
        for (int i = 0; i < eq; i++) { t2[i] = ds * eval_src_eq(r, p1, i); p2[i] = cur[i] + t2[i] / 2.0; }
        update_refs(r, p2);
        for (int i = 0; i < eq; i++) { t3[i] = ds * eval_src_eq(r, p2, i); p3[i] = cur[i] + t3[i]; }
        update_refs(r, p3);
        for (int i = 0; i < eq; i++) {
            t4[i] = ds * eval_src_eq(r, p3, i);
            nxt[i] = cur[i] + t1[i] / 6.0 + t2[i] / 3.0 + t3[i] / 3.0 + t4[i] / 6.0;
        }
        double dt = seg_time(r, cur, nxt);
        double da = seg_atten(r, cur, nxt, freq);
        if (per_step) {
            if (have_pend) { tt += pend_t; att += pend_a; }
            pend_t = dt; pend_a = da; have_pend = true;
        } else {
            seg_tt += dt; seg_att += da;
        }
        bool stop = false;
        if (s > r.cfg->s_max) { o.check = true; stop = true; }
        else if (break_check(r, nxt)) { o.check = true; stop = true; }
        else if (ground_check(r, nxt)) { o.check = false; stop = true; }
        if (stop) break;
        double* t = pm1; pm1 = cur; cur = nxt; nxt = t;
    }
    if (k == length - 1) o.check = true;   // step budget exhausted: treated as leaving the region
    if (!per_step) { tt += seg_tt; att += seg_att; }
    o.k = k + 1;
    memcpy(rows[0], pm1, sizeof(double) * 18);
    memcpy(rows[1], cur, sizeof(double) * 18);
    memcpy(rows[2], nxt, sizeof(double) * 18);
    return o;
}

}  // namespace d3
}  // namespace orc

using namespace orc;
using namespace orc::d3;

extern "C" int orc_fan_3d(const char* met_path, const char* fmt, const orc_fan_cfg* cfg,
                          const double* theta_deg, const double* phi_deg, int n_rays,
                          double* arrivals, int* n_arr, long long* steps, double* aux) {
    static_assert(sizeof(orc_fan_cfg) > 0, "");
    Atmo A;
    if (!load_profile(met_path, fmt, cfg->reverse_winds != 0, A.P)) return -1;
    A.z0 = cfg->z_grnd;
    A.z_max = A.z0;
    A.z_bndlyr = A.z0 + 2.0;
    A.tweak_abs = cfg->tweak_abs;
    const int nb = cfg->bounces + 1;
    const int eq_cnt = cfg->calc_amp ? 18 : 6;

    std::atomic<int> next_ray{0};
    auto worker = [&]() {
    for (int ir = next_ray++; ir < n_rays; ir = next_ray++) {
        Ray r;
        r.A = &A; r.cfg = cfg; r.calc_amp = cfg->calc_amp != 0; r.eq_cnt = eq_cnt;
        r.theta = theta_deg[ir] * kPi / 180.0;
        r.phi = kPi / 2.0 - phi_deg[ir] * kPi / 180.0;
        double rows[3][18];
        memset(rows, 0, sizeof(rows));
        double z_src = std::max(cfg->src[2], topo_z(r, cfg->src[0], cfg->src[1]));
        set_initial(r, rows[1], cfg->src[0], cfg->src[1], z_src);
        double tt = 0.0, att = 0.0, zmax = A.z0;
        int caustics = 0;
        long long st = 0;
        int na = 0;
        for (int bnc = 0; bnc <= cfg->bounces; bnc++) {
            SegOut o = prop_rk4(r, rows, zmax, cfg->freq, cfg->write_rays != 0, tt, att, &caustics);
            st += o.k;
            zmax = o.zmax;
            if (zmax < (A.z0 + cfg->turn_ht_min)) break;
            if (o.check || o.k < 2) break;
            const double* sk = rows[2];
            double incl = -asin(a_c(r, sk[0], sk[1], topo_z(r, sk[0], sk[1])) / a_c(r, cfg->src[0], cfg->src[1], z_src) * sk[5]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-sk[4], -sk[3]) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            double* out = arrivals + ((size_t)ir * nb + na) * ORC_ARR_COLS;
            out[0] = theta_deg[ir]; out[1] = phi_deg[ir]; out[2] = bnc;
            out[3] = sk[0]; out[4] = sk[1]; out[5] = tt;
            out[6] = sqrt(pow(sk[0] - cfg->src[0], 2) + pow(sk[1] - cfg->src[1], 2)) / tt;
            out[7] = zmax; out[8] = incl; out[9] = baz;
            out[10] = r.calc_amp ? 20.0 * log10(amp(r, sk)) : 0.0;
            out[11] = -2.0 * att;
            if (aux) {
                // Launch-angle sensitivity of the ground intercept, the
                // expressions find_eigenray uses for its Newton step
                // (geoac.eigenray.3d.cpp:334-348, flat ground).
                double* ax = aux + ((size_t)ir * nb + na) * ORC_AUX_COLS;
                double c_src = a_c(r, cfg->src[0], cfg->src[1], z_src);
                double c_grnd = a_c(r, sk[0], sk[1], topo_z(r, sk[0], sk[1]));
                double ds_dth = -c_src / c_grnd * sk[8] / sk[5];
                double ds_dph = -c_src / c_grnd * sk[14] / sk[5];
                double dx_dth = sk[6] + sk[3] * ds_dth, dy_dth = sk[7] + sk[4] * ds_dth;
                double dx_dph = sk[12] + sk[3] * ds_dph, dy_dph = sk[13] + sk[4] * ds_dph;
                ax[0] = r.calc_amp ? sqrt(dx_dth * dx_dth + dy_dth * dy_dth) : 0.0;
                ax[1] = r.calc_amp ? sqrt(dx_dph * dx_dph + dy_dph * dy_dph) : 0.0;
                ax[2] = r.calc_amp ? jacobian(r, sk) : 0.0;
                ax[3] = caustics;
            }
            na++;
            double nxt[18];
            set_refl(r, rows[0], rows[1], nxt);
            memcpy(rows[1], nxt, sizeof(nxt));
        }
        n_arr[ir] = na;
        steps[ir] = st;
    }
    };
    const int nt = std::max(1, cfg->n_threads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    return 0;
}
