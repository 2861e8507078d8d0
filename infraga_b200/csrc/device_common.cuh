// Shared device helpers: knot-table spline evaluation and the
// Sutherland-Bass absorption model.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace iga {

constexpr double kPi = 3.141592653589793238462643;   // value of Pi in geoac.params.3d.cpp:10
constexpr double kGamma = 1.4;                       // atmo::gam
constexpr double kRgas = 287.058;                    // atmo::R
constexpr int kStride = 10;                          // doubles per knot row (atmo_host.h)

// Altitude segment search on the interleaved knot table: walk from the
// cached segment `k` until tab[k].z <= z <= tab[k+1].z (z already clamped to
// the table range).  The walk keeps the cached segment when z sits on a
// knot, like interp::find_segment's cached index (interpolation.cpp:23-25).
__device__ __forceinline__ int seg_walk(const double* __restrict__ tab, int n, double z, int k) {
    while (k > 0 && z < tab[k * kStride]) --k;
    while (k < n - 2 && z > tab[(k + 1) * kStride]) ++k;
    return k;
}

// First guess of the segment for a fresh ray (uniform grids are exact up to
// rounding, non-uniform ones are corrected by seg_walk).
__device__ __forceinline__ int seg_guess(double z, double z_lo, double inv_dz, int n) {
    int k = (int)((z - z_lo) * inv_dz);
    return k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
}

// Hermite-form cubic on one segment, the form of interp::eval_all
// (interpolation.cpp:213-260): A = s0 dx - df, B = -s1 dx + df.
struct Cubic {
    double X, om, idx;   // local coordinate, 1-X, 1/dx
};

__device__ __forceinline__ Cubic cubic_at(const double* __restrict__ r0, double z) {
    Cubic q;
    q.idx = r0[1];
    q.X = (z - r0[0]) * q.idx;
    q.om = 1.0 - q.X;
    return q;
}

// value only
__device__ __forceinline__ double cubic_f(const double* __restrict__ r0, const Cubic& q, int col) {
    const double* r1 = r0 + kStride;
    const double dx = r1[0] - r0[0];
    const double f0 = r0[col], df = r1[col] - f0;
    const double A = r0[col + 1] * dx - df;
    const double B = -r1[col + 1] * dx + df;
    return f0 + q.X * (df + q.om * (A * q.om + B * q.X));
}

// value and first derivative
__device__ __forceinline__ void cubic_f1(const double* __restrict__ r0, const Cubic& q, int col, double& f, double& d1) {
    const double* r1 = r0 + kStride;
    const double dx = r1[0] - r0[0];
    const double f0 = r0[col], df = r1[col] - f0;
    const double A = r0[col + 1] * dx - df;
    const double B = -r1[col + 1] * dx + df;
    const double t = A * q.om + B * q.X;
    f = f0 + q.X * (df + q.om * t);
    d1 = (df + (1.0 - 2.0 * q.X) * t + q.X * q.om * (B - A)) * q.idx;
}

// value, first and second derivative
__device__ __forceinline__ void cubic_f2(const double* __restrict__ r0, const Cubic& q, int col, double& f, double& d1, double& d2) {
    const double* r1 = r0 + kStride;
    const double dx = r1[0] - r0[0];
    const double f0 = r0[col], df = r1[col] - f0;
    const double A = r0[col + 1] * dx - df;
    const double B = -r1[col + 1] * dx + df;
    const double t = A * q.om + B * q.X;
    f = f0 + q.X * (df + q.om * t);
    d1 = (df + (1.0 - 2.0 * q.X) * t + q.X * q.om * (B - A)) * q.idx;
    d2 = 2.0 * (B - 2.0 * A + (A - B) * 3.0 * q.X) * (q.idx * q.idx);
}

// Constants of the absorption model that do not depend on position
// (pow(10, const) gas fractions), computed once on the host.
struct SBConst {
    double x0_low;   // O2 fraction below 90 km
    double x1_low;   // N2 fraction below 76 km
    double x2;       // CO2 fraction
};

// exp10 and reciprocal cube root on either side of the compiler.
__host__ __device__ __forceinline__ double iga_exp10(double x) {
#ifdef __CUDA_ARCH__
    return exp10(x);
#else
    return pow(10.0, x);
#endif
}
__host__ __device__ __forceinline__ double iga_rcbrt(double x) {
#ifdef __CUDA_ARCH__
    return rcbrt(x);
#else
    return 1.0 / cbrt(x);
#endif
}

// Sutherland & Bass (2004) absorption in dB/km times tweak_abs.  Inputs are
// the sound speed [km/s] and density [g/cm^3] at the evaluation point and its
// altitude z [km].  SPH selects the spherical variant of the reference
// (atmo_state.abs.sph.cpp:11-147) over the Cartesian one
// (atmo_state.abs.cart.cpp:12-142); they differ in two places:
//  - the Cartesian N-profile polynomial uses z^2 where z^4 is meant (cart
//    line 78); the spherical one has z^4.  Both are reproduced.
//  - the rotational loss: Cartesian a_rot = alpha_2 beta_1 X_ON with
//    alpha_2 carrying 1/sqrt((1+cchi^2)(1+(sigma cchi)^2)); the spherical
//    a_rot has only 1/sqrt(1+cchi^2) under its root.
// The classical term a_cl (x 1.003 with the diffusion term) is the same
// expression in both, written in each file's own grouping.  The H2O branch
// for z > 100 km is unreachable in the reference (nested under z <= 30) and
// so absent.
template <bool SPH>
__host__ __device__ __forceinline__ double sb_alpha(double c_kms, double rho_gcc, double z, double freq,
                                                    double tweak_abs, const SBConst& k) {
    const double mu_o = 18.192e-6, T_o = 293.15, P_o = 101325.0, S = 117.0;
    const double cs = c_kms * 1.0e3;
    const double T_z = cs * cs / (kRgas * kGamma);
    const double P_z = rho_gcc * 1.0e3 * (cs * cs) / kGamma;
    const double mu = mu_o * sqrt(T_z / T_o) * ((1.0 + S / T_o) / (1.0 + S / T_z));
    const double nu = (8.0 * kPi * freq * mu) / (3.0 * P_z);

    const double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    double X0 = k.x0_low, X1 = k.x1_low;
    if (z > 90.0) X0 = iga_exp10(49.296 - (1.5524 * z) + (1.8714e-2 * z2) - (1.1069e-4 * z3) + (3.199e-7 * z4) - (3.6211e-10 * z5));
    if (z > 76.0) X1 = iga_exp10((1.3972e-1) - (5.6269e-3 * z) + (3.9407e-5 * z2) - (1.0737e-7 * z3));
    const double X2 = k.x2;
    const double X3 = iga_exp10(z > 80.0 ? (-4.234 - (3.0975e-2 * z))
                                     : (-19.027 + (1.3093 * z) - (4.6496e-2 * z2) + (7.8543e-4 * z3) - (6.5169e-6 * z4) + (2.1343e-8 * z5)));
    const double X4 = iga_exp10(z > 95.0 ? (-3.2456 + (4.6642e-2 * z) - (2.6894e-4 * z2) + (5.264e-7 * z3))
                                     : (-11.195 + (1.5408e-1 * z) - (1.4348e-3 * z2) + (1.0166e-5 * z3)));
    const double X5 = iga_exp10(-53.746 + (1.5439 * z) - (1.8824e-2 * z2) + (1.1587e-4 * z3) - (3.5399e-7 * (SPH ? z4 : z2)) + (4.2609e-10 * z5));
    const double X6 = iga_exp10(z > 30.0 ? (-4.2563 + (7.6245e-2 * z) - (2.1824e-3 * z2) - (2.3010e-6 * z3) + (2.4265e-7 * z4) - (1.2500e-9 * z5))
                                     : (-1.7491 + (4.4986e-2 * z) - (6.8549e-2 * z2) + (5.4639e-3 * z3) - (1.5539e-4 * z4) + (1.5063e-6 * z5)));
    const double X_ON = (X0 + X1) / 0.9903;

    const double Tm13 = iga_rcbrt(T_z);
    const double Z_rot0 = 54.1 * exp(-17.3 * Tm13);
    const double Z_rot1 = 63.3 * exp(-16.7 * Tm13);
    const double Z_rot_ = 1.0 / ((X1 / Z_rot1) + (X0 / Z_rot0));

    const double sigma = 5.0 / sqrt(21.0);
    const double nn = (4.0 / 5.0) * sqrt(3.0 / 7.0) * Z_rot_;
    const double chi = 3.0 * nn * nu / 4.0;
    const double cchi = 2.36 * chi;

    const double beta_0 = 2.0 * kPi * freq / cs;
    const double nu2 = nu * nu, sq = sqrt(1.0 + nu2);
    const double cc2 = cchi * cchi, sc2 = (sigma * cchi) * (sigma * cchi);
    double a_cl, a_rot;
    if (SPH) {
        a_cl = beta_0 * sqrt(0.5 * (sq - 1.0) * (1.0 + cc2) / ((1.0 + nu2) * (1.0 + sc2)));
        a_rot = beta_0 * X_ON * ((sigma * sigma - 1.0) * chi / (2.0 * sigma)) *
                sqrt(0.5 * (sq + 1.0) / ((1.0 + nu2) * (1.0 + cc2)));
    } else {
        const double beta_1 = sqrt(0.5 * (sq + 1.0) / (1.0 + nu2));
        const double beta_2 = sqrt((1.0 + cc2) / (1.0 + sc2));
        const double alpha_1 = beta_0 * sqrt(0.5 * (sq - 1.0) / (1.0 + nu2));
        const double alpha_2 = beta_0 * (((sigma / 2.0 - 1.0 / (2.0 * sigma)) * chi) / (sqrt((1.0 + cc2) * (1.0 + sc2))));
        a_cl = alpha_1 * beta_2;
        a_rot = alpha_2 * beta_1 * X_ON;
    }

    const double Tr = iga_rcbrt(T_z / T_o) - 1.0;
    const double A1 = (X0 + X1) * 24.0 * exp(-9.16 * Tr);
    const double A2 = (X4 + X5) * 2400.0;
    const double B = 40400.0 * exp(10.0 * Tr);
    const double C = 0.02 * exp(-11.2 * Tr);
    const double D = 0.391 * exp(8.41 * Tr);
    const double E = 9.0 * exp(-19.9 * Tr);
    const double F = 60000.0;
    const double G = 28000.0 * exp(-4.17 * Tr);
    const double H = 22000.0 * exp(-7.68 * Tr);
    const double I = 15100.0 * exp(-10.4 * Tr);
    const double J = 11500.0 * exp(-9.17 * Tr);
    const double K = (8.48e08) * exp(9.17 * Tr);
    const double L = exp(-7.72 * Tr);
    const double ZZ = H * X2 + I * (X0 + 0.5 * X4) + J * (X1 + 0.5 * X5) + K * (X6 + X3);
    const double hu = 100.0 * (X3 + X6);
    const double pre = (P_z / P_o) * (mu_o / mu);
    const double fv[4] = {pre * (A1 + A2 + B * hu * (C + hu) * (D + hu)), pre * (E + F * X3 + G * X6), pre * ZZ, pre * 1.2e5 * L};
    const double th[4] = {2239.1, 3352.0, 915.0, 1037.0};
    const double Cp[4] = {7.0 / 2.0, 7.0 / 2.0, 4.0, 4.0};
    const double Cv[4] = {5.0 / 2.0, 5.0 / 2.0, 3.0, 3.0};
    const double Xm[4] = {X0, X1, X2, X3};
    const double f2 = freq * freq;
    double a_vib = 0.0;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const double r = th[m] / T_z;
        const double e = exp(-r);
        const double C_R = (r * r * e) / ((1.0 - e) * (1.0 - e));
        const double A_max = (Xm[m] * (kPi / 2) * C_R) / (Cp[m] * (Cv[m] + C_R));
        const double q = freq / fv[m];
        a_vib += (A_max / cs) * ((2.0 * f2 / fv[m]) / (1.0 + q * q));
    }
    if (SPH) return (a_cl + a_rot + 0.003 * a_cl + a_vib) * tweak_abs * 8.685889e3;
    return (a_cl * 1.003 + a_rot + a_vib) * tweak_abs * 8.685889e3;
}

__host__ __device__ __forceinline__ double sb_alpha_cart(double c_kms, double rho_gcc, double z, double freq,
                                                         double tweak_abs, const SBConst& k) {
    return sb_alpha<false>(c_kms, rho_gcc, z, freq, tweak_abs, k);
}

}  // namespace iga
