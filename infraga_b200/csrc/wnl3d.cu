// Weakly non-linear waveform along 3D stratified rays (infraga-3d
// -wnl_wvfrm): geoac::wnl_wvfrm (geoac.eqset.3d.strat.cpp:753-1045) with the
// per-bounce driver of run_wnl_wvfrm (main.infraga.3d.cpp:1087-1420).
//
// The ray is traced by the FP64 fan kernel in its kPathWnl row mode (every
// RK4 row of every bounce with the Jacobian and the bounce's travel time).
// Then one CTA per ray runs the whole waveform evolution without returning
// to the host: the waveform u(t) (N samples), its spectrum U(f) and one
// complex work array live in shared memory, and each Heun step is
//   one thread: the linear splines along the ray (interp::linear_spline_1D;
//               the six share their knots, so one segment walk serves all),
//               beta, the step size,
//               the caustic test and the frequency-independent part of the
//               Sutherland-Bass absorption at the step's point;
//   all threads: the non-linear source term, one real FFT of it, the spectral
//               Heun update with absorption and filters, the max of f|U|,
//               and one inverse real FFT back to u(t).
// The reference forms A = FFT{u^2}, B = FFT{u d(u^2)/dt}, C = FFT{(d(u^2)/dt)^2}
// and adds their weighted sum; the FFT is linear, so the weighted sum of the
// three time series is transformed once instead (same result up to rounding).
// Real transforms of length N are complex transforms of length N/2 (radix-2,
// decimation in frequency forward, in time inverse, twiddles from a table)
// with the usual even/odd split, FFTW's r2c / c2r conventions (unnormalised;
// the c2r ignores the imaginary parts of the DC and Nyquist bins).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "fan3d_common.cuh"
#include "fansph_common.cuh"
#include "handle.h"
#include "nvtx.h"

using namespace iga_internal;

namespace iga {

constexpr int kWnlThreads = 512;
constexpr int kWnlMaxLen = 8192;
constexpr int kWnlInfo = 17;      // doubles of per-ray summary (IGA_WNL_INFO order)
constexpr int kWnlEventCols = 4;  // type, value, altitude, beta

// The frequency-independent part of sb_alpha<SPH> at one point
// (atmo_state.abs.cart.cpp:12-142, atmo_state.abs.sph.cpp:11-147): what the
// per-bin part below needs.
struct SBPoint {
    double cs, mu, P_z3;   // sound speed [m/s], viscosity, 3 P_z
    double nn;             // (4/5) sqrt(3/7) Z_rot
    double X_ON;
    double Acs[4];         // A_max / cs of the four vibrational modes
    double fv[4];          // relaxation frequencies
    double tweak;
};

template <bool SPH>
__device__ __forceinline__ SBPoint sb_point(double c_kms, double rho_gcc, double z, double tweak_abs, const SBConst& k) {
    SBPoint P;
    const double mu_o = 18.192e-6, T_o = 293.15, P_o = 101325.0, S = 117.0;
    const double cs = c_kms * 1.0e3;
    const double T_z = cs * cs / (kRgas * kGamma);
    const double P_z = rho_gcc * 1.0e3 * (cs * cs) / kGamma;
    const double mu = mu_o * sqrt(T_z / T_o) * ((1.0 + S / T_o) / (1.0 + S / T_z));
    const double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    double X0 = k.x0_low, X1 = k.x1_low;
    if (z > 90.0) X0 = iga_exp10(49.296 - (1.5524 * z) + (1.8714e-2 * z2) - (1.1069e-4 * z3) + (3.199e-7 * z4) - (3.6211e-10 * z5));
    if (z > 76.0) X1 = iga_exp10((1.3972e-1) - (5.6269e-3 * z) + (3.9407e-5 * z2) - (1.0737e-7 * z3));
    const double X2 = k.x2;
    const double X3 = iga_exp10(z > 80.0 ? (-4.234 - (3.0975e-2 * z))
                                     : (-19.027 + (1.3093 * z) - (4.6496e-2 * z2) + (7.8543e-4 * z3) - (6.5169e-6 * z4) + (2.1343e-8 * z5)));
    const double X4 = iga_exp10(z > 95.0 ? (-3.2456 + (4.6642e-2 * z) - (2.6894e-4 * z2) + (5.264e-7 * z3))
                                     : (-11.195 + (1.5408e-1 * z) - (1.4348e-3 * z2) + (1.0166e-5 * z3)));
    // the Cartesian N-profile polynomial's z^2 where z^4 is meant (cart line 78)
    const double X5 = iga_exp10(-53.746 + (1.5439 * z) - (1.8824e-2 * z2) + (1.1587e-4 * z3) - (3.5399e-7 * (SPH ? z4 : z2)) + (4.2609e-10 * z5));
    const double X6 = iga_exp10(z > 30.0 ? (-4.2563 + (7.6245e-2 * z) - (2.1824e-3 * z2) - (2.3010e-6 * z3) + (2.4265e-7 * z4) - (1.2500e-9 * z5))
                                     : (-1.7491 + (4.4986e-2 * z) - (6.8549e-2 * z2) + (5.4639e-3 * z3) - (1.5539e-4 * z4) + (1.5063e-6 * z5)));
    const double Tm13 = iga_rcbrt(T_z);
    const double Z_rot0 = 54.1 * exp(-17.3 * Tm13);
    const double Z_rot1 = 63.3 * exp(-16.7 * Tm13);
    const double Z_rot_ = 1.0 / ((X1 / Z_rot1) + (X0 / Z_rot0));
    P.cs = cs; P.mu = mu; P.P_z3 = 3.0 * P_z;
    P.nn = (4.0 / 5.0) * sqrt(3.0 / 7.0) * Z_rot_;
    P.X_ON = (X0 + X1) / 0.9903;
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
    P.fv[0] = pre * (A1 + A2 + B * hu * (C + hu) * (D + hu));
    P.fv[1] = pre * (E + F * X3 + G * X6);
    P.fv[2] = pre * ZZ;
    P.fv[3] = pre * 1.2e5 * L;
    const double th[4] = {2239.1, 3352.0, 915.0, 1037.0};
    const double Cp[4] = {7.0 / 2.0, 7.0 / 2.0, 4.0, 4.0};
    const double Cv[4] = {5.0 / 2.0, 5.0 / 2.0, 3.0, 3.0};
    const double Xm[4] = {X0, X1, X2, X3};
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const double r = th[m] / T_z;
        const double e = exp(-r);
        const double C_R = (r * r * e) / ((1.0 - e) * (1.0 - e));
        const double A_max = (Xm[m] * (kPi / 2) * C_R) / (Cp[m] * (Cv[m] + C_R));
        P.Acs[m] = A_max / cs;
    }
    P.tweak = tweak_abs;
    return P;
}

// sb_alpha<SPH>(c, rho, z, freq) given sb_point<SPH>(c, rho, z): the same
// operations in the same order.
template <bool SPH>
__device__ __forceinline__ double sb_bin(const SBPoint& P, double freq) {
    const double sigma = 5.0 / sqrt(21.0);
    const double nu = (8.0 * kPi * freq * P.mu) / P.P_z3;
    const double chi = 3.0 * P.nn * nu / 4.0;
    const double cchi = 2.36 * chi;
    const double beta_0 = 2.0 * kPi * freq / P.cs;
    const double nu2 = nu * nu, sq = sqrt(1.0 + nu2);
    const double cc2 = cchi * cchi, sc2 = (sigma * cchi) * (sigma * cchi);
    double a_cl, a_rot;
    if (SPH) {
        a_cl = beta_0 * sqrt(0.5 * (sq - 1.0) * (1.0 + cc2) / ((1.0 + nu2) * (1.0 + sc2)));
        a_rot = beta_0 * P.X_ON * ((sigma * sigma - 1.0) * chi / (2.0 * sigma)) *
                sqrt(0.5 * (sq + 1.0) / ((1.0 + nu2) * (1.0 + cc2)));
    } else {
        const double beta_1 = sqrt(0.5 * (sq + 1.0) / (1.0 + nu2));
        const double beta_2 = sqrt((1.0 + cc2) / (1.0 + sc2));
        const double alpha_1 = beta_0 * sqrt(0.5 * (sq - 1.0) / (1.0 + nu2));
        const double alpha_2 = beta_0 * (((sigma / 2.0 - 1.0 / (2.0 * sigma)) * chi) / (sqrt((1.0 + cc2) * (1.0 + sc2))));
        a_cl = alpha_1 * beta_2;
        a_rot = alpha_2 * beta_1 * P.X_ON;
    }
    const double f2 = freq * freq;
    double a_vib = 0.0;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const double q = freq / P.fv[m];
        a_vib += P.Acs[m] * ((2.0 * f2 / P.fv[m]) / (1.0 + q * q));
    }
    if (SPH) return (a_cl + a_rot + 0.003 * a_cl + a_vib) * P.tweak * 8.685889e3;
    return (a_cl * 1.003 + a_rot + a_vib) * P.tweak * 8.685889e3;
}

struct WnlArgs {
    Fan3DArgs f;             // atmosphere, ground and boundary layer, absorption constants
    double c_src;            // atmo::c at the source (the beta0 denominator)
    const double* rows;      // kPathWnl rows of all rays
    const long long* row_off;   // [n_rays + 1] first row of each ray, then the total
    const long long* row_n;     // [n_rays] rows of each ray
    double* tab;             // [rows][3] per-row scratch: s, beta, beta_caustic
    int n_rays;
    int len, logm;           // N samples, log2(N / 2)
    double dt;               // t[1] - t[0]
    const double* p_init;    // [N] source waveform [Pa]
    const double* dden;      // [N] t[n+1] - t[n-1] (one-sided at the ends)
    const double* tukey;     // [N] Tukey window (parameter 0.8)
    const double* freq;      // [N/2 + 1] 1/dt * n / N
    const double* filt1;     // [N/2 + 1] low-pass of the non-linear term
    const double* filt2;     // [N/2 + 1] low-pass of the whole spectrum
    const double2* tw;       // [N/2] exp(-2 pi i k / N)
    double ds_wvfrm, wvfrm_ref, out_step;
    long long max_steps;     // Heun steps per ray before the ray is given up (status 2)
    double* u_out;           // [n_rays][N] u = p / p0 at the end
    double* info;            // [n_rays][kWnlInfo]
    double* events;          // nullable: [n_rays][event_cap][kWnlEventCols]
    int event_cap;
    double* snaps;           // nullable: [n_rays][snap_cap][1 + N + 2 (N/2 + 1)]
    int snap_cap;
};

// Segment of x on the shared knots of the six splines (the s column of the
// scratch table, stride 3): a forward walk from `k` (s only grows within a
// bounce).  For x inside the knots this is the segment interp::find_segment
// (interpolation.cpp:14-48) returns from any cached index, except when x
// equals a knot, where the two neighbouring segments give the same value up
// to rounding; outside the knots the segment is kept (the reference keeps its
// cached one and prints a warning; counted in `oob`).
__device__ __forceinline__ int seg_of(double x, const double* S, int L, int k, int& oob) {
    if (!(x <= S[(L - 1) * 3] && x >= S[0])) { oob++; return k; }
    while (k < L - 2 && S[(k + 1) * 3] < x) k++;
    while (k > 0 && S[k * 3] > x) k--;
    return k;
}

// interp::eval_f of a linear spline on segment k, knots s and values at
// F[i * stride]; the slope (interp::set) from the same two knots.
__device__ __forceinline__ double lin_at(double x, const double* S, const double* F, int stride, int k) {
    const double s0 = S[k * 3], s1 = S[(k + 1) * 3];
    const double f0 = F[(size_t)k * stride], f1 = F[(size_t)(k + 1) * stride];
    return f0 + (x - s0) * ((f1 - f0) / (s1 - s0));
}

__device__ __forceinline__ int brev(int k, int logm) { return (int)(__brev((unsigned)k) >> (32 - logm)); }

// In-place complex FFT of length M in shared memory, forward sign,
// natural-order input, bit-reversed output (decimation in frequency).
__device__ void cfft_dif(double2* W, const double2* __restrict__ tw, int M) {
    for (int h = M >> 1; h >= 1; h >>= 1) {
        const int mh = M / h;
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            const int j = b & (h - 1);
            const int i0 = ((b - j) << 1) + j, i1 = i0 + h;
            const double2 x0 = W[i0], x1 = W[i1];
            const double2 w = tw[j * mh];
            const double dx = x0.x - x1.x, dy = x0.y - x1.y;
            W[i0] = make_double2(x0.x + x1.x, x0.y + x1.y);
            W[i1] = make_double2(dx * w.x - dy * w.y, dx * w.y + dy * w.x);
        }
        __syncthreads();
    }
}

// In-place complex FFT of length M, inverse sign, unnormalised,
// bit-reversed input, natural-order output (decimation in time).
__device__ void cfft_dit_inv(double2* W, const double2* __restrict__ tw, int M) {
    for (int h = 1; h < M; h <<= 1) {
        const int mh = M / h;
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            const int j = b & (h - 1);
            const int i0 = ((b - j) << 1) + j, i1 = i0 + h;
            const double2 w = tw[j * mh];
            const double2 x0 = W[i0], x1 = W[i1];
            const double tx = x1.x * w.x + x1.y * w.y, ty = x1.y * w.x - x1.x * w.y;   // x1 conj(w)
            W[i0] = make_double2(x0.x + tx, x0.y + ty);
            W[i1] = make_double2(x0.x - tx, x0.y - ty);
        }
        __syncthreads();
    }
}

// Bin k (0..M) of the real FFT of length N = 2M from the bit-reversed
// complex FFT Z of the packed series z[m] = x[2m] + i x[2m+1].
__device__ __forceinline__ double2 rfft_bin(const double2* W, const double2* __restrict__ tw, int k, int M, int logm) {
    const double2 Z1 = W[brev(k & (M - 1), logm)];
    const double2 Z2 = W[brev((M - k) & (M - 1), logm)];
    const double Ex = 0.5 * (Z1.x + Z2.x), Ey = 0.5 * (Z1.y - Z2.y);
    const double Ox = 0.5 * (Z1.y + Z2.y), Oy = -0.5 * (Z1.x - Z2.x);
    const double2 w = k < M ? tw[k] : make_double2(-1.0, 0.0);
    return make_double2(Ex + (w.x * Ox - w.y * Oy), Ey + (w.x * Oy + w.y * Ox));
}

// Packed input bin k (0..M-1) of the inverse real FFT from the half
// spectrum U (imaginary parts of bins 0 and M dropped, as a c2r does).
__device__ __forceinline__ double2 irfft_pack(const double2* U, const double2* __restrict__ tw, int k, int M) {
    double2 X1 = U[k], X2 = U[M - k];
    if (k == 0) { X1.y = 0.0; X2.y = 0.0; }
    const double Ax = X1.x + X2.x, Ay = X1.y - X2.y;
    const double Dx = X1.x - X2.x, Dy = X1.y + X2.y;
    const double2 w = tw[k];
    const double Bx = Dx * w.x + Dy * w.y, By = Dy * w.x - Dx * w.y;   // D conj(w)
    return make_double2(Ax - By, Ay + Bx);
}

__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    return red[32];
}

// Scalars of the step loop, written by thread 0 and read by all.
struct WnlScal {
    double s, ds, s_tot, s_prev, Uf_max;
    double beta_c, beta_n, w1, w2, w3, fac;   // fac = -c(s) / c0
    double p0, c0, rho0, nu0, cg0, D0, beta0, t_ref, ray_length;
    double snap_label;
    SBPoint sp;
    long long steps;
    int shifts, snap, L, oob, n_ev, n_snap, started;
    int ks;                        // segment of s on the splines' knots
};

// atmo::c / rho / u / v at a row's height coordinate (3D: altitude z; SPH:
// radius r, altitude r - r_earth), clamped to the profile as
// atmo_state.3d.strat.cpp:148-180 and atmo_state.sph.strat.cpp do; u, v with
// the boundary-layer scaling.
struct AtmoPt { double c, rho, u, v; };
template <bool SPH>
__device__ __forceinline__ AtmoPt atmo_at(const Fan3DArgs& a, double h) {
    const double z = SPH ? h - a.r_earth : h;
    const double ze = fmin(fmax(z, a.z_lo), a.z_hi);
    const int sg = seg_walk(a.knots, a.n_knots, ze, seg_guess(ze, a.z_lo, a.inv_dz, a.n_knots));
    const double* r0 = a.knots + sg * kStride;
    const Cubic q = cubic_at(r0, ze);
    const double sc = SPH ? bl_scale_sph(a, h) : bl_scale(a, z);
    AtmoPt p;
    p.c = cubic_f(r0, q, 2);
    p.u = cubic_f(r0, q, 4) * sc;
    p.v = cubic_f(r0, q, 6) * sc;
    p.rho = cubic_f(r0, q, 8);
    return p;
}

__device__ __forceinline__ double nu_mag(const double* r) {
    return sqrt(r[3] * r[3] + r[4] * r[4] + r[5] * r[5]);
}

// |c_g| at a row from c nu / |nu| plus the winds: 3D (x, y, z) takes (u, v, 0),
// SPH (r, lat, lon) takes (w = 0, v, u) (main.infraga.3d.cpp:1321-1325,
// main.infraga.sph.cpp:1303-1307).
template <bool SPH>
__device__ __forceinline__ double group_speed(const double* r, const AtmoPt& p, double nu) {
    const double g0 = p.c * r[3] / nu + (SPH ? 0.0 : p.u);
    const double g1 = p.c * r[4] / nu + p.v;
    const double g2 = p.c * r[5] / nu + (SPH ? p.u : 0.0);
    return sqrt(g0 * g0 + g1 * g1 + g2 * g2);
}

// Chord between rows r0 and r1: wnl_wvfrm's spline knots (3D: Euclidean;
// SPH: dr, r0 dlat, r0 cos(lat0) dlon, geoac.eqset.sph.strat.cpp:907-911) or,
// with MID, run_wnl_wvfrm's search for the reference row (SPH: at the
// segment's midpoint radius and latitude, main.infraga.sph.cpp:1294-1299).
template <bool SPH, bool MID>
__device__ __forceinline__ double chord(const double* r0, const double* r1) {
    const double d0 = r1[0] - r0[0], d1 = r1[1] - r0[1], d2 = r1[2] - r0[2];
    if (!SPH) return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    const double r = MID ? r0[0] + d0 / 2.0 : r0[0];
    const double t = MID ? r0[1] + d1 / 2.0 : r0[1];
    const double a1 = r * d1, a2 = r * cos(t) * d2;
    return sqrt(d0 * d0 + a1 * a1 + a2 * a2);
}

// SPH: infraga-sph's wnl_wvfrm (geoac.eqset.sph.strat.cpp:855-1130) with its
// differences: spherical chords, a 1e-7 km step floor (1e-5 in 3D), strict
// caustic tests (s + ds < s_tot, D(s) D(s + ds) < 0), the spherical absorption.
template <bool SPH>
__global__ void __launch_bounds__(kWnlThreads, 1) wnl3d_kernel(const __grid_constant__ WnlArgs A) {
    extern __shared__ double sm[];
    const int N = A.len, M = N >> 1, logm = A.logm;
    double* u = sm;                                              // [N]
    double2* U = reinterpret_cast<double2*>(sm + N);             // [M + 1]
    double2* W = U + (M + 1);                                    // [M]
    WnlScal& S = *reinterpret_cast<WnlScal*>(W + M);
    double* red = reinterpret_cast<double*>(&S + 1);             // [40]: block_max, then two broadcasts
    const int ray = blockIdx.x;
    if (ray >= A.n_rays) return;
    const Fan3DArgs& a = A.f;
    const double* R = A.rows + (size_t)A.row_off[ray] * kWnlCols;
    double* Tb = A.tab + (size_t)A.row_off[ray] * 3;
    // rows the trace wrote, within the range reserved for the ray
    const long long nrow = min(A.row_n[ray], A.row_off[ray + 1] - A.row_off[ray]);
    double* ev = A.events ? A.events + (size_t)ray * A.event_cap * kWnlEventCols : nullptr;
    const size_t snap_w = 1 + (size_t)N + 2 * (size_t)(M + 1);
    double* sn = A.snaps ? A.snaps + (size_t)ray * A.snap_cap * snap_w : nullptr;
    const int tid = threadIdx.x, T = blockDim.x;

    for (int n = tid; n < N; n += T) u[n] = 0.0;
    if (tid == 0) {
        S.ray_length = 0.0; S.started = 0; S.steps = 0; S.shifts = 0; S.oob = 0; S.n_ev = 0; S.n_snap = 0;
        S.p0 = 0.0; S.t_ref = 0.0; S.c0 = S.rho0 = S.nu0 = S.cg0 = S.D0 = S.beta0 = 0.0;
    }
    __syncthreads();

    long long b = 0;   // first row of the current bounce segment
    long long last_row = -1;
    double tt_sum = 0.0;   // run_wnl_wvfrm's travel_time_sum: each bounce to its row k - 1
    while (b < nrow) {
        long long e = b;   // rows b..e: m = 0..K of one bounce
        while (e + 1 < nrow && R[(e + 1) * kWnlCols + 9] != 0.0) e++;
        last_row = e;
        const int K = (int)(e - b);
        if (K >= 1) tt_sum += R[(e - 1) * kWnlCols + 7];
        // ---- run_wnl_wvfrm's bounce step (main.infraga.3d.cpp:1311-1347) ----
        int k1 = -1, first = 0;
        if (tid == 0) {
            if (!S.started) {
                for (int j = 0; j < K; j++) {
                    const double* r0 = R + (b + j) * kWnlCols;
                    const double* r1 = r0 + kWnlCols;
                    S.ray_length += chord<SPH, true>(r0, r1);
                    if (S.ray_length >= A.wvfrm_ref) {
                        // reference quantities at row j + 1
                        const AtmoPt p = atmo_at<SPH>(a, r1[SPH ? 0 : 2]);
                        S.c0 = p.c; S.rho0 = p.rho;
                        S.nu0 = nu_mag(r1);
                        S.cg0 = group_speed<SPH>(r1, p, S.nu0);
                        S.D0 = r1[6];
                        S.t_ref = r1[7];
                        S.started = 1;
                        k1 = j + 1; first = 1;
                        break;
                    }
                }
            } else {
                k1 = 0;
            }
            S.L = k1 < 0 ? -1 : K - k1;      // rows k1 .. K-1 (geoac::wnl_wvfrm's k1, k2 = k)
            S.s_prev = first ? A.wvfrm_ref : S.ray_length;
            red[33] = (double)k1; red[34] = (double)first;
        }
        __syncthreads();
        k1 = (int)red[33]; first = (int)red[34];
        if (k1 >= 0) {
            if (first) {   // p0 = max |p|, u = p / p0
                double m = 0.0;
                for (int n = tid; n < N; n += T) m = fmax(m, fabs(A.p_init[n]));
                m = block_max(m, red);
                for (int n = tid; n < N; n += T) u[n] = A.p_init[n] / m;
                if (tid == 0) {
                    S.p0 = m;
                    S.beta0 = 1.2 * S.p0 / ((S.rho0 * 1.0e3) * ((S.c0 * 1.0e3) * (S.c0 * 1.0e3))) * (S.nu0 * S.c0) /
                              (S.cg0 * A.c_src);
                }
                __syncthreads();
            }
            const int L = S.L;
            const double* Rs = R + (b + k1) * kWnlCols;   // the segment's first row
            double* Ts = Tb + (b + k1) * 3;
            // ---- spline knots (geoac.eqset.3d.strat.cpp:791-831) ----
            for (int i = tid; i < L; i += T) {   // chord to the next row, summed below
                if (i + 1 < L) {
                    const double* r0 = Rs + (size_t)i * kWnlCols;
                    Ts[(size_t)(i + 1) * 3] = chord<SPH, false>(r0, r0 + kWnlCols);
                }
            }
            __syncthreads();
            if (tid == 0 && L > 0) {
                double s = 0.0;
                Ts[0] = 0.0;
                for (int i = 1; i < L; i++) { s += Ts[(size_t)i * 3]; Ts[(size_t)i * 3] = s; }
                S.s_tot = s;
            }
            __syncthreads();
            {
                const double k0 = S.D0 * S.rho0 * (S.cg0 * S.cg0 * S.cg0);
                const double k2 = S.c0 * (S.nu0 * S.nu0 * S.nu0);
                for (int i = tid; i < L; i += T) {
                    const double* r = Rs + (size_t)i * kWnlCols;
                    const AtmoPt p = atmo_at<SPH>(a, r[SPH ? 0 : 2]);
                    const double nu = nu_mag(r);
                    const double c3 = p.c * p.c * p.c, n3 = nu * nu * nu;
                    Ts[(size_t)i * 3 + 1] = S.beta0 * sqrt(fabs(k0 / (r[6] * p.rho * c3) * (p.c * n3) / k2));
                    if (i >= 1) {
                        const double dD = (r[6] - r[6 - kWnlCols]) / (Ts[(size_t)i * 3] - Ts[(size_t)(i - 1) * 3]);
                        Ts[(size_t)i * 3 + 2] = S.beta0 * sqrt(fabs(k0 / (dD * p.rho * c3) * (p.c * n3) / k2));
                    }
                }
            }
            __syncthreads();
            if (tid == 0 && L > 1) Ts[2] = Ts[5];   // beta_caustic[0] = beta_caustic[1]
            // ---- U = FFT{u}, Uf_max (:858-869) ----
            for (int m = tid; m < M; m += T) W[m] = make_double2(u[2 * m], u[2 * m + 1]);
            __syncthreads();
            cfft_dif(W, A.tw, M);
            double fm = 0.0;
            for (int k = tid; k <= M; k += T) {
                const double2 X = rfft_bin(W, A.tw, k, M, logm);
                U[k] = X;
                fm = fmax(fm, A.freq[k] * sqrt(X.x * X.x + X.y * X.y));
            }
            fm = block_max(fm, red);
            if (tid == 0) {
                S.Uf_max = fm; S.s = 0.0; S.ds = A.ds_wvfrm;
                S.ks = 0;
            }
            __syncthreads();
            // ---- Heun steps (:871-995), at most max_steps over the ray ----
            while (L > 1 && S.s < S.s_tot && S.steps < A.max_steps) {
                if (tid == 0) {
                    const double s = S.s, sp = S.s_prev;
                    const double* sx = Ts;
                    int& oob = S.oob;
                    S.snap = 0;
                    if (A.out_step < 1.0e4 &&
                        fabs(A.out_step * ceil((s + sp + S.ds) / A.out_step) - A.out_step * ceil((s + sp) / A.out_step)) > 0.0) {
                        S.snap = 1;
                        S.snap_label = A.out_step * ceil((s + sp) / A.out_step);
                    }
                    const int ks = seg_of(s, sx, L, S.ks, oob);
                    S.ks = ks;
                    const double Ds = lin_at(s, sx, Rs + 6, kWnlCols, ks);
                    const double bc = fabs(Ds) >= 0.5 ? lin_at(s, sx, Ts + 1, 3, ks) : lin_at(s, sx, Ts + 2, 3, ks);
                    // std::min / std::max as the reference calls them: a NaN step stays NaN
                    // (and ends the loop through s)
                    double ds = A.ds_wvfrm / (kPi * S.Uf_max * bc);
                    ds = (1.0 < ds) ? 1.0 : ds;
                    ds = (ds < (SPH ? 1.0e-7 : 1.0e-5)) ? (SPH ? 1.0e-7 : 1.0e-5) : ds;
                    const double s_last = sx[(size_t)(L - 1) * 3];
                    const double sn = (s_last < s + ds) ? s_last : s + ds;
                    const int kn = seg_of(sn, sx, L, ks, oob);
                    const double Dn = lin_at(sn, sx, Rs + 6, kWnlCols, kn);
                    const double bn = fabs(Dn) >= 0.5 ? lin_at(sn, sx, Ts + 1, 3, kn) : lin_at(sn, sx, Ts + 2, 3, kn);
                    if (fabs(10.0 * ceil((s + sp + ds) / 10.0) - 10.0 * ceil((s + sp) / 10.0)) > 0.0) {
                        const double zs = SPH ? lin_at(s, sx, Rs + 0, kWnlCols, ks) - a.r_earth
                                              : lin_at(s, sx, Rs + 2, kWnlCols, ks);
                        if (ev && S.n_ev < A.event_cap) {
                            double* o = ev + (size_t)S.n_ev * kWnlEventCols;
                            o[0] = 0.0; o[1] = 10.0 * ceil((s + sp) / 10.0); o[2] = zs; o[3] = bc;
                        }
                        S.n_ev++;
                    }
                    int shift = 0;
                    if (SPH ? (s + ds < S.s_tot) : (s + ds <= S.s_tot)) {
                        const double D1s = lin_at(s + ds, sx, Rs + 6, kWnlCols, seg_of(s + ds, sx, L, ks, oob));
                        const double D0s = Ds;
                        if (SPH ? (D0s * D1s < 0.0) : (D0s * D1s <= 0.0)) {
                            shift = 1;
                            if (ev && S.n_ev < A.event_cap) {
                                double* o = ev + (size_t)S.n_ev * kWnlEventCols;
                                o[0] = 1.0; o[1] = s + sp; o[2] = 0.0; o[3] = 0.0;
                            }
                            S.n_ev++;
                            S.shifts++;
                        }
                    }
                    // absorption point (the reference evaluates it inside the bin loop)
                    // (the horizontal coordinates do not enter a stratified atmosphere)
                    const double hs = lin_at(s, sx, Rs + (SPH ? 0 : 2), kWnlCols, ks);
                    const AtmoPt p = atmo_at<SPH>(a, hs);
                    S.sp = sb_point<SPH>(p.c, p.rho, SPH ? hs - a.r_earth : hs, a.tweak_abs, a.sb);
                    S.fac = -p.c / S.c0;
                    S.ds = ds; S.beta_c = bc; S.beta_n = bn;
                    S.w1 = ds * (bc + bn) / 2.0;
                    S.w2 = (ds * ds) / 2.0 * bc * bn;
                    S.w3 = (ds * ds * ds) / 8.0 * (bc * bc) * bn;
                    S.snap = S.snap | (shift << 1);
                }
                __syncthreads();
                const int flags = S.snap;
                if ((flags & 1) && sn) {   // sc_spectrum / sc_waveform at this step's start
                    if (S.n_snap < A.snap_cap) {
                        double* o = sn + (size_t)S.n_snap * snap_w;
                        if (tid == 0) o[0] = S.snap_label;
                        for (int n = tid; n < N; n += T) o[1 + n] = u[n];
                        for (int k = tid; k <= M; k += T) { o[1 + N + 2 * k] = U[k].x; o[2 + N + 2 * k] = U[k].y; }
                    }
                    __syncthreads();
                    if (tid == 0) S.n_snap++;
                }
                if ((flags & 1) && !sn && tid == 0) S.n_snap++;
                // non-linear source w1 u^2 + w2 u d(u^2)/dt + w3 (d(u^2)/dt)^2, packed
                const double w1 = S.w1, w2 = S.w2, w3 = S.w3;
                for (int m = tid; m < M; m += T) {
                    double q[2];
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int n = 2 * m + h;
                        const double un = u[n];
                        const double u2 = un * un;
                        double du2;
                        if (n == 0) du2 = (u[1] * u[1] - u2) / A.dden[0];
                        else if (n == N - 1) du2 = (u2 - u[N - 2] * u[N - 2]) / A.dden[N - 1];
                        else du2 = (u[n + 1] * u[n + 1] - u[n - 1] * u[n - 1]) / A.dden[n];
                        q[h] = w1 * u2 + w2 * (un * du2) + w3 * (du2 * du2);
                    }
                    W[m] = make_double2(q[0], q[1]);
                }
                __syncthreads();
                cfft_dif(W, A.tw, M);
                // spectral step: caustic phase shift, Heun update, absorption, filters
                const double ds = S.ds, fac = S.fac;
                const SBPoint sp = S.sp;
                fm = 0.0;
                for (int k = tid; k <= M; k += T) {
                    const double2 Q = rfft_bin(W, A.tw, k, M, logm);
                    double2 X = U[k];
                    if (flags & 2) X = make_double2(-X.y, X.x);
                    const double fr = A.freq[k];
                    const double pf = kPi * fr;
                    X.x -= pf * Q.y * A.filt1[k];
                    X.y += pf * Q.x * A.filt1[k];
                    const double absorp = iga_exp10(fac * sb_bin<SPH>(sp, fr) * ds / 10.0);
                    const double g = absorp * A.filt2[k];
                    X.x *= g; X.y *= g;
                    U[k] = X;
                    fm = fmax(fm, fr * sqrt(X.x * X.x + X.y * X.y));
                }
                fm = block_max(fm, red);   // (its barriers also order the U writes before the reads below)
                for (int k = tid; k < M; k += T) W[brev(k, logm)] = irfft_pack(U, A.tw, k, M);
                __syncthreads();
                cfft_dit_inv(W, A.tw, M);
                const double nd = (double)N;
                for (int m = tid; m < M; m += T) {
                    const double2 z = W[m];
                    u[2 * m] = z.x * A.tukey[2 * m] / nd;
                    u[2 * m + 1] = z.y * A.tukey[2 * m + 1] / nd;
                }
                if (tid == 0) { S.Uf_max = fm; S.s += ds; S.steps++; }
                __syncthreads();
            }
            if (tid == 0) {
                const double st = L > 0 ? S.s_tot : 0.0;
                if (first) S.ray_length = st;
                else S.ray_length += st;
            }
            __syncthreads();
        }
        b = e + 1;
    }
    // ---- output (main.infraga.3d.cpp:1376-1411) ----
    for (int n = tid; n < N; n += T) A.u_out[(size_t)ray * N + n] = u[n];
    if (tid == 0) {
        double* o = A.info + (size_t)ray * kWnlInfo;
        double scale_sq = 0.0;
        if (last_row >= 0 && S.started) {
            const double* r = R + last_row * kWnlCols;
            const AtmoPt p = atmo_at<SPH>(a, r[SPH ? 0 : 2]);
            const double nu = sqrt(r[3] * r[3] + r[4] * r[4] + r[5] * r[5]);
            const double cg = group_speed<SPH>(r, p, nu);
            scale_sq = sqrt(fabs((p.rho * (p.c * p.c * p.c) * nu) / (S.rho0 * (S.c0 * S.c0 * S.c0) * S.nu0) *
                                 (S.cg0 * S.D0) / (cg * r[6])));
        }
        o[0] = !S.started ? 1.0 : (S.steps >= A.max_steps ? 2.0 : 0.0);
        o[1] = (double)S.steps;
        o[2] = (double)S.shifts;
        o[3] = (double)S.n_ev;
        o[4] = (double)S.n_snap;
        o[5] = S.t_ref;
        o[6] = S.p0;
        o[7] = scale_sq;
        o[8] = S.ray_length;
        o[9] = S.c0; o[10] = S.rho0; o[11] = S.nu0; o[12] = S.cg0; o[13] = S.D0;
        o[14] = (double)S.oob;
        o[15] = S.beta0;
        o[16] = tt_sum;
    }
}

}  // namespace iga

namespace {

struct DevMem {   // cudaMalloc'd scratch freed on scope exit
    std::vector<void*> ptrs;
    ~DevMem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    int get(T** out, size_t count) {
        void* p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(wnl)");
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return IGA_OK;
    }
    template <class T>
    int put(T** out, const T* src, size_t count, cudaStream_t st) {
        int rc = get(out, count);
        if (rc) return rc;
        IGA_CUDA(cudaMemcpyAsync(*out, src, count * sizeof(T), cudaMemcpyHostToDevice, st), "H2D wnl tables");
        return IGA_OK;
    }
};

struct StreamGuard {
    cudaStream_t st = nullptr;
    ~StreamGuard() {
        if (st) cudaStreamDestroy(st);
    }
};

constexpr double kPiRef = 3.141592653589793238462643;   // Pi of geoac.params.3d.cpp:10

}  // namespace

extern "C" int iga_wnl_params_default(iga_atmo_t h, iga_wnl_params* p) {
    if (!h || !p) return IGA_E_INVALID;
    std::memset(p, 0, sizeof(*p));
    int rc = iga_fan_params_default(h, &p->fan);
    if (rc) return rc;
    p->fan.calc_amp = 1;
    p->fan.write_rays = 1;
    p->ds_wvfrm = 0.5;                  // geoac::ds_wvfrm (geoac.params.3d.cpp)
    p->wvfrm_ref = 1.0;                 // run_wnl_wvfrm's wvfrm_ref
    p->out_step = 1.0e10;               // wvfrm_out_step
    p->filt1_g = 0.5; p->filt1_n1 = 4.0; p->filt1_n2 = 0.5;    // waveforms.cpp:31-37
    p->filt2_g = 0.75; p->filt2_n1 = 2.0; p->filt2_n2 = 1.0;
    p->max_steps = 1000000;
    return IGA_OK;
}

extern "C" int iga_wnl_run(iga_atmo_t h, const iga_wnl_params* wp, const double* theta_deg, const double* phi_deg,
                           int n_rays, const double* wv_t, const double* wv_p, int len, double* u_out, double* info,
                           double* arrivals, int* n_arr, int* ray_status, double* events, int event_cap,
                           double* snaps, int snap_cap) {
    if (!h || !wp) return IGA_E_INVALID;
    if (n_rays < 0 || event_cap < 0 || snap_cap < 0) return IGA_E_INVALID;
    if (n_rays > 0 && (!theta_deg || !phi_deg || !wv_t || !wv_p || !u_out || !info)) return IGA_E_INVALID;
    if ((event_cap > 0 && !events) || (snap_cap > 0 && !snaps)) return IGA_E_INVALID;
    if (len < 16 || len > iga::kWnlMaxLen || (len & (len - 1)) != 0) {
        g_cuda_err = "waveform length: a power of two from 16 to 8192 samples";
        return IGA_E_UNSUPPORTED;
    }
    if (h->kind != 0 || h->has_topo) {
        g_cuda_err = "weakly non-linear waveform: stratified flat-ground atmospheres only (3D or spherical geometry)";
        return IGA_E_UNSUPPORTED;
    }
    const bool sph = wp->fan.geometry == IGA_GEOM_SPH;
    if (!(wp->ds_wvfrm > 0.0)) return IGA_E_INVALID;
    iga_fan_params q = wp->fan;
    q.calc_amp = 1;
    q.write_rays = 1;               // run_wnl_wvfrm sums time and absorption per step (:1296-1299)
    q.precision = IGA_FP64;
    q.turn_ht_min = -1.0e30;        // no turning-height cut in run_wnl_wvfrm
    if (sph) q.time_max = 1.0e30;   // nor the spherical run_prop's travel-time cap
    int rc = validate(&q, n_rays);
    if (rc) return rc;
    if (n_rays == 0) return IGA_OK;
    NvtxRange nv("iga_wnl_run");
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    StreamGuard sg;
    IGA_CUDA(cudaStreamCreateWithFlags(&sg.st, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaStream_t st = sg.st;
    const int nb = q.bounces + 1;
    const size_t n = (size_t)n_rays;
    const int N = len, M = len / 2;

    DevMem mem;
    double *d_th, *d_ph, *d_arr;
    int *d_n, *d_status;
    long long* d_steps;
    void* d_ws;
    if ((rc = mem.put(&d_th, theta_deg, n, st)) || (rc = mem.put(&d_ph, phi_deg, n, st)) ||
        (rc = mem.get(&d_arr, n * nb * IGA_ARRIVAL_COLS)) || (rc = mem.get(&d_n, n)) || (rc = mem.get(&d_status, n)) ||
        (rc = mem.get(&d_steps, n)) || (rc = mem.get(reinterpret_cast<unsigned char**>(&d_ws), iga_fan_workspace_bytes())))
        return rc;
    // step counts, then every row of every bounce (kPathWnl)
    {
        iga_fan_params c = q;
        c.calc_amp = 0;
        if ((rc = fan_device(h, &c, d_th, d_ph, n_rays, d_arr, d_n, d_steps, nullptr, nullptr, d_ws, st, 0))) return rc;
    }
    std::vector<long long> steps(n), off(n + 1, 0);
    IGA_CUDA(cudaMemcpyAsync(steps.data(), d_steps, sizeof(long long) * n, cudaMemcpyDeviceToHost, st), "D2H steps");
    IGA_CUDA(cudaStreamSynchronize(st), "wnl step-count pass");
    for (size_t i = 0; i < n; i++) off[i + 1] = off[i] + iga::path_rows_bound(iga::kPathWnl, steps[i], nb);
    PathSpec ps;
    ps.mode = iga::kPathWnl;
    long long* d_off;
    double* d_tab;
    if ((rc = mem.get(&ps.rows, (size_t)off[n] * iga::kWnlCols)) || (rc = mem.put(&d_off, off.data(), n + 1, st)) ||
        (rc = mem.get(&ps.n, n)) || (rc = mem.get(&d_tab, (size_t)off[n] * 3)))
        return rc;
    ps.off = d_off;
    if ((rc = fan_device(h, &q, d_th, d_ph, n_rays, d_arr, d_n, d_steps, d_status, nullptr, d_ws, st, 0, &ps))) return rc;

    // waveform tables, as wnl_wvfrm builds them (geoac.eqset.3d.strat.cpp:835-855)
    const double dt = wv_t[1] - wv_t[0];
    std::vector<double> dden(N), tukey(N), freq(M + 1), f1(M + 1), f2(M + 1), tw(2 * (size_t)M);
    dden[0] = wv_t[1] - wv_t[0];
    for (int i = 1; i < N - 1; i++) dden[i] = wv_t[i + 1] - wv_t[i - 1];
    dden[N - 1] = wv_t[N - 1] - wv_t[N - 2];
    const double tp = 0.8;
    for (int i = 0; i < N; i++) {
        if (i < tp * (N - 1) / 2.0) tukey[i] = 1.0 / 2.0 * (1.0 + cos(kPiRef * (2.0 * i / (tp * (N - 1)) - 1.0)));
        else if (i > (N - 1) * (1.0 - tp / 2.0))
            tukey[i] = 1.0 / 2.0 * (1.0 + cos(kPiRef * (2.0 * i / (tp * (N - 1)) - 2.0 / tp + 1.0)));
        else tukey[i] = 1.0;
    }
    const int fft_len = M + 1;
    for (int k = 0; k <= M; k++) {
        freq[k] = 1.0 / dt * k / N;
        f1[k] = pow(1.0 + pow(k / (wp->filt1_g * fft_len), wp->filt1_n1), -wp->filt1_n2);
        f2[k] = pow(1.0 + pow(k / (wp->filt2_g * fft_len), wp->filt2_n1), -wp->filt2_n2);
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < M; k++) {
        tw[2 * k] = cos(two_pi * (double)k / (double)N);
        tw[2 * k + 1] = -sin(two_pi * (double)k / (double)N);
    }
    iga::WnlArgs A{};
    if ((rc = build_args(h, &q, A.f))) return rc;
    double *d_p, *d_dden, *d_tuk, *d_freq, *d_f1, *d_f2, *d_tw, *d_u, *d_info, *d_ev = nullptr, *d_sn = nullptr;
    if ((rc = mem.put(&d_p, wv_p, N, st)) || (rc = mem.put(&d_dden, dden.data(), N, st)) ||
        (rc = mem.put(&d_tuk, tukey.data(), N, st)) || (rc = mem.put(&d_freq, freq.data(), M + 1, st)) ||
        (rc = mem.put(&d_f1, f1.data(), M + 1, st)) || (rc = mem.put(&d_f2, f2.data(), M + 1, st)) ||
        (rc = mem.put(&d_tw, tw.data(), 2 * (size_t)M, st)) || (rc = mem.get(&d_u, n * N)) ||
        (rc = mem.get(&d_info, n * iga::kWnlInfo)))
        return rc;
    const size_t snap_w = 1 + (size_t)N + 2 * (size_t)(M + 1);
    if (event_cap > 0) {
        if ((rc = mem.get(&d_ev, n * event_cap * iga::kWnlEventCols))) return rc;
        IGA_CUDA(cudaMemsetAsync(d_ev, 0, sizeof(double) * n * event_cap * iga::kWnlEventCols, st), "memset events");
    }
    if (snap_cap > 0 && (rc = mem.get(&d_sn, n * snap_cap * snap_w))) return rc;
    A.c_src = A.f.c0;
    A.rows = ps.rows; A.row_off = d_off; A.row_n = ps.n; A.tab = d_tab; A.n_rays = n_rays;
    A.len = N;
    A.logm = 0;
    while ((1 << A.logm) < M) A.logm++;
    A.dt = dt;
    A.p_init = d_p; A.dden = d_dden; A.tukey = d_tuk; A.freq = d_freq; A.filt1 = d_f1; A.filt2 = d_f2;
    A.tw = reinterpret_cast<const double2*>(d_tw);
    A.ds_wvfrm = wp->ds_wvfrm; A.wvfrm_ref = wp->wvfrm_ref; A.out_step = wp->out_step;
    A.max_steps = wp->max_steps > 0 ? wp->max_steps : 1000000;
    A.u_out = d_u; A.info = d_info;
    A.events = d_ev; A.event_cap = event_cap;
    A.snaps = d_sn; A.snap_cap = snap_cap;
    const size_t smem = sizeof(double) * ((size_t)N + 2 * (size_t)(M + 1) + 2 * (size_t)M) + sizeof(iga::WnlScal) +
                        40 * sizeof(double);
    auto kern = sph ? iga::wnl3d_kernel<true> : iga::wnl3d_kernel<false>;
    IGA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "wnl smem attribute");
    kern<<<n_rays, iga::kWnlThreads, smem, st>>>(A);
    IGA_CUDA(cudaGetLastError(), "wnl kernel launch");

    IGA_CUDA(cudaMemcpyAsync(u_out, d_u, sizeof(double) * n * N, cudaMemcpyDeviceToHost, st), "D2H wnl waveforms");
    IGA_CUDA(cudaMemcpyAsync(info, d_info, sizeof(double) * n * iga::kWnlInfo, cudaMemcpyDeviceToHost, st), "D2H wnl info");
    if (arrivals)
        IGA_CUDA(cudaMemcpyAsync(arrivals, d_arr, sizeof(double) * n * nb * IGA_ARRIVAL_COLS, cudaMemcpyDeviceToHost, st),
                 "D2H arrivals");
    if (n_arr) IGA_CUDA(cudaMemcpyAsync(n_arr, d_n, sizeof(int) * n, cudaMemcpyDeviceToHost, st), "D2H n_arr");
    if (ray_status) IGA_CUDA(cudaMemcpyAsync(ray_status, d_status, sizeof(int) * n, cudaMemcpyDeviceToHost, st), "D2H status");
    if (d_ev)
        IGA_CUDA(cudaMemcpyAsync(events, d_ev, sizeof(double) * n * event_cap * iga::kWnlEventCols, cudaMemcpyDeviceToHost, st),
                 "D2H wnl events");
    if (d_sn)
        IGA_CUDA(cudaMemcpyAsync(snaps, d_sn, sizeof(double) * n * snap_cap * snap_w, cudaMemcpyDeviceToHost, st),
                 "D2H wnl snapshots");
    IGA_CUDA(cudaStreamSynchronize(st), "wnl kernel");
    // truncated event or snapshot output: the counts in info give the room needed
    for (size_t i = 0; i < n; i++)
        if (info[i * iga::kWnlInfo + 3] > event_cap && event_cap > 0) return IGA_E_TRUNCATED;
    for (size_t i = 0; i < n; i++)
        if (info[i * iga::kWnlInfo + 4] > snap_cap && snap_cap > 0) return IGA_E_TRUNCATED;
    return IGA_OK;
}
