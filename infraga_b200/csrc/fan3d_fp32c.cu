// FP32-compensated ray-fan and eigenray-trace kernels: 3D Cartesian,
// stratified, flat ground.
//
// Same ray/Jacobian equations, RK4 driver, stop checks and bounce logic as
// the FP64 kernel (fan3d_fp64.cu, following geoac.eqset.3d.strat.cpp and
// rk4solver.cpp), with the arithmetic split by what each quantity needs:
//
//   * the four ray equations (x, y, z, nu_z) and the spline values and slopes
//     they read (c, u, v) in FP64, from a power-basis FP64 table in shared
//     memory; square roots and reciprocals from an FP32 estimate refined by
//     one Newton step in FP64;
//   * the eight Jacobian auxiliaries (X_th, mu_th_z, X_ph, mu_ph_z) in FP32:
//     their right-hand side in FP32 and their state summed with TwoSum
//     (hi/lo pairs), so the sum of ~1e5 small increments keeps FP64-like
//     accuracy;
//   * Sutherland-Bass absorption from an FP64-built table of alpha(z) (a
//     stratified profile makes alpha a function of altitude only);
//   * boundary-layer scaling, set_ds, travel time, absorption sums, ground
//     intercept, reflection and amplitude in FP64.
//
// The ray equations stay in FP64 because rays that graze a duct boundary have
// launch sensitivities |d(range)/d(inclination)| of 1e6..7e7 km/rad: an FP32
// ray state (whose ulp is ~6e-8 of the launch angle itself) moves their ground
// intercept by hundreds of metres.  With the ray equations in FP64 the
// intercept, travel time and turning height follow the FP64 kernel to
// rounding; the auxiliaries only set the amplitude, which tolerates FP32
// arithmetic once their state is summed with compensation.
#include <type_traits>

#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fan3d_common.cuh"

namespace iga {

namespace {

// 256 threads x 2 CTAs per SM caps the fan kernel at 128 registers: 16
// resident warps per SM (168 registers and 12 warps at 192 x 2 ran 9% slower,
// its few spills notwithstanding)
#ifndef IGA_FANC_THREADS
#define IGA_FANC_THREADS 256
#endif
#ifndef IGA_FANC_MINB
#define IGA_FANC_MINB 2
#endif
constexpr int kThreadsC = IGA_FANC_THREADS;
// Above this height X = exp(-(z-zg)/0.1) < 2e-22: S = (1-X)/(1+X) rounds to 1
// in FP64 and the X-terms of S' and S'' vanish against the spline slopes.
constexpr double kBlCutoffC = 5.0;

template <bool AMP> struct AuxN { static constexpr int n = AMP ? 8 : 1; };

// Focusing test.  Near a caustic the ray tube collapses: the Jacobian D at an
// arrival falls far below the largest |D| the ray has had, and the amplitude
// becomes ill-conditioned -- an error in the auxiliaries early on the path
// reaches the arrival amplified by 1e4..1e5 (the same amplification shows
// with the auxiliaries in FP64, one rounding order lower).  A ray that meets
// an arrival with |D| < kFocusRatio * max|D| before its first caustic is
// traced again from its launch with FP64 auxiliaries (about 1% of the rays
// of a 10-bounce fan); every other ray keeps its FP32 auxiliaries.
constexpr double kFocusRatio = 0.2;

// Per-ray constants: nu_x, nu_y and |nu_h|^2 in FP64 for the ray equations,
// copies and the mu_x, mu_y components in the auxiliaries' type T.
template <class T>
struct RayConstC {
    double nx, ny, nh2;
    T nxf, nyf, mtx, mty, mpx, mpy;
};

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ int seg_walk_c(const double* __restrict__ tab, int n, double z, int k) {
    while (k > 0 && z < tab[k * kStrideC]) --k;
    while (k < n - 2 && z > tab[(k + 1) * kStrideC]) ++k;
    return k;
}

// 1/sqrt(x) for x in the normal FP32 range: the FP32 estimate refined by one
// Newton step in FP64 (relative error below 1e-13).
__device__ __forceinline__ double rsqrt_c(double x) {
    const double r = (double)rsqrtf((float)x);
    const double h = 0.5 * x * r;
    return r * fma(-h, r, 1.5);
}

// Knuth's TwoSum: adds inc to the pair (hi, lo) and renormalises it.
template <class T>
__device__ __forceinline__ void acc_pair(T& hi, T& lo, T inc) {
    const T s = hi + inc;
    const T bb = s - hi;
    const T e = (hi - (s - bb)) + (inc - bb);
    const T l = lo + e;
    hi = s + l;
    lo = l - (hi - s);
}

// No-slip boundary-layer scaling S = (1-X)/(1+X), X = exp(-h/bl) over flat
// ground (bndlyr_sc / bndlyr_dsc, atmo_state.3d.strat.cpp:85-142) and its first
// two h-derivatives, in FP64: the wind and its gradient enter the ray equations,
// and for rays near a duct boundary an FP32 scaling shifts the intercept by
// tens of metres.  Only the lowest kBlCutoffC km pay for the exponential.
struct BlScale {
    double s0, ds, dds;
};

template <bool D2>
__device__ __forceinline__ BlScale bl_scale_c(double hz, double inv_bl) {
    BlScale b{1.0, 0.0, 0.0};
    if (hz < kBlCutoffC) {
        const double X = exp(-hz * inv_bl);
        const double iop = 1.0 / (1.0 + X);
        b.s0 = (1.0 - X) * iop;
        const double dX = -X * inv_bl;
        b.ds = -2.0 * dX * (iop * iop);
        if (D2) b.dds = -2.0 * (X * inv_bl * inv_bl * (iop * iop) - 2.0 * dX * dX * (iop * iop * iop));
    }
    return b;
}

// Right-hand side at state (yd, ya): update_refs (geoac.eqset.3d.strat.cpp:
// 225-328) + eval_src_eq (:333-389) on flat ground, the same algebra as rhs()
// in fan3d_common.cuh; ray part fd[0..3] in FP64, auxiliaries fa[0..7]
// (X_th, mu_th_z, X_ph, mu_ph_z) in T (FP32, or FP64 for a re-traced ray).
template <bool AMP, class T>
__device__ __forceinline__ void rhs_c(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                      const double* yd, const T* ya, const RayConstC<T>& rc, double* fd, T* fa) {
    const double z = yd[2];
    const double ze = fmin(fmax(z, a.z_lo), a.z_hi);
    seg = seg_walk_c(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStrideC;
    const double idx = r0[1];
    const double X = (ze - r0[0]) * idx;
    // power basis f = a0 + X (a1 + X (a2 + X a3)), f' = (a1 + 2X a2 + 3X^2 a3) / dz
    const double X2 = 2.0 * X, X3 = 3.0 * X * X;
    const double c = fma(X, fma(X, fma(X, r0[5], r0[4]), r0[3]), r0[2]);
    const double cz = fma(X3, r0[5], fma(X2, r0[4], r0[3])) * idx;
    const double u0 = fma(X, fma(X, fma(X, r0[9], r0[8]), r0[7]), r0[6]);
    const double u0z = fma(X3, r0[9], fma(X2, r0[8], r0[7])) * idx;
    const double v0 = fma(X, fma(X, fma(X, r0[13], r0[12]), r0[11]), r0[10]);
    const double v0z = fma(X3, r0[13], fma(X2, r0[12], r0[11])) * idx;
    const BlScale bl = bl_scale_c<AMP>(z - a.z0, a.inv_bl);
    const double sc0 = bl.s0, dsc = bl.ds;
    const double u = u0 * sc0, v = v0 * sc0;
    const double uz = u0z * sc0 + u0 * dsc;
    const double vz = v0z * sc0 + v0 * dsc;
    const double nz = yd[3];
    const double num2 = rc.nh2 + nz * nz;
    const double inum = rsqrt_c(num2);
    const double num = num2 * inum;
    const double cin = c * inum;
    const double cgx = cin * rc.nx + u;
    const double cgy = cin * rc.ny + v;
    const double cgz = cin * nz;
    const double icg = rsqrt_c(cgx * cgx + cgy * cgy + cgz * cgz);
    fd[0] = cgx * icg;
    fd[1] = cgy * icg;
    fd[2] = cgz * icg;
    const double Kz = num * cz + rc.nx * uz + rc.ny * vz;
    fd[3] = -icg * Kz;
    if (AMP) {
        // f'' = (2 a2 + 6 X a3) / dz^2, formed in T (auxiliaries only)
        const T idx2 = (T)(idx * idx), Xf6 = T(6) * (T)X;
        const T czz = fma_t(Xf6, (T)r0[5], T(2) * (T)r0[4]) * idx2;
        const T u0zz = fma_t(Xf6, (T)r0[9], T(2) * (T)r0[8]) * idx2;
        const T v0zz = fma_t(Xf6, (T)r0[13], T(2) * (T)r0[12]) * idx2;
        const T s0f = (T)bl.s0, dsf = (T)bl.ds, ddsf = (T)bl.dds;
        const T uzz = u0zz * s0f + T(2) * (T)u0z * dsf + (T)u0 * ddsf;
        const T vzz = v0zz * s0f + T(2) * (T)v0z * dsf + (T)v0 * ddsf;
        const T czf = (T)cz, uzf = (T)uz, vzf = (T)vz;
        const T inumf = (T)inum, icgf = (T)icg, numf = (T)num, Kzf = (T)Kz;
        const T cgxf = (T)cgx, cgyf = (T)cgy, cgzf = (T)cgz, nzf = (T)nz;
        const T cinf = (T)cin, cin2 = cinf * inumf;
        const T Xtz = ya[2], Xpz = ya[6], mtz = ya[3], mpz = ya[7];
        const T dc3 = Xtz * czf, dc4 = Xpz * czf;
        const T du3 = Xtz * uzf, du4 = Xpz * uzf;
        const T dv3 = Xtz * vzf + Xpz * vzf;   // reference's dv[3]/dv[4] accumulation (eqset.3d.strat.cpp:298)
        const T dnu0 = (rc.nxf * rc.mtx + rc.nyf * rc.mty + nzf * mtz) * inumf;
        const T dnu1 = (rc.nxf * rc.mpx + rc.nyf * rc.mpy + nzf * mpz) * inumf;
        const T g0x = rc.nxf * inumf * dc3 + cinf * rc.mtx - cin2 * rc.nxf * dnu0 + du3;
        const T g0y = rc.nyf * inumf * dc3 + cinf * rc.mty - cin2 * rc.nyf * dnu0 + dv3;
        const T g0z = nzf * inumf * dc3 + cinf * mtz - cin2 * nzf * dnu0;
        const T g1x = rc.nxf * inumf * dc4 + cinf * rc.mpx - cin2 * rc.nxf * dnu1 + du4;
        const T g1y = rc.nyf * inumf * dc4 + cinf * rc.mpy - cin2 * rc.nyf * dnu1;
        const T g1z = nzf * inumf * dc4 + cinf * mpz - cin2 * nzf * dnu1;
        const T dm0 = (cgxf * g0x + cgyf * g0y + cgzf * g0z) * icgf;
        const T dm1 = (cgxf * g1x + cgyf * g1y + cgzf * g1z) * icgf;
        const T icg2 = icgf * icgf;
        fa[0] = g0x * icgf - cgxf * icg2 * dm0;
        fa[1] = g0y * icgf - cgyf * icg2 * dm0;
        fa[2] = g0z * icgf - cgzf * icg2 * dm0;
        fa[4] = g1x * icgf - cgxf * icg2 * dm1;
        fa[5] = g1y * icgf - cgyf * icg2 * dm1;
        fa[6] = g1z * icgf - cgzf * icg2 * dm1;
        fa[3] = dm0 * icg2 * Kzf - icgf * (dnu0 * czf + numf * (Xtz * czz) + rc.mtx * uzf + rc.mty * vzf +
                                           rc.nxf * (Xtz * uzz) + rc.nyf * (Xtz * vzz));
        fa[7] = dm1 * icg2 * Kzf - icgf * (dnu1 * czf + numf * (Xpz * czz) + rc.mpx * uzf + rc.mpy * vzf +
                                           rc.nxf * (Xpz * uzz) + rc.nyf * (Xpz * vzz));
    }
}

// One RK4 step (rk4solver.cpp:30-55) of size ds from (yd, ya): the increments
// incd (FP64) and inca (T), and the stage-1 direction f1 = c_g/|c_g| for the
// caustic test.
template <bool AMP, class T>
__device__ __forceinline__ void rk4_c(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                      double ds, const double* yd, const T* ya, const RayConstC<T>& rc,
                                      double* incd, T* inca, double* f1) {
    constexpr int NA = AuxN<AMP>::n;
    const T dsf = (T)ds;
    const T sixth = T(1) / T(6), third = T(1) / T(3), half = T(0.5);
    double stgd[4], fd[4];
    T stga[NA], fa[NA];
    rhs_c<AMP>(tab, a, seg, yd, ya, rc, fd, fa);
#pragma unroll
    for (int i = 0; i < 3; i++) f1[i] = fd[i];
#pragma unroll
    for (int i = 0; i < 4; i++) { const double t = ds * fd[i]; incd[i] = t * (1.0 / 6.0); stgd[i] = yd[i] + t * 0.5; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] = t * sixth; stga[i] = ya[i] + t * half; }
    }
    rhs_c<AMP>(tab, a, seg, stgd, stga, rc, fd, fa);
#pragma unroll
    for (int i = 0; i < 4; i++) { const double t = ds * fd[i]; incd[i] += t * (1.0 / 3.0); stgd[i] = yd[i] + t * 0.5; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] += t * third; stga[i] = ya[i] + t * half; }
    }
    rhs_c<AMP>(tab, a, seg, stgd, stga, rc, fd, fa);
#pragma unroll
    for (int i = 0; i < 4; i++) { const double t = ds * fd[i]; incd[i] += t * (1.0 / 3.0); stgd[i] = yd[i] + t; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] += t * third; stga[i] = ya[i] + t; }
    }
    rhs_c<AMP>(tab, a, seg, stgd, stga, rc, fd, fa);
#pragma unroll
    for (int i = 0; i < 4; i++) incd[i] += (ds * fd[i]) * (1.0 / 6.0);
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) inca[i] += (dsf * fa[i]) * sixth;
    }
}

// set_ds (geoac.eqset.3d.strat.cpp:214-220), as the FP64 kernel forms it, so
// both precisions step through the same rows near the ground.
__device__ __forceinline__ double step_c(const Fan3DArgs& a, double z) {
    double ds = a.ds_max;
    if (z < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(z - a.z0) / 0.2);
    return ds;
}

// Travel-time and absorption increments of the step yd -> yd + incd at its
// midpoint (travel_time :486-511, c, u, v in FP64; atten :688-699 with
// alpha(z) from the FP64-built table, tweak_abs applied here).
template <class T>
__device__ __forceinline__ void seg_increment_c(const double* __restrict__ tab, const Fan3DArgs& a, int& seg,
                                                const double* yd, const double* incd, const RayConstC<T>& rc,
                                                double& dt, double& da) {
    const double seg_ds = sqrt(incd[0] * incd[0] + incd[1] * incd[1] + incd[2] * incd[2]);
    const double zm = yd[2] + 0.5 * incd[2];
    const double nzm = yd[3] + 0.5 * incd[3];
    const double ze = fmin(fmax(zm, a.z_lo), a.z_hi);
    seg = seg_walk_c(tab, a.n_knots, ze, seg);
    const double* r0 = tab + seg * kStrideC;
    const double X = (ze - r0[0]) * r0[1];
    const double c = fma(X, fma(X, fma(X, r0[5], r0[4]), r0[3]), r0[2]);
    const double sc = bl_scale_c<false>(zm - a.z0, a.inv_bl).s0;
    const double u = fma(X, fma(X, fma(X, r0[9], r0[8]), r0[7]), r0[6]) * sc;
    const double v = fma(X, fma(X, fma(X, r0[13], r0[12]), r0[11]), r0[10]) * sc;
    const double cin = c * rsqrt_c(rc.nh2 + nzm * nzm);
    const double cgx = cin * rc.nx + u, cgy = cin * rc.ny + v, cgz = cin * nzm;
    dt = seg_ds * rsqrt_c(cgx * cgx + cgy * cgy + cgz * cgz);
    const float ua = (float)(zm - a.alpha_z0) * (float)a.alpha_inv_h;
    int ia = (int)ua;
    ia = ia < 0 ? 0 : (ia > a.alpha_n - 2 ? a.alpha_n - 2 : ia);
    const float w = fminf(fmaxf(ua - (float)ia, 0.0f), 1.0f);
    const float al0 = __ldg(a.alpha_tab + ia), al1 = __ldg(a.alpha_tab + ia + 1);
    da = (double)((al0 + w * (al1 - al0)) * (float)a.tweak_abs) * seg_ds;
}

// geoac::set_initial (geoac.eqset.3d.strat.cpp:58-105) from (x0, y0, src_z)
// into the split state.
template <bool AMP, class T>
__device__ __forceinline__ void init_c(const Fan3DArgs& a, double theta, double phi, double x0, double y0, double* yd,
                                       T* ya, T* yl, RayConstC<T>& rc) {
    double y[12];
    RayConst r;
    ray_init<AMP>(a, theta, phi, y, r);
    y[0] = x0; y[1] = y0;
#pragma unroll
    for (int i = 0; i < 4; i++) yd[i] = y[i];
    if (AMP) {
#pragma unroll
        for (int i = 0; i < 8; i++) { ya[i] = (T)y[4 + i]; yl[i] = (T)(y[4 + i] - (double)ya[i]); }
    }
    rc.nx = r.nx; rc.ny = r.ny; rc.nh2 = r.nx * r.nx + r.ny * r.ny;
    rc.nxf = (T)r.nx; rc.nyf = (T)r.ny;
    rc.mtx = (T)r.mtx; rc.mty = (T)r.mty; rc.mpx = (T)r.mpx; rc.mpy = (T)r.mpy;
}

// Rows k-1 (r1) and the step k-2 -> k-1 (d1) in FP64, 12-state layout.  The
// auxiliaries' step is kept in FP32 for both types: it enters only the
// intercept extrapolation, scaled by dz_grnd / dz_k <= 1, where its rounding
// is ~1e-10 of the state.
template <bool AMP, class T>
__device__ __forceinline__ void last_rows_c(const double* yd, const T* ya, const T* yl, const double* dprev,
                                            const float* dprevf, double* r1, double* d1) {
#pragma unroll
    for (int i = 0; i < 4; i++) { r1[i] = yd[i]; d1[i] = dprev[i * blockDim.x]; }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        r1[4 + i] = AMP ? (double)ya[i] + (double)yl[i] : 0.0;
        d1[4 + i] = AMP ? (double)dprevf[i * blockDim.x] : 0.0;
    }
}

// approx_intercept + flat-ground set_refl (geoac.eqset.3d.strat.cpp:110-209)
// in FP64 from rows k-1 and k-2, into the split state.
template <bool AMP, class T>
__device__ __forceinline__ void reflect_c(const Fan3DArgs& a, const double* r1, const double* d1, const RayConstC<T>& rc,
                                          double* yd, T* ya, T* yl) {
    const double dz_grnd = a.z0 - r1[2];
    const double dz_k = d1[2];
    double p[12];
#pragma unroll
    for (int i = 0; i < 12; i++) p[i] = r1[i] + d1[i] / dz_k * dz_grnd;
    yd[0] = p[0]; yd[1] = p[1]; yd[2] = a.z0; yd[3] = -p[3];
    if (AMP) {
        const double ds0_dth = -a.c0 / a.c_gnd * p[6] / p[3];
        const double ds0_dph = -a.c0 / a.c_gnd * p[10] / p[3];
        const double dnuz_ds = -1.0 / a.c_gnd * (a.c0 / a.c_gnd * a.dcz_g + rc.nx * a.duz_g + rc.ny * a.dvz_g);
        const double q[8] = {p[4], p[5], -p[6], -p[7] + (-2.0 * dnuz_ds) * ds0_dth,
                             p[8], p[9], -p[10], -p[11] + (-2.0 * dnuz_ds) * ds0_dph};
#pragma unroll
        for (int i = 0; i < 8; i++) { ya[i] = (T)q[i]; yl[i] = (T)(q[i] - (double)ya[i]); }
    }
}

// Shared memory of a launch: the FP64 table (SMEM; otherwise it is read from
// global memory through the read-only cache), then per lane the previous
// step's increments ([4][blockDim.x] FP64, [8][blockDim.x] FP32).
constexpr size_t kSmemTableMax = 160 * 1024;   // larger tables (profiles over ~1,800 knots) stay in global memory

inline bool table_in_smem(const Fan3DArgs& a) { return (size_t)a.n_knots * kStrideC * sizeof(double) <= kSmemTableMax; }

inline size_t smem_c(const Fan3DArgs& a, int threads, bool smem_table) {
    return (smem_table ? (size_t)a.n_knots * kStrideC * sizeof(double) : 0) +
           (size_t)threads * (4 * sizeof(double) + 8 * sizeof(float));
}

template <bool SMEM>
__device__ __forceinline__ const double* stage_table_c(const Fan3DArgs& a, double* s_mem) {
    if (!SMEM) return a.knots_c;
    const int tot = a.n_knots * kStrideC;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) s_mem[i] = a.knots_c[i];
    __syncthreads();
    return s_mem;
}

// One ray of the fan, launch to last bounce, with the auxiliaries in T.
// Returns true, with nothing of the ray's record final, when T is FP32 and the
// ray reaches a focusing arrival (kFocusRatio) before its first caustic: the
// caller then traces it again with T = double.
template <bool AMP, class T>
__device__ __forceinline__ bool fan_ray_c(const Fan3DArgs& a, const double* __restrict__ tab, double* dprev,
                                          float* dprevf, int ray) {
    constexpr int NA = AuxN<AMP>::n;
    constexpr bool ESCALATE = AMP && sizeof(T) == sizeof(float);
    const int nb = a.bounces + 1;
    const double theta0 = a.theta_deg[ray] * kPi / 180.0;
    const double phi0 = kPi / 2.0 - a.phi_deg[ray] * kPi / 180.0;

    double yd[4];
    T ya[NA], yl[NA];
    RayConstC<T> rc;
    init_c<AMP>(a, theta0, phi0, a.src_x, a.src_y, yd, ya, yl, rc);
    int seg = seg_guess(fmin(fmax(a.src_z, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
    int bnc = 0, kb = 0, na = 0, caustics = 0;
    bool focused = false;
    T D_prev = T(0), D_max = T(0);
    long long steps = 0;
    // tt/att: the ray's time and absorption sums; pt/pa: the bounce's partial
    // sums (bulk mode) or the pending last-segment increments (write_rays mode)
    double s = 0.0, tt = 0.0, att = 0.0, pt = 0.0, pa = 0.0, zmax = a.z0;
#pragma unroll
    for (int i = 0; i < 4; i++) dprev[i * blockDim.x] = 0.0;
    if (AMP) {
#pragma unroll
        for (int i = 0; i < 8; i++) dprevf[i * blockDim.x] = 0.0f;
    }

    while (true) {
        zmax = fmax(zmax, yd[2]);
        const double ds = step_c(a, yd[2]);
        s += ds;
        double incd[4], f1[3];
        T inca[NA];
        rk4_c<AMP>(tab, a, seg, ds, yd, ya, rc, incd, inca, f1);
        if (AMP && (a.aux || ESCALATE) && kb >= 1) {
            // caustics: sign changes of D between rows 1..k-1 of the bounce
            const T f0 = (T)f1[0], g1 = (T)f1[1], g2 = (T)f1[2];
            const T D = f0 * (ya[1] * ya[6] - ya[5] * ya[2]) - ya[0] * (g1 * ya[6] - g2 * ya[5]) +
                        ya[4] * (g1 * ya[2] - g2 * ya[1]);
            if (kb >= 2 && D * D_prev < T(0)) caustics++;
            D_prev = D;
            if (ESCALATE) D_max = fmax(D_max, fabs(D));
        }
        kb++;
        {
            double dt, da;
            seg_increment_c(tab, a, seg, yd, incd, rc, dt, da);
            if (a.write_rays) { tt += pt; att += pa; pt = dt; pa = da; }   // main.infraga.3d.cpp:451-453
            else { pt += dt; pa += da; }                                    // :486-487
        }
        double nd[4];
#pragma unroll
        for (int i = 0; i < 4; i++) nd[i] = yd[i] + incd[i];
        // stop checks (rk4solver.cpp:57-75, break/ground_check :438-453)
        const double rx = nd[0] - a.src_x, ry = nd[1] - a.src_y;
        bool esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) || (nd[0] > a.x_max) || (nd[0] < a.x_min) ||
                   (nd[1] > a.y_max) || (nd[1] < a.y_min) || (nd[2] > a.alt_max);
        const bool gnd = !esc && (nd[2] < a.z0);
        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(nd[2]) || !isfinite(nd[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < 4; i++) { dprev[i * blockDim.x] = incd[i]; yd[i] = nd[i]; }
            if (AMP) {
#pragma unroll
                for (int i = 0; i < 8; i++) { dprevf[i * blockDim.x] = (float)inca[i]; acc_pair(ya[i], yl[i], inca[i]); }
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.3d.cpp:436-538) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        int status = -1;
        if (zmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        if (status < 0) {
            // arrival record from the first below-ground row K (rk)
            double r1[12], d1[12], rk[12];
            last_rows_c<AMP>(yd, ya, yl, dprev, dprevf, r1, d1);
#pragma unroll
            for (int i = 0; i < 12; i++) rk[i] = r1[i] + (i < 4 ? incd[i] : (AMP ? (double)inca[i - 4] : 0.0));
            const RayConst rcd{rc.nx, rc.ny, (double)rc.mtx, (double)rc.mty, (double)rc.mpx, (double)rc.mpy};
            double jac = 0.0, amp = 0.0;
            if (AMP) {
                int segd = seg_guess(fmin(fmax(rk[2], a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
                const double theta = a.theta_deg[ray] * kPi / 180.0;
                const double phi = kPi / 2.0 - a.phi_deg[ray] * kPi / 180.0;
                amp = amp_db(a.knots, a, segd, rk, rcd, theta, phi, &jac);
                if (ESCALATE && !focused && caustics == 0 && fabs(jac) < kFocusRatio * (double)D_max) {
                    if (a.retrace) return true;
                    focused = true;
                }
            }
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double incl = -asin(a.c_ratio * rk[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-rc.ny, -rc.nx) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            const double ex = rk[0] - a.src_x, ey = rk[1] - a.src_y;
            out[0] = a.theta_deg[ray];
            out[1] = a.phi_deg[ray];
            out[2] = (double)bnc;
            out[3] = rk[0];
            out[4] = rk[1];
            out[5] = tt;
            out[6] = sqrt(ex * ex + ey * ey) / tt;
            out[7] = zmax;
            out[8] = incl;
            out[9] = baz;
            out[10] = amp;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux(ax, a, rk, rcd, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            reflect_c<AMP>(a, r1, d1, rc, yd, ya, yl);
            bnc++;
            if (bnc > a.bounces) status = 0;
        }
        if (status < 0) {
            s = 0.0; kb = 0;
            continue;
        }
        // ray finished: its record
        a.n_arr[ray] = na;
        a.ray_steps[ray] = steps;
        if (a.ray_status)
            a.ray_status[ray] = status | (sizeof(T) == sizeof(double) ? kRayAuxFp64 : 0) | (focused ? kRayFocus : 0);
        return false;
    }
}

// Persistent fan kernel: each thread takes the next ray from the queue when
// its ray ends, so lanes do not idle until the warp's longest ray.  A ray
// that needs FP64 auxiliaries is marked (n_arr = -1) and left to
// fan3d_fp32c_retrace_kernel: tracing it here would hold the other 31 lanes
// of its warp for the length of a ray.
template <bool AMP, bool SMEM>
__global__ void __launch_bounds__(kThreadsC, IGA_FANC_MINB) fan3d_fp32c_kernel(const __grid_constant__ Fan3DArgs a) {
    extern __shared__ double s_memc[];
    const double* tab = stage_table_c<SMEM>(a, s_memc);
    double* s_lane = s_memc + (SMEM ? (size_t)a.n_knots * kStrideC : 0);
    double* dprev = s_lane + threadIdx.x;
    float* dprevf = reinterpret_cast<float*>(s_lane + 4 * blockDim.x) + threadIdx.x;
    for (int ray = (int)atomicAdd(a.queue, 1u); ray < a.n_rays; ray = (int)atomicAdd(a.queue, 1u))
        if (fan_ray_c<AMP, float>(a, tab, dprev, dprevf, ray)) a.n_arr[ray] = -1;
}

// The marked rays of a fan, traced from launch with FP64 auxiliaries (about
// 1% of a 10-bounce fan): one CTA per SM scans the fan's rays through a
// second queue counter, so the few marked rays spread over the SMs.
constexpr int kThreadsR = 128;

template <bool SMEM>
__global__ void __launch_bounds__(kThreadsR, 1)
    fan3d_fp32c_retrace_kernel(const __grid_constant__ Fan3DArgs a, unsigned int* __restrict__ queue) {
    extern __shared__ double s_memc[];
    const double* tab = stage_table_c<SMEM>(a, s_memc);
    double* s_lane = s_memc + (SMEM ? (size_t)a.n_knots * kStrideC : 0);
    double* dprev = s_lane + threadIdx.x;
    float* dprevf = reinterpret_cast<float*>(s_lane + 4 * blockDim.x) + threadIdx.x;
    for (int ray = (int)atomicAdd(queue, 1u); ray < a.n_rays; ray = (int)atomicAdd(queue, 1u))
        if (a.n_arr[ray] < 0) fan_ray_c<true, double>(a, tab, dprev, dprevf, ray);
}

// Eigenray-search traces in FP32-compensated form: one request per thread,
// n_seg prop_rk4 segments with flat-ground reflections (same contract as
// trace3d_fp64_kernel in eig3d.cu, including the record mode's per-step
// time/absorption sums and turning height from 0 over rows 1..k-1,
// geoac.eigenray.3d.cpp:229-262).  The search's bracket and Newton updates
// stay in FP64 on the host.  Sweep traces carry no auxiliaries; Newton and
// record traces carry them in FP64, so the search takes the FP64 search's
// iterates (the Newton step reads the launch-angle derivatives of the
// landing point, which an FP32 error moves near a fold of the fan) and the
// eigenray's amplitude keeps FP64 conditioning.
template <bool AMP, class T>
__device__ __forceinline__ void trace_req_c(const Fan3DArgs& a, const double* __restrict__ tab, double* dprev,
                                            float* dprevf, const TraceReq& q, TraceRes* o_ptr, SegRes* seg_out,
                                            int seg_stride, int r) {
    constexpr int NA = AuxN<AMP>::n;
    const bool record = (q.flags & kRecord) != 0, stop = (q.flags & kStopOnEscape) != 0;
    double yd[4], incd[4] = {0.0, 0.0, 0.0, 0.0};
    T ya[NA], yl[NA], inca[NA];
    RayConstC<T> rc;
    init_c<AMP>(a, q.theta, q.phi, q.x0, q.y0, yd, ya, yl, rc);
#pragma unroll
    for (int i = 0; i < NA; i++) inca[i] = T(0);
    int seg = seg_guess(fmin(fmax(a.src_z, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
    double tt = 0.0, att = 0.0, zmax = 0.0;
    long long steps = 0;
    bool esc = false;
    for (int sg = 0; sg < q.n_seg; sg++) {
        double s = 0.0, pt = 0.0, pa = 0.0;
        int kb = 0;
        bool capped = false;
#pragma unroll
        for (int i = 0; i < 4; i++) dprev[i * blockDim.x] = 0.0;
        if (AMP) {
#pragma unroll
            for (int i = 0; i < 8; i++) dprevf[i * blockDim.x] = 0.0f;
        }
        while (true) {
            if (record && kb >= 1) zmax = fmax(zmax, yd[2]);
            const double ds = step_c(a, yd[2]);
            s += ds;
            double f1[3];
            rk4_c<AMP>(tab, a, seg, ds, yd, ya, rc, incd, inca, f1);
            kb++;
            if (record) {
                double dt, da;
                seg_increment_c(tab, a, seg, yd, incd, rc, dt, da);
                tt += pt; att += pa; pt = dt; pa = da;
            }
            double nd[4];
#pragma unroll
            for (int i = 0; i < 4; i++) nd[i] = yd[i] + incd[i];
            const double rx = nd[0] - q.x0, ry = nd[1] - q.y0;
            esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) || (nd[0] > a.x_max) ||
                  (nd[0] < a.x_min) || (nd[1] > a.y_max) || (nd[1] < a.y_min) || (nd[2] > a.alt_max);
            const bool gnd = !esc && (nd[2] < a.z0);
            if (!esc && !gnd) {
                if (kb >= a.length - 1) { capped = true; esc = true; }
                else if (!isfinite(nd[2]) || !isfinite(nd[3])) esc = true;
            }
            if (!esc && !gnd) {
#pragma unroll
                for (int i = 0; i < 4; i++) { dprev[i * blockDim.x] = incd[i]; yd[i] = nd[i]; }
                if (AMP) {
#pragma unroll
                    for (int i = 0; i < 8; i++) { dprevf[i * blockDim.x] = (float)inca[i]; acc_pair(ya[i], yl[i], inca[i]); }
                }
                continue;
            }
            break;
        }
        steps += capped ? a.length : kb;
        if (seg_out) {
            SegRes& g = seg_out[(size_t)r * seg_stride + sg];
            g.x = yd[0] + incd[0];
            g.y = yd[1] + incd[1];
            g.steps = steps;
            g.escaped = esc ? 1 : 0;
        }
        if (sg == q.n_seg - 1 || (esc && stop)) break;
        double r1[12], d1[12];
        last_rows_c<AMP>(yd, ya, yl, dprev, dprevf, r1, d1);
        reflect_c<AMP>(a, r1, d1, rc, yd, ya, yl);
#pragma unroll
        for (int i = 0; i < 4; i++) incd[i] = 0.0;
#pragma unroll
        for (int i = 0; i < NA; i++) inca[i] = T(0);
    }
    double rk[12];
#pragma unroll
    for (int i = 0; i < 4; i++) rk[i] = yd[i] + incd[i];
#pragma unroll
    for (int i = 0; i < 8; i++) rk[4 + i] = AMP ? (double)ya[i] + (double)yl[i] + (double)inca[i] : 0.0;
    TraceRes& o = *o_ptr;
#pragma unroll
    for (int i = 0; i < 12; i++) o.y[i] = rk[i];
    o.rc[0] = rc.nx; o.rc[1] = rc.ny; o.rc[2] = rc.mtx; o.rc[3] = rc.mty; o.rc[4] = rc.mpx; o.rc[5] = rc.mpy;
    o.steps = steps;
    o.escaped = esc ? 1 : 0;
    if (record) {
        o.tt = tt; o.att = att; o.zmax = zmax;
        const RayConst rcd{rc.nx, rc.ny, (double)rc.mtx, (double)rc.mty, (double)rc.mpx, (double)rc.mpy};
        int segd = seg_guess(fmin(fmax(rk[2], a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        o.amp_db = AMP ? amp_db(a.knots, a, segd, rk, rcd, q.theta, q.phi, nullptr) : 0.0;
        const double ze = fmin(fmax(rk[2], a.z_lo), a.z_hi);
        segd = seg_walk(a.knots, a.n_knots, ze, segd);
        const double* r0 = a.knots + segd * kStride;
        const double c_k = cubic_f(r0, cubic_at(r0, ze), 2);
        o.incl = -asin(c_k / a.c0 * rk[3]) * (180.0 / kPi);
        double baz = 90.0 - atan2(-rcd.ny, -rcd.nx) * (180.0 / kPi);
        while (baz > 180.0) baz -= 360.0;
        while (baz < -180.0) baz += 360.0;
        o.baz = baz;
    }
}

template <bool AMP, bool SMEM>
__global__ void __launch_bounds__(kThreadsC, AMP ? 1 : IGA_FANC_MINB)
    trace3d_fp32c_kernel(const __grid_constant__ Fan3DArgs a, const TraceReq* __restrict__ reqs,
                         TraceRes* __restrict__ out, int n, unsigned int* __restrict__ queue,
                         SegRes* __restrict__ seg_out, int seg_stride) {
    extern __shared__ double s_memc[];
    const double* tab = stage_table_c<SMEM>(a, s_memc);
    double* s_lane = s_memc + (SMEM ? (size_t)a.n_knots * kStrideC : 0);
    double* dprev = s_lane + threadIdx.x;
    float* dprevf = reinterpret_cast<float*>(s_lane + 4 * blockDim.x) + threadIdx.x;
    // persistent: each thread takes the next request when its trace ends, so
    // lanes whose trace finished early do not idle until the warp's longest one
    using T = typename std::conditional<AMP, double, float>::type;
    for (int r = (int)atomicAdd(queue, 1u); r < n; r = (int)atomicAdd(queue, 1u))
        trace_req_c<AMP, T>(a, tab, dprev, dprevf, reqs[r], out + r, seg_out, seg_stride, r);
}

template <bool AMP, bool SMEM>
cudaError_t launch_trace_c(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, cudaStream_t st,
                           SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = trace3d_fp32c_kernel<AMP, SMEM>;
    const size_t smem = smem_c(a, kThreadsC, SMEM);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kThreadsC, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kThreadsC, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride);
    return cudaGetLastError();
}

template <bool AMP, bool SMEM>
cudaError_t launch_c(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    // threads per block: the caller's choice (a multiple of 32 up to kThreadsC) or kThreadsC
    const int threads = a.block > 0 ? a.block : kThreadsC;
    auto kern = fan3d_fp32c_kernel<AMP, SMEM>;
    const size_t smem = smem_c(a, threads, SMEM);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, n_sm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    long long want = ((long long)a.n_rays + threads - 1) / threads;
    long long grid = (long long)n_sm * per_sm;
    if (want < grid) grid = want;
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    if (grid < 1) grid = 1;
    if (grid_used) *grid_used = (int)grid;
    kern<<<(unsigned)grid, threads, smem, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess || !AMP || !a.retrace) return e;
    // the rays marked for FP64 auxiliaries, after the fan on the same stream;
    // its queue is the workspace's second counter (cleared with the first)
    auto rk = fan3d_fp32c_retrace_kernel<SMEM>;
    const size_t smem_r = smem_c(a, kThreadsR, SMEM);
    if ((e = cudaFuncSetAttribute(rk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r)) != cudaSuccess)
        return e;
    const long long grid_r = std::min<long long>(n_sm, ((long long)a.n_rays + kThreadsR - 1) / kThreadsR);
    rk<<<(unsigned)grid_r, kThreadsR, smem_r, stream>>>(a, a.queue + 1);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fan3d_fp32c(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    if (table_in_smem(a))
        return calc_amp ? launch_c<true, true>(a, stream, grid_used) : launch_c<false, true>(a, stream, grid_used);
    return calc_amp ? launch_c<true, false>(a, stream, grid_used) : launch_c<false, false>(a, stream, grid_used);
}

cudaError_t launch_trace_fp32c(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, bool amp,
                               cudaStream_t st, unsigned int* d_queue, SegRes* seg_out, int seg_stride) {
    if (table_in_smem(a))
        return amp ? launch_trace_c<true, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
                   : launch_trace_c<false, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
    return amp ? launch_trace_c<true, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
               : launch_trace_c<false, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
}

}  // namespace iga
