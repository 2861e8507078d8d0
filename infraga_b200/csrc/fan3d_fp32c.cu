// FP32-compensated ray-fan kernel: 3D Cartesian, stratified, flat ground.
//
// Same ray/Jacobian equations, RK4 driver, stop checks and bounce logic as
// the FP64 kernel (fan3d_fp64.cu, following geoac.eqset.3d.strat.cpp and
// rk4solver.cpp), with the arithmetic split by what each quantity needs:
//   * RK4 stages and spline evaluation in FP32 (SFU exp/rsqrt);
//   * x, y, z and nu_z carried as hi/lo float pairs updated with TwoSum, so
//     2000 km of 1 m..50 m steps accumulate without FP32 drift;
//   * segment vectors taken from the RK4 increments themselves (not from
//     differences of large coordinates), path length, travel time and
//     absorption summed in FP64;
//   * Sutherland-Bass absorption from an FP64-built table of alpha(z) (a
//     stratified profile makes alpha a function of altitude only);
//   * ground intercept, reflection and amplitude in FP64 (rare events).
#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fan3d_common.cuh"

namespace iga {

namespace {

#ifndef IGA_FANC_THREADS
#define IGA_FANC_THREADS 128
#endif
#ifndef IGA_FANC_MINB
#define IGA_FANC_MINB 4
#endif
constexpr int kThreadsC = IGA_FANC_THREADS;
// Above this height X = exp(-(z-zg)/0.1) < 2e-22 and drops out of every FP32 term.
constexpr float kBlCutoffKmF = 5.0f;

template <bool AMP> struct DimF { static constexpr int n = AMP ? 12 : 4; };

struct RayConstF {
    float nx, ny, mtx, mty, mpx, mpy;
};

__device__ __forceinline__ int seg_walk_f(const float* __restrict__ tab, int n, float z, int k) {
    while (k > 0 && z < tab[k * kStrideF]) --k;
    while (k < n - 2 && z > tab[(k + 1) * kStrideF]) ++k;
    return k;
}

struct CubicF {
    float X, idx;
};

__device__ __forceinline__ CubicF cubic_at_f(const float* __restrict__ r0, float z) {
    CubicF q;
    q.idx = r0[1];
    q.X = (z - r0[0]) * q.idx;
    return q;
}

// Power-basis cubic of one field on the segment: col = 2 (c), 6 (u), 10 (v).
__device__ __forceinline__ float cubicf_f(const float* __restrict__ r0, const CubicF& q, int col) {
    const float a0 = r0[col], a1 = r0[col + 1], a2 = r0[col + 2], a3 = r0[col + 3];
    return a0 + q.X * (a1 + q.X * (a2 + q.X * a3));
}

template <bool D2>
__device__ __forceinline__ void cubicf_d(const float* __restrict__ r0, const CubicF& q, int col, float& f, float& d1, float& d2) {
    const float a0 = r0[col], a1 = r0[col + 1], a2 = r0[col + 2], a3 = r0[col + 3];
    const float X = q.X;
    f = a0 + X * (a1 + X * (a2 + X * a3));
    d1 = (a1 + X * (2.0f * a2 + 3.0f * a3 * X)) * q.idx;
    if (D2) d2 = (2.0f * a2 + 6.0f * a3 * X) * (q.idx * q.idx);
}

// Knuth's TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// RHS of the 12 (or 4) varying equations in FP32; see rhs() in fan3d_fp64.cu
// for the derivation from update_refs / eval_src_eq.
template <bool AMP>
__device__ __forceinline__ void rhs_f(const float* __restrict__ tab, const Fan3DArgs& a, float z0f, float inv_blf,
                                      float zlo, float zhi, int& seg, const float* y, const RayConstF& rc, float* f) {
    const float z = y[2];
    const float ze = fminf(fmaxf(z, zlo), zhi);
    seg = seg_walk_f(tab, a.n_knots, ze, seg);
    const float* r0 = tab + seg * kStrideF;
    const CubicF q = cubic_at_f(r0, ze);
    float c, cz, czz = 0.f, u0, u0z, u0zz = 0.f, v0, v0z, v0zz = 0.f;
    cubicf_d<AMP>(r0, q, 2, c, cz, czz);
    cubicf_d<AMP>(r0, q, 6, u0, u0z, u0zz);
    cubicf_d<AMP>(r0, q, 10, v0, v0z, v0zz);
    const float hz = z - z0f;
    float sc0 = 1.0f, dsc2 = 0.0f, ddsc22 = 0.0f;
    if (hz < kBlCutoffKmF) {
        const float Xb = __expf(-hz * inv_blf);
        const float iop = __fdividef(1.0f, 1.0f + Xb);
        sc0 = (1.0f - Xb) * iop;
        const float dX2 = -Xb * inv_blf;
        dsc2 = -2.0f * dX2 * (iop * iop);
        if (AMP) ddsc22 = -2.0f * (Xb * inv_blf * inv_blf * (iop * iop) - 2.0f * dX2 * dX2 * (iop * iop * iop));
    }
    const float u = u0 * sc0, v = v0 * sc0;
    const float uz = u0z * sc0 + u0 * dsc2;
    const float vz = v0z * sc0 + v0 * dsc2;
    const float nz = y[3];
    const float num2 = rc.nx * rc.nx + rc.ny * rc.ny + nz * nz;
    const float inum = rsqrtf(num2);
    const float num = num2 * inum;
    const float cgx = c * rc.nx * inum + u;
    const float cgy = c * rc.ny * inum + v;
    const float cgz = c * nz * inum;
    const float icg = rsqrtf(cgx * cgx + cgy * cgy + cgz * cgz);
    f[0] = cgx * icg;
    f[1] = cgy * icg;
    f[2] = cgz * icg;
    const float Kz = num * cz + rc.nx * uz + rc.ny * vz;
    f[3] = -icg * Kz;
    if (AMP) {
        const float uzz = u0zz * sc0 + 2.0f * u0z * dsc2 + u0 * ddsc22;
        const float vzz = v0zz * sc0 + 2.0f * v0z * dsc2 + v0 * ddsc22;
        const float Xtz = y[6], Xpz = y[10], mtz = y[7], mpz = y[11];
        const float dc3 = Xtz * cz, dc4 = Xpz * cz;
        const float du3 = Xtz * uz, du4 = Xpz * uz;
        const float dv3 = Xtz * vz + Xpz * vz;   // reference's dv[3]/dv[4] accumulation (eqset.3d.strat.cpp:298)
        const float dnu0 = (rc.nx * rc.mtx + rc.ny * rc.mty + nz * mtz) * inum;
        const float dnu1 = (rc.nx * rc.mpx + rc.ny * rc.mpy + nz * mpz) * inum;
        const float cin = c * inum, cin2 = cin * inum;
        const float g0x = rc.nx * inum * dc3 + cin * rc.mtx - cin2 * rc.nx * dnu0 + du3;
        const float g0y = rc.ny * inum * dc3 + cin * rc.mty - cin2 * rc.ny * dnu0 + dv3;
        const float g0z = nz * inum * dc3 + cin * mtz - cin2 * nz * dnu0;
        const float g1x = rc.nx * inum * dc4 + cin * rc.mpx - cin2 * rc.nx * dnu1 + du4;
        const float g1y = rc.ny * inum * dc4 + cin * rc.mpy - cin2 * rc.ny * dnu1;
        const float g1z = nz * inum * dc4 + cin * mpz - cin2 * nz * dnu1;
        const float dm0 = (cgx * g0x + cgy * g0y + cgz * g0z) * icg;
        const float dm1 = (cgx * g1x + cgy * g1y + cgz * g1z) * icg;
        const float icg2 = icg * icg;
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

template <bool AMP>
__global__ void __launch_bounds__(kThreadsC, IGA_FANC_MINB) fan3d_fp32c_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = DimF<AMP>::n;
    extern __shared__ float s_memf[];
    float* s_dprev = s_memf;                       // [N][blockDim.x] previous step's increments
    float* s_tab = s_memf + N * blockDim.x;         // FP32 knot table
    {
        const int tot = a.n_knots * kStrideF;
        for (int i = threadIdx.x; i < tot; i += blockDim.x) s_tab[i] = a.knots_f[i];
        __syncthreads();
    }
    const float* tab = s_tab;
    float* dprev = s_dprev + threadIdx.x;

    const int nb = a.bounces + 1;
    const float z0f = (float)a.z0, inv_blf = (float)a.inv_bl;
    const float zlo = (float)a.z_lo, zhi = (float)a.z_hi;
    const float zbl = (float)a.z_bl;
    const float ds_max = (float)a.ds_max, ds_span = (float)(a.ds_max - a.ds_min);
    const float tweak = (float)a.tweak_abs;

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    float y[N];         // hi parts for 0..3; plain FP32 for the auxiliaries
    float lo[4];        // lo parts of x, y, z, nu_z
    RayConstF rc;
    int seg, bnc, kb, na, caustics;
    float D_prev = 0.0f;
    long long steps;
    double s, tt, att, pt, pa;
    float zmax;

    auto set_pair = [](double v, float& h, float& l) { h = (float)v; l = (float)(v - (double)h); };

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * kPi / 180.0;
        const double phi = kPi / 2.0 - a.phi_deg[r] * kPi / 180.0;
        // geoac::set_initial in FP64, then split
        const double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
        const double mx = a.u0s / a.c0, my = a.v0s / a.c0;
        const double n0x = ct * cp, n0y = ct * sp, n0z = st;
        const double ms = 1.0 + (n0x * mx + n0y * my);
        const double ims = 1.0 / ms, ims2 = ims * ims;
        set_pair(a.src_x, y[0], lo[0]);
        set_pair(a.src_y, y[1], lo[1]);
        set_pair(a.src_z, y[2], lo[2]);
        set_pair(n0z * ims, y[3], lo[3]);
        rc.nx = (float)(n0x * ims);
        rc.ny = (float)(n0y * ims);
        if (AMP) {
            const double tx = -st * cp, ty = -st * sp, tz = ct;
            const double px = -ct * sp, py = ct * cp;
            const double tm = tx * mx + ty * my, pm = px * mx + py * my;
            rc.mtx = (float)(tx * ims - n0x * ims2 * tm);
            rc.mty = (float)(ty * ims - n0y * ims2 * tm);
            y[7] = (float)(tz * ims - n0z * ims2 * tm);
            rc.mpx = (float)(px * ims - n0x * ims2 * pm);
            rc.mpy = (float)(py * ims - n0y * ims2 * pm);
            y[11] = (float)(-n0z * ims2 * pm);
            y[4] = y[5] = y[6] = 0.0f;
            y[8] = y[9] = y[10] = 0.0f;
        } else {
            rc.mtx = rc.mty = rc.mpx = rc.mpy = 0.0f;
        }
        seg = seg_guess(fmin(fmax(a.src_z, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        zmax = z0f;
#pragma unroll
        for (int i = 0; i < N; i++) dprev[i * blockDim.x] = 0.0f;
    };
    start_ray(ray);

    while (true) {
        const float zc = y[2] + lo[2];
        zmax = fmaxf(zmax, zc);
        float ds = ds_max;   // set_ds (geoac.eqset.3d.strat.cpp:214-220)
        if (zc < zbl) ds -= ds_span * __expf(-(zc - z0f) * 5.0f);
        s += (double)ds;
        float inc[N], stg[N], f[N];
        rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, y, rc, f);
        if (AMP && a.aux && kb >= 1) {   // caustics between rows 1..k-1 of the bounce
            const float D = ray_jacobian(f, y);
            if (kb >= 2 && D * D_prev < 0.0f) caustics++;
            D_prev = D;
        }
#pragma unroll
        for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] = t * (1.0f / 6.0f); stg[i] = y[i] + t * 0.5f; }
        rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 3.0f); stg[i] = y[i] + t * 0.5f; }
        rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 3.0f); stg[i] = y[i] + t; }
        rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
        for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 6.0f); }
        kb++;

        // segment increments at the midpoint, from the step vector itself
        {
            const float seg_ds = sqrtf(inc[0] * inc[0] + inc[1] * inc[1] + inc[2] * inc[2]);
            const float zm = y[2] + (lo[2] + 0.5f * inc[2]);
            const float nzm = y[3] + (lo[3] + 0.5f * inc[3]);
            const float ze = fminf(fmaxf(zm, zlo), zhi);
            seg = seg_walk_f(tab, a.n_knots, ze, seg);
            const float* r0 = tab + seg * kStrideF;
            const CubicF q = cubic_at_f(r0, ze);
            const float c = cubicf_f(r0, q, 2);
            float sc = 1.0f;
            if (zm < zbl) { const float X = __expf(-(zm - z0f) * inv_blf); sc = __fdividef(1.0f - X, 1.0f + X); }
            const float u = cubicf_f(r0, q, 6) * sc, v = cubicf_f(r0, q, 10) * sc;
            const float inum = rsqrtf(rc.nx * rc.nx + rc.ny * rc.ny + nzm * nzm);
            const float cgx = c * rc.nx * inum + u, cgy = c * rc.ny * inum + v, cgz = c * nzm * inum;
            const float dt = seg_ds * rsqrtf(cgx * cgx + cgy * cgy + cgz * cgz);
            // alpha(z) table (linear), tweak_abs applied here
            const float ua = (float)((double)zm - a.alpha_z0) * (float)a.alpha_inv_h;
            int ia = (int)ua;
            ia = ia < 0 ? 0 : (ia > a.alpha_n - 2 ? a.alpha_n - 2 : ia);
            const float w = fminf(fmaxf(ua - (float)ia, 0.0f), 1.0f);
            const float al0 = __ldg(a.alpha_tab + ia), al1 = __ldg(a.alpha_tab + ia + 1);
            const float da = (al0 + w * (al1 - al0)) * tweak * seg_ds;
            if (a.write_rays) { tt += pt; att += pa; pt = (double)dt; pa = (double)da; }
            else { pt += (double)dt; pa += (double)da; }
        }

        // new row (not yet committed): hi/lo for 0..3
        float nh[4], nl[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float e;
            two_sum(y[i], inc[i], nh[i], e);
            nl[i] = lo[i] + e;
        }
        const float zn = nh[2] + nl[2];
        const float rx = (nh[0] - (float)a.src_x) + nl[0], ry = (nh[1] - (float)a.src_y) + nl[1];
        const float xn = nh[0] + nl[0], yn = nh[1] + nl[1];
        bool esc = (s > a.s_max) || (sqrtf(rx * rx + ry * ry) > (float)a.rng_max) ||
                   (xn > (float)a.x_max) || (xn < (float)a.x_min) || (yn > (float)a.y_max) || (yn < (float)a.y_min) ||
                   (zn > (float)a.alt_max);
        const bool gnd = !esc && ((nh[2] - z0f) + nl[2] < 0.0f);
        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(zn) || !isfinite(nh[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < N; i++) dprev[i * blockDim.x] = inc[i];
#pragma unroll
            for (int i = 0; i < 4; i++) {   // renormalise the pair
                const float hh = nh[i] + nl[i];
                lo[i] = nl[i] - (hh - nh[i]);
                y[i] = hh;
            }
#pragma unroll
            for (int i = 4; i < N; i++) y[i] += inc[i];
            continue;
        }

        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        int status = -1;
        if (zmax < z0f + (float)a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        if (status < 0) {
            // rows K-1 (y/lo), K (y + inc) and the step K-2 -> K-1 (dprev), in FP64
            double r1[12], rk[12], d1[12];
#pragma unroll
            for (int i = 0; i < N; i++) {
                const double base = (double)y[i] + (i < 4 ? (double)lo[i] : 0.0);
                r1[i] = base;
                rk[i] = base + (double)inc[i];
                d1[i] = (double)dprev[i * blockDim.x];
            }
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            const double nxd = rc.nx, nyd = rc.ny;
            const double incl = -asin(a.c_ratio * rk[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-nyd, -nxd) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            const double ex = rk[0] - a.src_x, ey = rk[1] - a.src_y;
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = rk[0];
            out[4] = rk[1];
            out[5] = tt;
            out[6] = sqrt(ex * ex + ey * ey) / tt;
            out[7] = (double)zmax;
            out[8] = incl;
            out[9] = baz;
            RayConst rcd{nxd, nyd, (double)rc.mtx, (double)rc.mty, (double)rc.mpx, (double)rc.mpy};
            double jac = 0.0;
            if (AMP) {
                int segd = seg_guess(fmin(fmax(rk[2], a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
                out[10] = amp_db(a.knots, a, segd, rk, rcd, th_deg * kPi / 180.0, kPi / 2.0 - ph_deg * kPi / 180.0, &jac);
            } else {
                out[10] = 0.0;
            }
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux(ax, a, rk, rcd, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            // approx_intercept + set_refl (geoac.eqset.3d.strat.cpp:110-209) in FP64
            const double dz_grnd = a.z0 - r1[2];
            const double dz_k = d1[2];
            double p[12];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = r1[i] + d1[i] / dz_k * dz_grnd;
            set_pair(p[0], y[0], lo[0]);
            set_pair(p[1], y[1], lo[1]);
            set_pair(a.z0, y[2], lo[2]);
            set_pair(-p[3], y[3], lo[3]);
            if (AMP) {
                y[4] = (float)p[4]; y[5] = (float)p[5]; y[6] = (float)(-p[6]);
                y[8] = (float)p[8]; y[9] = (float)p[9]; y[10] = (float)(-p[10]);
                const double ds0_dth = -a.c0 / a.c_gnd * p[6] / p[3];
                const double ds0_dph = -a.c0 / a.c_gnd * p[10] / p[3];
                const double dnuz_ds = -1.0 / a.c_gnd * (a.c0 / a.c_gnd * a.dcz_g + nxd * a.duz_g + nyd * a.dvz_g);
                y[7] = (float)(-p[7] + (-2.0 * dnuz_ds) * ds0_dth);
                y[11] = (float)(-p[11] + (-2.0 * dnuz_ds) * ds0_dph);
            }
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
        ray = (int)atomicAdd(a.queue, 1u);
        if (ray >= a.n_rays) break;
        start_ray(ray);
    }
}

// Eigenray-search traces in FP32-compensated form: one request per thread,
// n_seg prop_rk4 segments with flat-ground reflections, the last row in FP64
// (same contract as trace3d_fp64_kernel in eig3d.cu, including the record
// mode's per-step time/absorption sums and turning height from 0 over rows
// 1..k-1, geoac.eigenray.3d.cpp:229-262).  The search's bracket and Newton
// updates stay in FP64 on the host.
template <bool AMP>
__global__ void __launch_bounds__(kThreadsC) trace3d_fp32c_kernel(const __grid_constant__ Fan3DArgs a,
                                                                 const TraceReq* __restrict__ reqs,
                                                                 TraceRes* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                 SegRes* __restrict__ seg_out, int seg_stride) {
    constexpr int N = DimF<AMP>::n;
    extern __shared__ float s_memf[];
    float* s_dprev = s_memf;
    float* s_tab = s_memf + N * blockDim.x;
    {
        const int tot = a.n_knots * kStrideF;
        for (int i = threadIdx.x; i < tot; i += blockDim.x) s_tab[i] = a.knots_f[i];
        __syncthreads();
    }
    // persistent: each thread takes the next request when its trace ends, so
    // lanes whose trace finished early do not idle until the warp's longest one
    for (int r = (int)atomicAdd(queue, 1u); r < n; r = (int)atomicAdd(queue, 1u)) {
        const float* tab = s_tab;
        float* dprev = s_dprev + threadIdx.x;
        const TraceReq q = reqs[r];
        const bool record = (q.flags & kRecord) != 0, stop = (q.flags & kStopOnEscape) != 0;
        const float z0f = (float)a.z0, inv_blf = (float)a.inv_bl;
        const float zlo = (float)a.z_lo, zhi = (float)a.z_hi;
        const float zbl = (float)a.z_bl;
        const float ds_max = (float)a.ds_max, ds_span = (float)(a.ds_max - a.ds_min);
        const float tweak = (float)a.tweak_abs;
        auto set_pair = [](double v, float& h, float& l) { h = (float)v; l = (float)(v - (double)h); };

        float y[N], lo[4], inc[N];
        RayConstF rc;
        {
            const double theta = q.theta, phi = q.phi;
            const double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
            const double mx = a.u0s / a.c0, my = a.v0s / a.c0;
            const double n0x = ct * cp, n0y = ct * sp, n0z = st;
            const double ms = 1.0 + (n0x * mx + n0y * my);
            const double ims = 1.0 / ms, ims2 = ims * ims;
            set_pair(q.x0, y[0], lo[0]);
            set_pair(q.y0, y[1], lo[1]);
            set_pair(a.src_z, y[2], lo[2]);
            set_pair(n0z * ims, y[3], lo[3]);
            rc.nx = (float)(n0x * ims);
            rc.ny = (float)(n0y * ims);
            if (AMP) {
                const double tx = -st * cp, ty = -st * sp, tz = ct;
                const double px = -ct * sp, py = ct * cp;
                const double tm = tx * mx + ty * my, pm = px * mx + py * my;
                rc.mtx = (float)(tx * ims - n0x * ims2 * tm);
                rc.mty = (float)(ty * ims - n0y * ims2 * tm);
                y[7] = (float)(tz * ims - n0z * ims2 * tm);
                rc.mpx = (float)(px * ims - n0x * ims2 * pm);
                rc.mpy = (float)(py * ims - n0y * ims2 * pm);
                y[11] = (float)(-n0z * ims2 * pm);
                y[4] = y[5] = y[6] = 0.0f;
                y[8] = y[9] = y[10] = 0.0f;
            } else {
                rc.mtx = rc.mty = rc.mpx = rc.mpy = 0.0f;
            }
        }
        int seg = seg_guess(fmin(fmax(a.src_z, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        double tt = 0.0, att = 0.0;
        float zmax = 0.0f;
        long long steps = 0;
        bool esc = false;
#pragma unroll
        for (int i = 0; i < N; i++) inc[i] = 0.0f;
        for (int sg = 0; sg < q.n_seg; sg++) {
            double s = 0.0, pt = 0.0, pa = 0.0;
            int kb = 0;
            bool capped = false;
#pragma unroll
            for (int i = 0; i < N; i++) dprev[i * blockDim.x] = 0.0f;
            while (true) {
                const float zc = y[2] + lo[2];
                if (record && kb >= 1) zmax = fmaxf(zmax, zc);
                float ds = ds_max;
                if (zc < zbl) ds -= ds_span * __expf(-(zc - z0f) * 5.0f);
                s += (double)ds;
                float stg[N], f[N];
                rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, y, rc, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] = t * (1.0f / 6.0f); stg[i] = y[i] + t * 0.5f; }
                rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 3.0f); stg[i] = y[i] + t * 0.5f; }
                rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 3.0f); stg[i] = y[i] + t; }
                rhs_f<AMP>(tab, a, z0f, inv_blf, zlo, zhi, seg, stg, rc, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const float t = ds * f[i]; inc[i] += t * (1.0f / 6.0f); }
                kb++;
                if (record) {
                    const float seg_ds = sqrtf(inc[0] * inc[0] + inc[1] * inc[1] + inc[2] * inc[2]);
                    const float zm = y[2] + (lo[2] + 0.5f * inc[2]);
                    const float nzm = y[3] + (lo[3] + 0.5f * inc[3]);
                    const float ze = fminf(fmaxf(zm, zlo), zhi);
                    seg = seg_walk_f(tab, a.n_knots, ze, seg);
                    const float* r0 = tab + seg * kStrideF;
                    const CubicF cq = cubic_at_f(r0, ze);
                    const float c = cubicf_f(r0, cq, 2);
                    float sc = 1.0f;
                    if (zm < zbl) { const float X = __expf(-(zm - z0f) * inv_blf); sc = __fdividef(1.0f - X, 1.0f + X); }
                    const float u = cubicf_f(r0, cq, 6) * sc, v = cubicf_f(r0, cq, 10) * sc;
                    const float inum = rsqrtf(rc.nx * rc.nx + rc.ny * rc.ny + nzm * nzm);
                    const float cgx = c * rc.nx * inum + u, cgy = c * rc.ny * inum + v, cgz = c * nzm * inum;
                    const float dt = seg_ds * rsqrtf(cgx * cgx + cgy * cgy + cgz * cgz);
                    const float ua = (float)((double)zm - a.alpha_z0) * (float)a.alpha_inv_h;
                    int ia = (int)ua;
                    ia = ia < 0 ? 0 : (ia > a.alpha_n - 2 ? a.alpha_n - 2 : ia);
                    const float w = fminf(fmaxf(ua - (float)ia, 0.0f), 1.0f);
                    const float al0 = __ldg(a.alpha_tab + ia), al1 = __ldg(a.alpha_tab + ia + 1);
                    const float da = (al0 + w * (al1 - al0)) * tweak * seg_ds;
                    tt += pt; att += pa; pt = (double)dt; pa = (double)da;
                }
                float nh[4], nl[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    float e;
                    two_sum(y[i], inc[i], nh[i], e);
                    nl[i] = lo[i] + e;
                }
                const float zn = nh[2] + nl[2];
                const float rx = (nh[0] - (float)q.x0) + nl[0], ry = (nh[1] - (float)q.y0) + nl[1];
                const float xn = nh[0] + nl[0], yn = nh[1] + nl[1];
                esc = (s > a.s_max) || (sqrtf(rx * rx + ry * ry) > (float)a.rng_max) || (xn > (float)a.x_max) ||
                      (xn < (float)a.x_min) || (yn > (float)a.y_max) || (yn < (float)a.y_min) || (zn > (float)a.alt_max);
                const bool gnd = !esc && ((nh[2] - z0f) + nl[2] < 0.0f);
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(zn) || !isfinite(nh[3])) esc = true;
                }
                if (!esc && !gnd) {
#pragma unroll
                    for (int i = 0; i < N; i++) dprev[i * blockDim.x] = inc[i];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float hh = nh[i] + nl[i];
                        lo[i] = nl[i] - (hh - nh[i]);
                        y[i] = hh;
                    }
#pragma unroll
                    for (int i = 4; i < N; i++) y[i] += inc[i];
                    continue;
                }
                break;
            }
            steps += capped ? a.length : kb;
            if (seg_out) {
                SegRes& g = seg_out[(size_t)r * seg_stride + sg];
                g.x = (double)y[0] + (double)lo[0] + (double)inc[0];
                g.y = (double)y[1] + (double)lo[1] + (double)inc[1];
                g.steps = steps;
                g.escaped = esc ? 1 : 0;
            }
            if (sg == q.n_seg - 1 || (esc && stop)) break;
            // approx_intercept + flat-ground set_refl in FP64 from rows k-1 and k-2
            double r1[12], d1[12], p[12];
#pragma unroll
            for (int i = 0; i < N; i++) {
                r1[i] = (double)y[i] + (i < 4 ? (double)lo[i] : 0.0);
                d1[i] = (double)dprev[i * blockDim.x];
            }
            const double dz_grnd = a.z0 - r1[2];
            const double dz_k = d1[2];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = r1[i] + d1[i] / dz_k * dz_grnd;
            set_pair(p[0], y[0], lo[0]);
            set_pair(p[1], y[1], lo[1]);
            set_pair(a.z0, y[2], lo[2]);
            set_pair(-p[3], y[3], lo[3]);
            if (AMP) {
                y[4] = (float)p[4]; y[5] = (float)p[5]; y[6] = (float)(-p[6]);
                y[8] = (float)p[8]; y[9] = (float)p[9]; y[10] = (float)(-p[10]);
                const double ds0_dth = -a.c0 / a.c_gnd * p[6] / p[3];
                const double ds0_dph = -a.c0 / a.c_gnd * p[10] / p[3];
                const double dnuz_ds = -1.0 / a.c_gnd * (a.c0 / a.c_gnd * a.dcz_g + (double)rc.nx * a.duz_g + (double)rc.ny * a.dvz_g);
                y[7] = (float)(-p[7] + (-2.0 * dnuz_ds) * ds0_dth);
                y[11] = (float)(-p[11] + (-2.0 * dnuz_ds) * ds0_dph);
            }
#pragma unroll
            for (int i = 0; i < N; i++) inc[i] = 0.0f;
        }
        double rk[12];
#pragma unroll
        for (int i = 0; i < 12; i++) rk[i] = 0.0;
#pragma unroll
        for (int i = 0; i < N; i++) rk[i] = (double)y[i] + (i < 4 ? (double)lo[i] : 0.0) + (double)inc[i];
        TraceRes& o = out[r];
#pragma unroll
        for (int i = 0; i < 12; i++) o.y[i] = rk[i];
        o.rc[0] = rc.nx; o.rc[1] = rc.ny; o.rc[2] = rc.mtx; o.rc[3] = rc.mty; o.rc[4] = rc.mpx; o.rc[5] = rc.mpy;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        if (record) {
            o.tt = tt; o.att = att; o.zmax = (double)zmax;
            RayConst rcd{(double)rc.nx, (double)rc.ny, (double)rc.mtx, (double)rc.mty, (double)rc.mpx, (double)rc.mpy};
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
}

template <bool AMP>
cudaError_t launch_trace_c(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, cudaStream_t st,
                           SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = trace3d_fp32c_kernel<AMP>;
    const size_t smem = (size_t)DimF<AMP>::n * kThreadsC * sizeof(float) + (size_t)a.n_knots * kStrideF * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kThreadsC, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kThreadsC, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride);
    return cudaGetLastError();
}

template <bool AMP>
cudaError_t launch_c(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    // threads per block: the caller's choice (a multiple of 32 up to kThreadsC) or kThreadsC
    const int threads = a.block > 0 ? a.block : kThreadsC;
    auto kern = fan3d_fp32c_kernel<AMP>;
    const size_t smem = (size_t)DimF<AMP>::n * threads * sizeof(float) + (size_t)a.n_knots * kStrideF * sizeof(float);
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
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fan3d_fp32c(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    return calc_amp ? launch_c<true>(a, stream, grid_used) : launch_c<false>(a, stream, grid_used);
}

cudaError_t launch_trace_fp32c(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, bool amp,
                               cudaStream_t st, unsigned int* d_queue, SegRes* seg_out, int seg_stride) {
    return amp ? launch_trace_c<true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
               : launch_trace_c<false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
}

}  // namespace iga
