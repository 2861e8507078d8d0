// Ray traces of the spherical eigenray search (stratified atmosphere, flat
// ground at r_earth + z0): the spherical counterpart of trace3d_fp64_kernel.
//
// One request per thread: launch from the request's source latitude and
// longitude, integrate n_seg prop_rk4 segments with flat-ground reflections
// between them and return the last row.  Record mode sums travel time and
// absorption per step and the turning height over rows 1..k-1 of every
// segment from 0, and forms the arrival columns the way find_eigenray writes
// them (src/geoac/geoac.eigenray.sph.cpp:230-317), including its arrival
// inclination with c taken at a radius equal to the source ALTITUDE (so at
// the bottom of the profile, atmo::c clamps it; :284).
#include "eig3d.cuh"
#include "fan3d_common.cuh"
#include "fansph_common.cuh"

namespace iga {
namespace {

constexpr int kSphTraceThreads = 128;

template <bool AMP>
__global__ void __launch_bounds__(kSphTraceThreads) tracesph_fp64_kernel(const __grid_constant__ Fan3DArgs a,
                                                                         const TraceReq* __restrict__ reqs,
                                                                         TraceRes18* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                         SegRes* __restrict__ seg_out, int seg_stride,
                                                                         double c_incl_src) {
    constexpr int N = DimSph<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    double* s_tab = s_mem + N * kSphTraceThreads;
    const int tot = a.n_knots * kStride;
    for (int i = threadIdx.x; i < tot; i += blockDim.x) s_tab[i] = a.knots[i];
    __syncthreads();
    const double* tab = s_tab;
    // persistent: each thread takes the next request when its trace ends, so
    // lanes whose trace finished early do not idle until the warp's longest one
    for (int r = (int)atomicAdd(queue, 1u); r < n; r = (int)atomicAdd(queue, 1u)) {
        double* prev = s_prev + threadIdx.x;
        const TraceReq q = reqs[r];
        const bool record = (q.flags & kRecord) != 0, stop = (q.flags & kStopOnEscape) != 0;
        const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;
        const double cos_slat = cos(q.x0);
        // break_check's range test from this request's source (beyond_range)
        auto beyond = [&](double lat, double lon) {
            const double s1 = sin((q.x0 - lat) * 0.5), s2 = sin((q.y0 - lon) * 0.5);
            const double h = s1 * s1 + cos(lat) * cos_slat * (s2 * s2);
            if (!a.rng_exact_only && fabs(h - a.hav_rng) > 1e-9 * a.hav_rng) return h > a.hav_rng;
            return 2.0 * a.r_earth * asin(sqrt(h)) > a.rng_max;
        };

        double y[N];
        ray_init_sph<AMP>(a, q.theta, q.phi, y);
        y[1] = q.x0;
        y[2] = q.y0;
        int seg = seg_guess(fmin(fmax(y[0] - a.r_earth, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        double tt = 0.0, att = 0.0, rmax = 0.0;
        long long steps = 0;
        double acc[N];
        bool esc = false;
        for (int sg = 0; sg < q.n_seg; sg++) {
            double s = 0.0, pt = 0.0, pa = 0.0;
            int kb = 0;
            bool capped = false;
#pragma unroll
            for (int i = 0; i < N; i++) prev[i * kSphTraceThreads] = y[i];
            while (true) {
                if (record && kb >= 1) rmax = fmax(rmax, y[0] - a.r_earth);
                double ds = a.ds_max;   // set_ds (geoac.eqset.sph.strat.cpp:216-222)
                if (y[0] - a.r_earth < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - a.r_grnd) / 0.2);
                s += ds;
                double stg[N], f[N];
                rhs_sph<AMP>(tab, a, seg, y, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
                // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
                for (int st = 0; st < 3; st++) {
                    rhs_sph<AMP>(tab, a, seg, stg, f);
                    const double w = st < 2 ? c_third : c_sixth;
                    const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
                    for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
                }
                kb++;
                // s_max and break_check (in-place longitude wrap first), ground_check
                esc = s > a.s_max;
                if (!esc) {
                    if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
                    else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
                    esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                          beyond(acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                          (acc[2] < a.lon_min || acc[2] > a.lon_max);
                }
                const bool gnd = !esc && (acc[0] - a.r_earth <= a.z0) && (acc[0] < a.r_grnd);
                if (record) {
                    double dt, da;
                    seg_increment_sph(tab, a, seg, y, acc, dt, da);
                    tt += pt; att += pa; pt = dt; pa = da;
                }
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(acc[0]) || !isfinite(acc[1]) || !isfinite(acc[3])) esc = true;
                }
                if (!esc && !gnd) {
#pragma unroll
                    for (int i = 0; i < N; i++) { prev[i * kSphTraceThreads] = y[i]; y[i] = acc[i]; }
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
            // approx_intercept + set_refl on flat ground (as the spherical fan kernel)
            const double dr_grnd = a.r_grnd - y[0];
            const double dr_k = y[0] - prev[0];
            double p[N];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * kSphTraceThreads]) / dr_k * dr_grnd;
            y[0] = a.r_grnd; y[1] = p[1]; y[2] = p[2];
            y[3] = -p[3]; y[4] = p[4]; y[5] = p[5];
            if (AMP) {
                const double dnu_r = (((a.refl_k1 + p[4] * a.dvz_g) + p[5] * a.duz_g) + a.refl_k2 * (p[4] * p[4] + p[5] * p[5])) *
                                     a.refl_k3;
                const double ds0_dth = a.refl_mcr * p[6] / p[3];
                const double ds0_dph = a.refl_mcr * p[12] / p[3];
                y[6] = -p[6]; y[7] = p[7]; y[8] = p[8];
                y[9] = -p[9] + (-2.0 * dnu_r) * ds0_dth;
                y[10] = p[10]; y[11] = p[11];
                y[12] = -p[12]; y[13] = p[13]; y[14] = p[14];
                y[15] = -p[15] + (-2.0 * dnu_r) * ds0_dph;
                y[16] = p[16]; y[17] = p[17];
            }
        }
        TraceRes18& o = out[r];
#pragma unroll
        for (int i = 0; i < 18; i++) o.y[i] = i < N ? acc[i] : 0.0;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        // flat ground under every row
        o.c_src = a.c0; o.c_grnd = a.c_gnd; o.z_grnd = a.r_grnd; o.dzg[0] = 0.0; o.dzg[1] = 0.0;
        if (record) {
            o.tt = tt; o.att = att; o.zmax = rmax;
            o.amp_db = AMP ? amp_db_sph(tab, a, seg, acc, q.theta, q.phi, nullptr) : 0.0;
            const double ze = fmin(fmax(acc[0] - a.r_earth, a.z_lo), a.z_hi);
            seg = seg_walk(tab, a.n_knots, ze, seg);
            const double* r0 = tab + seg * kStride;
            const double c_k = cubic_f(r0, cubic_at(r0, ze), 2);
            o.incl = -asin(c_k / c_incl_src * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * (180.0 / kPi);
            while (baz < -180.0) baz += 360.0;
            while (baz > 180.0) baz -= 360.0;
            o.baz = baz;
        } else {
            o.tt = o.att = o.zmax = o.amp_db = o.incl = o.baz = 0.0;
        }
    }
}

template <bool AMP>
cudaError_t launch_impl(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, cudaStream_t st,
                        SegRes* seg_out, int seg_stride, double c_incl_src, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = tracesph_fp64_kernel<AMP>;
    const size_t smem =
        (size_t)DimSph<AMP>::n * kSphTraceThreads * sizeof(double) + (size_t)a.n_knots * kStride * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kSphTraceThreads, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kSphTraceThreads, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride, c_incl_src);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_trace_sph(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                             cudaStream_t st, SegRes* seg_out, int seg_stride, double c_incl_src,
                             unsigned int* d_queue) {
    return amp ? launch_impl<true>(a, d_req, d_res, n, st, seg_out, seg_stride, c_incl_src, d_queue)
               : launch_impl<false>(a, d_req, d_res, n, st, seg_out, seg_stride, c_incl_src, d_queue);
}

}  // namespace iga
