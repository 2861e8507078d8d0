// Eigenray search for the 3D and spherical stratified solvers on flat ground.
//
// Every (source-receiver pair, bounce count) search is an independent chain
// of ray traces whose control flow depends on each trace's result; the host
// runs all chains as state machines that replay the reference's
// est_eigenray / find_eigenray logic exactly (geoac.eigenray.3d.cpp:34-371,
// geoac.eigenray.sph.cpp:42-380), and every round collects the traces all
// chains need next into one launch of trace3d_fp64_kernel (or the spherical
// tracesph_fp64_kernel, eigsph.cu).  While a chain sweeps inclinations with a fixed
// step, the angles it will try next are known in advance, so it submits a
// chunk of them at once and keeps the results up to the first bracket.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "eig3d.cuh"
#include "fan3d_common.cuh"
#include "handle.h"
#include "nvtx.h"

namespace iga {
namespace {

constexpr int kTraceThreads = 128;

// One request per thread: launch, integrate n_seg prop_rk4 segments with
// flat-ground reflections between them, return the last row.  Record mode
// accumulates travel time / absorption per step and the turning height over
// rows 1..k-1 of each segment starting from 0, as find_eigenray's final trace
// does (geoac.eigenray.3d.cpp:229-262).
template <bool AMP>
__global__ void __launch_bounds__(kTraceThreads) trace3d_fp64_kernel(const __grid_constant__ Fan3DArgs a,
                                                                    const TraceReq* __restrict__ reqs,
                                                                    TraceRes* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                    SegRes* __restrict__ seg_out, int seg_stride) {
    constexpr int N = Dim<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    double* s_tab = s_mem + N * kTraceThreads;
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

        double y[N];
        RayConst rc;
        ray_init<AMP>(a, q.theta, q.phi, y, rc);
        y[0] = q.x0;
        y[1] = q.y0;
        int seg = seg_guess(fmin(fmax(y[2], a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        double tt = 0.0, att = 0.0, zmax = 0.0;
        long long steps = 0;
        double acc[N];
        bool esc = false;
        for (int sg = 0; sg < q.n_seg; sg++) {
            double s = 0.0, pt = 0.0, pa = 0.0;
            int kb = 0;
            bool capped = false;
#pragma unroll
            for (int i = 0; i < N; i++) prev[i * kTraceThreads] = y[i];
            while (true) {
                if (record && kb >= 1) zmax = fmax(zmax, y[2]);
                double ds = a.ds_max;
                if (y[2] < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[2] - a.z0) / 0.2);
                s += ds;
                double stg[N], f[N];
                rhs<AMP>(tab, a, seg, y, rc, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
                // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
                for (int st = 0; st < 3; st++) {
                    rhs<AMP>(tab, a, seg, stg, rc, f);
                    const double w = st < 2 ? c_third : c_sixth;
                    const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
                    for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
                }
                kb++;
                if (record) {
                    double dt, da;
                    seg_increment(tab, a, seg, y, acc, rc, dt, da);
                    tt += pt; att += pa; pt = dt; pa = da;
                }
                const double rx = acc[0] - q.x0, ry = acc[1] - q.y0;
                esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) || (acc[0] > a.x_max) ||
                      (acc[0] < a.x_min) || (acc[1] > a.y_max) || (acc[1] < a.y_min) || (acc[2] > a.alt_max);
                const bool gnd = !esc && (acc[2] < a.z0);
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(acc[2]) || !isfinite(acc[3])) esc = true;
                }
                if (!esc && !gnd) {
#pragma unroll
                    for (int i = 0; i < N; i++) { prev[i * kTraceThreads] = y[i]; y[i] = acc[i]; }
                    continue;
                }
                break;
            }
            steps += capped ? a.length : kb;
            if (seg_out) {
                SegRes& g = seg_out[(size_t)r * seg_stride + sg];
                g.x = acc[0]; g.y = acc[1]; g.steps = steps; g.escaped = esc ? 1 : 0;
            }
            if (sg == q.n_seg - 1 || (esc && stop)) break;
            // reflection from rows k-2 (prev) and k-1 (y), flat ground
            const double dz_grnd = a.z0 - y[2];
            const double dz_k = y[2] - prev[2 * kTraceThreads];
            double p[N];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * kTraceThreads]) / dz_k * dz_grnd;
            y[0] = p[0]; y[1] = p[1]; y[2] = a.z0; y[3] = -p[3];
            if (AMP) {
                y[4] = p[4]; y[5] = p[5]; y[6] = -p[6];
                y[8] = p[8]; y[9] = p[9]; y[10] = -p[10];
                const double ds0_dth = -a.c0 / a.c_gnd * p[6] / p[3];
                const double ds0_dph = -a.c0 / a.c_gnd * p[10] / p[3];
                const double dnuz_ds = -1.0 / a.c_gnd * (a.c0 / a.c_gnd * a.dcz_g + rc.nx * a.duz_g + rc.ny * a.dvz_g);
                y[7] = -p[7] + (-2.0 * dnuz_ds) * ds0_dth;
                y[11] = -p[11] + (-2.0 * dnuz_ds) * ds0_dph;
            }
        }
        TraceRes& o = out[r];
#pragma unroll
        for (int i = 0; i < 12; i++) o.y[i] = i < N ? acc[i] : 0.0;
        o.rc[0] = rc.nx; o.rc[1] = rc.ny; o.rc[2] = rc.mtx; o.rc[3] = rc.mty; o.rc[4] = rc.mpx; o.rc[5] = rc.mpy;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        if (record) {
            o.tt = tt; o.att = att; o.zmax = zmax;
            o.amp_db = AMP ? amp_db(tab, a, seg, acc, rc, q.theta, q.phi, nullptr) : 0.0;
            // arrival inclination with c at the (clamped) below-ground altitude,
            // as find_eigenray writes it (geoac.eigenray.3d.cpp:265)
            const double ze = fmin(fmax(acc[2], a.z_lo), a.z_hi);
            seg = seg_walk(tab, a.n_knots, ze, seg);
            const double* r0 = tab + seg * kStride;
            const double c_k = cubic_f(r0, cubic_at(r0, ze), 2);
            o.incl = -asin(c_k / a.c0 * acc[3]) * (180.0 / kPi);
            double baz = 90.0 - atan2(-rc.ny, -rc.nx) * (180.0 / kPi);
            while (baz > 180.0) baz -= 360.0;
            while (baz < -180.0) baz += 360.0;
            o.baz = baz;
        }
    }
}

template <bool AMP>
cudaError_t launch_trace(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, cudaStream_t st,
                         unsigned int* d_queue, SegRes* seg_out = nullptr, int seg_stride = 0) {
    if (n <= 0) return cudaSuccess;
    auto kern = trace3d_fp64_kernel<AMP>;
    const size_t smem = (size_t)Dim<AMP>::n * kTraceThreads * sizeof(double) + (size_t)a.n_knots * kStride * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kTraceThreads, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kTraceThreads, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- host side

constexpr double kRad = kPi / 180.0;

struct Chain {
    int pair = 0, nb = 0;
    // 3D: source / receiver x, y [km]; spherical: latitude, longitude [rad]
    double sx = 0, sy = 0, rx = 0, ry = 0, rcvr_rng = 0, rcvr_az = 0;
    double phi0 = 0;             // first launch azimuth of a sweep (geoac::phi convention)
    enum Phase { kEst, kNewton, kRecordTrace, kDone } phase = kEst;
    bool direct = false;         // find_eigenray alone (run_eig_direct): no sweep before or after
    double theta_start = 0;
    // est_eigenray state
    double th_min = 0, th_max = 0, dth = 0, dph = 0, r = 0, r_prev = 0, phi = 0, th = 0, th_next = 0;
    int iterations = 0;
    bool th_max_reached = false;
    // find_eigenray state (dth/dph start at 0: the reference leaves them
    // uninitialised until the first Newton update)
    double theta = 0, phi_n = 0, dr_prev = 0, step_sc = 1, ndth = 0, ndph = 0;
    int n = 0;
    // requests of the current round
    std::vector<double> sweep;   // inclinations submitted (est phase)
    std::vector<int> sweep_req;  // their (shared) sweep requests
    int req0 = 0;                // first request index in its batch
    std::vector<std::vector<double>> rows;
};

struct Settings {
    double theta_max, dth_big, dth_sml, damping, tolerance, az_err_lim, rng_max;
    int iterations, chunk;
    // spherical search (geoac.eigenray.sph.cpp): great-circle ranges and
    // bearings, strict upper inclination bound, mod_dth after 3 corrections,
    // Newton traces through every bounce; flat-ground radius and the sound
    // speeds of its Newton derivatives
    bool sph = false;
    double r_grnd = 0, c_src = 0, c_grnd = 0;
    int fixed_step_iters() const { return sph ? 3 : 2; }
    bool in_sweep(double th, double th_max) const { return sph ? th < th_max : th <= th_max; }
};

// globe::gc_dist and globe::bearing (util/globe.cpp:16-28), host side
double gc_dist_h(double lat1, double lon1, double lat2, double lon2) {
    const double t1 = pow(sin((lat2 - lat1) / 2.0), 2);
    const double t2 = cos(lat1) * cos(lat2) * pow(sin((lon2 - lon1) / 2.0), 2);
    return 2.0 * kEarthRadiusKm * asin(sqrt(t1 + t2));
}
double bearing_h(double lat1, double lon1, double lat2, double lon2) {
    const double t1 = sin(lon2 - lon1);
    const double t2 = cos(lat1) * tan(lat2) - sin(lat1) * cos(lon2 - lon1);
    return atan2(t1, t2);
}

double mod_dth(const Settings& S, double dr, double dr_dtheta) {   // geoac::mod_dth (geoac.eigenray.3d.cpp:32)
    return S.dth_big - (S.dth_big - S.dth_sml) * exp(-1.0 / 2.0 * pow(dr / dr_dtheta, 2));
}

void est_begin(Chain& c, const Settings& S, double theta_start) {
    c.phase = Chain::kEst;
    c.theta_start = theta_start;
    c.th_min = theta_start;
    c.th_max = S.theta_max;
    c.iterations = 0;
    c.dth = S.dth_big;
    c.dph = 100.0;
    c.phi = c.phi0;
    c.th_max_reached = false;
    c.r = c.rcvr_rng;
    c.r_prev = c.rcvr_rng;
    c.th = c.th_min;
}

// After est_eigenray (and find_eigenray, if it ran): run_eig_search's
// theta_start = theta_next and loop condition (main.infraga.3d.cpp:943-949).
void search_continue(Chain& c, const Settings& S) {
    if (c.direct) { c.phase = Chain::kDone; return; }
    const double ts = c.th_next;
    if (ts < S.theta_max) est_begin(c, S, ts);
    else c.phase = Chain::kDone;
}

void newton_begin(Chain& c, double th_est, double ph_est) {
    c.phase = Chain::kNewton;
    c.theta = th_est;
    c.phi_n = ph_est;
    c.dr_prev = 10000.0;
    c.step_sc = 1.0;
    c.ndth = 0.0;
    c.ndph = 0.0;
    c.n = 0;
}

// One body of est_eigenray's inclination loop for the trace at c.th.
// Returns true when the chain leaves the sweep (later speculative results
// are then discarded).
bool est_step(Chain& c, const Settings& S, const TraceRes& res) {
    if (c.th + c.dth >= c.th_max) c.th_max_reached = true;
    const double theta = c.th;
    c.r = S.sph ? gc_dist_h(c.sx, c.sy, res.y[0], res.y[1]) : sqrt(pow(res.y[0] - c.sx, 2) + pow(res.y[1] - c.sy, 2));
    if (res.escaped) c.r = S.rng_max;
    if (((c.r - c.rcvr_rng) * (c.r_prev - c.rcvr_rng) <= 0.0) && (c.r < S.rng_max) && (c.r_prev < S.rng_max) &&
        (c.th > c.th_min)) {
        if (c.iterations == 0) c.th_next = c.th;
        if (S.sph) {
            c.dph = bearing_h(c.sx, c.sy, c.rx, c.ry) * (180.0 / kPi);
            c.dph -= bearing_h(c.sx, c.sy, res.y[0], res.y[1]) * (180.0 / kPi);
        } else {
            c.dph = atan2(res.y[1] - c.sy, res.y[0] - c.sx) * (180.0 / kPi);
            c.dph -= atan2(c.ry - c.sy, c.rx - c.sx) * (180.0 / kPi);
        }
        while (c.dph > 180.0) c.dph -= 360.0;
        while (c.dph < -180.0) c.dph += 360.0;
        if (fabs(c.dph) < S.az_err_lim) {
            newton_begin(c, theta - c.dth, c.phi);
            return true;
        }
        c.phi -= c.dph * (kPi / 180.0) * 0.9;
        c.th_min = std::max(c.th - 5.0 * (kPi / 180.0), c.th_min);
        c.iterations++;
        // break out of the inclination loop
        if (c.th_max_reached) { c.th_next = c.th_max; search_continue(c, S); return true; }
        if (!(fabs(c.dph * (180.0 / kPi)) > S.az_err_lim && c.iterations < 5)) { search_continue(c, S); return true; }
        c.r = c.rcvr_rng; c.r_prev = c.rcvr_rng; c.th = c.th_min;
        return true;
    }
    if (c.iterations >= S.fixed_step_iters()) c.dth = mod_dth(S, c.r - c.rcvr_rng, (c.r - c.r_prev) / (2.0 * c.dth));
    c.r_prev = c.r;
    c.th += c.dth;
    if (!S.in_sweep(c.th, c.th_max)) {   // loop ran out (th_max_reached is set on its last pass)
        if (c.th_max_reached) { c.th_next = c.th_max; search_continue(c, S); return true; }
        if (!(fabs(c.dph * (180.0 / kPi)) > S.az_err_lim && c.iterations < 5)) { search_continue(c, S); return true; }
        c.r = c.rcvr_rng; c.r_prev = c.rcvr_rng; c.th = c.th_min;
        return true;
    }
    return false;
}

// One iteration of find_eigenray's Newton loop on the trace at (theta, phi).
void newton_step(Chain& c, const Settings& S, const Fan3DArgs& a, const TraceRes& res) {
    if (res.escaped) {
        c.theta -= c.ndth * c.step_sc;
        c.phi_n -= c.ndph * c.step_sc;
        c.step_sc /= 2.0;
    } else {
        const double x = res.y[0], dx = c.rx - x;
        const double y = res.y[1], dy = c.ry - y;
        const double dr = sqrt(pow(dx, 2) + pow(dy, 2));
        if (dr < S.tolerance) {
            c.phase = Chain::kRecordTrace;
            return;
        } else if (c.n > 0 && dr > c.dr_prev) {
            c.theta -= c.ndth * c.step_sc;
            c.phi_n -= c.ndph * c.step_sc;
            c.step_sc /= 2.0;
        } else {
            c.step_sc = std::min(1.0, c.step_sc * 1.25);
            const double c_src = a.c0, c_grnd = a.c_gnd;
            const double nx = res.rc[0], ny = res.rc[1], nz = res.y[3];
            const double ds_dth = -c_src / c_grnd * res.y[6] / nz;
            const double ds_dph = -c_src / c_grnd * res.y[10] / nz;
            const double dx_dth = res.y[4] + nx * ds_dth, dy_dth = res.y[5] + ny * ds_dth;
            const double dx_dph = res.y[8] + nx * ds_dph, dy_dph = res.y[9] + ny * ds_dph;
            const double det = pow(1.0 + S.damping, 2) * (dx_dth * dy_dph - dx_dph * dy_dth);
            c.ndth = ((1.0 + S.damping) * dy_dph * dx - dx_dph * dy) / det;
            c.ndph = ((1.0 + S.damping) * dx_dth * dy - dy_dth * dx) / det;
            c.theta += c.ndth * c.step_sc;
            c.phi_n += c.ndph * c.step_sc;
            c.dr_prev = dr;
        }
    }
    if (sqrt(c.ndth * c.ndth + c.ndph * c.ndph) * c.step_sc < 1.0e-12) { search_continue(c, S); return; }
    c.n++;
}

// One iteration of the spherical find_eigenray Newton loop
// (geoac.eigenray.sph.cpp:176-371).  The trace returns the ground under its
// last row (radius, gradient, sound speed there; flat ground gives a zero
// gradient, and the terrain terms then vanish exactly).  The reference's long
// double block is done in double.
void newton_step_sph(Chain& c, const Settings& S, const TraceRes18& res) {
    if (res.escaped) {
        c.theta -= c.ndth * c.step_sc;
        c.phi_n -= c.ndph * c.step_sc;
        c.step_sc /= 2.0;
    } else {
        const double* s = res.y;
        const double dr = gc_dist_h(s[1], s[2], c.rx, c.ry);
        if (dr < S.tolerance) {
            c.phase = Chain::kRecordTrace;
            return;
        } else if (c.n > 0 && dr > c.dr_prev) {
            c.theta -= c.ndth * c.step_sc;
            c.phi_n -= c.ndph * c.step_sc;
            c.step_sc /= 2.0;
        } else {
            c.step_sc = std::min(1.0, c.step_sc * 1.25);
            const double dlat = c.rx - s[1], dlon = c.ry - s[2];
            const double r_grnd = res.z_grnd, c_grnd = res.c_grnd, c_src = res.c_src;
            const double rc = r_grnd * cos(s[1]);
            const double dzg_dlat = res.dzg[0] / r_grnd, dzg_dlon = res.dzg[1] / rc;
            const double ds_norm = s[3] - dzg_dlat * s[4] - dzg_dlon * s[5];
            const double ds_dth = -c_src / c_grnd * (s[6] - dzg_dlat * r_grnd * s[7] - dzg_dlon * rc * s[8]) / ds_norm;
            const double ds_dph = -c_src / c_grnd * (s[12] - dzg_dlat * r_grnd * s[13] - dzg_dlon * rc * s[14]) / ds_norm;
            const double dlat_dth = s[7] + s[4] / r_grnd * ds_dth, dlon_dth = s[8] + s[5] / rc * ds_dth;
            const double dlat_dph = s[13] + s[4] / r_grnd * ds_dph, dlon_dph = s[14] + s[5] / rc * ds_dph;
            // (1 + damping)^2 multiplies the first product only, as written in the reference
            const double det = pow(1.0 + S.damping, 2) * dlat_dth * dlon_dph - dlat_dph * dlon_dth;
            c.ndth = ((1.0 + S.damping) * dlon_dph * dlat - dlat_dph * dlon) / det;
            c.ndph = ((1.0 + S.damping) * dlat_dth * dlon - dlon_dth * dlat) / det;
            c.theta += c.ndth * c.step_sc;
            c.phi_n += c.ndph * c.step_sc;
            c.dr_prev = dr;
        }
    }
    if (sqrt(c.ndth * c.ndth + c.ndph * c.ndph) * c.step_sc < 1.0e-12) { search_continue(c, S); return; }
    c.n++;
}

// One iteration of the 3D find_eigenray Newton loop on a range-dependent
// atmosphere with terrain (geoac.eigenray.3d.cpp:320-355, the is_topo
// branch; without terrain the gradient is zero and it reduces exactly to the
// flat form), 18-state layout.
void newton_step_3dr(Chain& c, const Settings& S, const TraceRes18& res) {
    if (res.escaped) {
        c.theta -= c.ndth * c.step_sc;
        c.phi_n -= c.ndph * c.step_sc;
        c.step_sc /= 2.0;
    } else {
        const double* s = res.y;
        const double x = s[0], dx = c.rx - x;
        const double y = s[1], dy = c.ry - y;
        const double dr = sqrt(pow(dx, 2) + pow(dy, 2));
        if (dr < S.tolerance) {
            c.phase = Chain::kRecordTrace;
            return;
        } else if (c.n > 0 && dr > c.dr_prev) {
            c.theta -= c.ndth * c.step_sc;
            c.phi_n -= c.ndph * c.step_sc;
            c.step_sc /= 2.0;
        } else {
            c.step_sc = std::min(1.0, c.step_sc * 1.25);
            const double c_src = res.c_src, c_grnd = res.c_grnd, gx = res.dzg[0], gy = res.dzg[1];
            const double den = s[5] - gx * s[3] - gy * s[4];
            const double ds_dth = -c_src / c_grnd * (s[8] - gx * s[6] - gy * s[7]) / den;
            const double ds_dph = -c_src / c_grnd * (s[14] - gx * s[12] - gy * s[13]) / den;
            const double dx_dth = s[6] + s[3] * ds_dth, dy_dth = s[7] + s[4] * ds_dth;
            const double dx_dph = s[12] + s[3] * ds_dph, dy_dph = s[13] + s[4] * ds_dph;
            const double det = pow(1.0 + S.damping, 2) * (dx_dth * dy_dph - dx_dph * dy_dth);
            c.ndth = ((1.0 + S.damping) * dy_dph * dx - dx_dph * dy) / det;
            c.ndph = ((1.0 + S.damping) * dx_dth * dy - dy_dth * dx) / det;
            c.theta += c.ndth * c.step_sc;
            c.phi_n += c.ndph * c.step_sc;
            c.dr_prev = dr;
        }
    }
    if (sqrt(c.ndth * c.ndth + c.ndph * c.ndph) * c.step_sc < 1.0e-12) { search_continue(c, S); return; }
    c.n++;
}

}  // namespace
}  // namespace iga

using namespace iga;
using namespace iga_internal;

extern "C" int iga_eig_params_default(iga_atmo_t h, iga_eig_params* p) {
    if (!h || !p) return IGA_E_INVALID;
    memset(p, 0, sizeof(*p));
    // propagation defaults of the handle's own solver (range-dependent: its
    // geometry, region and source at the region's centre)
    int rc = h->kind == 0 ? iga_fan_params_default(h, &p->fan)
                          : iga_fan_params_init(h, h->kind == 1 ? IGA_GEOM_SPH : IGA_GEOM_3D, &p->fan);
    if (rc) return rc;
    p->incl_min = 0.5; p->incl_max = 45.0;
    p->incl_step_min = 0.001; p->incl_step_max = 0.1;
    p->damping = 1.0e-3; p->tolerance = 0.1; p->az_err_lim = 2.0;
    p->bnc_min = 0; p->bnc_max = 0;
    p->iterations = 25;
    p->chunk = 0;
    return IGA_OK;
}

namespace iga_internal {

// The whole search on one stream, results in host vectors (iga_eig_run and
// the request server).  Device scratch is stream-ordered (cudaMallocAsync /
// cudaFreeAsync), so searches on different streams overlap on the GPU.
int eig_search(iga_atmo_s* h, const iga_eig_params* P, const iga_eig_pair* pairs, int n_pairs, cudaStream_t st,
               std::vector<double>& out_rows, std::vector<int>& out_pair, long long& steps_out,
               const EigDirect* direct) {
    out_rows.clear(); out_pair.clear(); steps_out = 0;
    if (!h || !P || n_pairs < 0 || (n_pairs > 0 && !pairs)) return IGA_E_INVALID;
    iga_fan_params fp = P->fan;
    const bool sph = fp.geometry == IGA_GEOM_SPH;
    fp.bounces = 0;
    fp.calc_amp = 1;
    fp.write_rays = 1;
    int rc = validate(&fp, 1);
    if (rc) return rc;
    // range-dependent handles (kind 1 spherical, 2 Cartesian) search in the
    // geometry they were loaded for
    const bool rngdep = h->kind != 0;
    if (rngdep && sph != (h->kind == 1)) {
        g_cuda_err = "range-dependent atmosphere: eigenray search in the geometry it was loaded for";
        return IGA_E_UNSUPPORTED;
    }
    if ((sph || rngdep) && fp.precision != IGA_FP64) {
        g_cuda_err = "spherical and range-dependent eigenray searches: FP64 only";
        return IGA_E_UNSUPPORTED;
    }
    // 18-state traces: spherical and range-dependent solvers
    const bool wide = sph || rngdep;
    if (P->bnc_min < 0 || P->bnc_max < P->bnc_min || P->iterations < 0 || !(P->tolerance > 0.0) ||
        !(P->incl_step_max > 0.0) || !(P->incl_step_min > 0.0) || !(P->incl_max > P->incl_min))
        return IGA_E_INVALID;
    if (n_pairs == 0) return IGA_OK;
    for (int i = 1; i < n_pairs; i++) {
        if (pairs[i].src[2] != pairs[0].src[2]) {
            g_cuda_err = "iga_eig_run: all pairs of one call must share the source altitude";
            return IGA_E_UNSUPPORTED;
        }
        if (rngdep && (pairs[i].src[0] != pairs[0].src[0] || pairs[i].src[1] != pairs[0].src[1])) {
            g_cuda_err = "iga_eig_run: range-dependent searches of one call must share the source";
            return IGA_E_UNSUPPORTED;
        }
    }
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    // the launch arguments carry the source altitude; each trace request
    // carries its own source x, y (latitude, longitude)
    fp.src[0] = (sph || rngdep) ? pairs[0].src[0] : 0.0;
    fp.src[1] = (sph || rngdep) ? pairs[0].src[1] : 0.0;
    fp.src[2] = pairs[0].src[2];
    Fan3DArgs a;
    rc = build_args(h, &fp, a);
    if (rc) return rc;
    double c_incl_src = 0.0;   // spherical find_eigenray: c at radius = source altitude, i.e. the lowest knot
    if (sph && !rngdep) {
        double f, d1, d2;
        iga::spline_eval(h->prof.z, h->prof.c, h->prof.cs, h->prof.z.front(), f, d1, d2);
        c_incl_src = f;
    }
    const bool f32 = fp.precision == IGA_FP32C || fp.precision == IGA_FP32C_FLAGGED;
    if (f32 && (rc = fp32c_setup(h, fp.freq, a))) return rc;

    Settings S;
    S.theta_max = P->incl_max * (kPi / 180.0);
    S.dth_big = P->incl_step_max * (kPi / 180.0);
    S.dth_sml = P->incl_step_min * (kPi / 180.0);
    S.damping = P->damping; S.tolerance = P->tolerance; S.az_err_lim = P->az_err_lim;
    S.rng_max = fp.rng_max; S.iterations = P->iterations; S.chunk = P->chunk;
    S.sph = sph;
    S.r_grnd = a.r_grnd; S.c_src = a.c0; S.c_grnd = a.c_gnd;
    double theta_min = P->incl_min * (kPi / 180.0);
    if (sph) {   // run_eig_search's theta_grnd (main.infraga.sph.cpp:965-981, sph.rngdep the same)
        double theta_grnd;
        if (rngdep && h->has_topo) {
            // over terrain the reference takes the steepest ground slope over
            // azimuths 0, 3, ..., 357 deg plus 0.1, in DEGREES, and compares it
            // with the inclination bounds in radians; kept as written
            double zt, dz[2];
            iga::terrain_eval1(h->topo, a.src_x, a.src_y, zt, dz);
            if (a.src_z - zt < 0.01) {
                theta_grnd = 0.0;
                const double dzgdx = 1.0 / (kEarthRadiusKm * cos(a.src_x)) * dz[1];
                const double dzgdy = 1.0 / kEarthRadiusKm * dz[0];
                for (double pv = 0.0; pv < 360.0; pv += 3.0)
                    theta_grnd = std::max(theta_grnd, atan(dzgdx * sin(pv * kPi / 180.0) + dzgdy * cos(pv * kPi / 180.0)) *
                                                          (180.0 / kPi) + 0.1);
            } else {
                theta_grnd = -89.9 * (kPi / 180.0);
            }
        } else {
            theta_grnd = a.src_z - (a.r_grnd - a.r_earth) < 0.01 ? 0.1 * (kPi / 180.0) : -89.9 * (kPi / 180.0);
        }
        theta_min = std::max(theta_min, theta_grnd);
    }

    std::vector<Chain> chains;
    for (int ip = 0; ip < n_pairs; ip++) {
        for (int nb = P->bnc_min; nb <= P->bnc_max; nb++) {
            Chain c;
            c.pair = ip; c.nb = nb;
            c.sx = pairs[ip].src[0]; c.sy = pairs[ip].src[1];
            c.rx = pairs[ip].rcvr[0]; c.ry = pairs[ip].rcvr[1];
            if (sph) {   // run_eig_search converts degrees (main.infraga.sph.cpp:889-890)
                c.sx *= (kPi / 180.0); c.sy *= (kPi / 180.0);
                c.rx *= (kPi / 180.0); c.ry *= (kPi / 180.0);
                c.rcvr_rng = gc_dist_h(c.sx, c.sy, c.rx, c.ry);
                c.rcvr_az = bearing_h(c.sx, c.sy, c.rx, c.ry);
                c.phi0 = kPi / 2.0 - c.rcvr_az;
            } else {
                c.rcvr_rng = sqrt(pow(c.rx - c.sx, 2) + pow(c.ry - c.sy, 2));
                c.rcvr_az = atan2(c.ry - c.sy, c.rx - c.sx);
                c.phi0 = c.rcvr_az;
            }
            if (direct) {
                c.direct = true;
                newton_begin(c, direct[ip].theta, direct[ip].phi);
            } else if (theta_min < S.theta_max) {
                est_begin(c, S, theta_min);
            } else {
                c.phase = Chain::kDone;
            }
            chains.push_back(std::move(c));
        }
    }

    TraceReq* d_req = nullptr;
    unsigned char* d_res = nullptr;   // TraceRes or TraceRes18 records
    const size_t res_bytes = wide ? sizeof(TraceRes18) : sizeof(TraceRes);
    SegRes* d_seg = nullptr;
    unsigned int* d_q = nullptr;   // request counters of the sweep and the Newton/record launches
    size_t cap_req = 0;
    long long steps_tot = 0;
    const int max_seg = P->bnc_max + 1;
    auto release = [&]() {
        if (d_req) cudaFreeAsync(d_req, st);
        if (d_res) cudaFreeAsync(d_res, st);
        if (d_seg) cudaFreeAsync(d_seg, st);
        if (d_q) cudaFreeAsync(d_q, st);
        d_req = nullptr; d_res = nullptr; d_seg = nullptr; d_q = nullptr;
    };
    cudaEvent_t round_done = nullptr;
    {
        cudaError_t e = cudaEventCreateWithFlags(&round_done, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate(eigen round)");
    }
    auto fail = [&](int code) { release(); cudaEventDestroy(round_done); return code; };

    std::vector<TraceReq> req6, req18;
    std::vector<TraceRes> res18;
    std::vector<TraceRes18> res18s;
    std::vector<SegRes> seg6, seg6s;   // per request (request order) / as traced (launch order)
    std::vector<int> order6;
    std::vector<TraceReq> sorted6;
    // searches of one pair for different bounce counts sweep the same launch
    // angles until their first bracket: one trace serves them all
    std::map<std::array<double, 4>, int> uniq;
    // IGA_EIG_VERBOSE=1: per-call work summary on stderr (diagnostics only)
    const char* vb = getenv("IGA_EIG_VERBOSE");
    const bool verbose = vb != nullptr;
    const bool per_round = vb && vb[0] == '2';
    long long n_rounds = 0, n6 = 0, n18 = 0, st6 = 0, st18 = 0;
    const auto t_begin = std::chrono::steady_clock::now();
    NvtxRange nv_search(direct ? "iga_eig_direct" : "iga_eig_search");
    while (true) {
        NvtxRange nv_round("eig round");
        req6.clear(); req18.clear(); uniq.clear();
        int sweeping = 0;
        for (auto& c : chains) if (c.phase == Chain::kEst && c.iterations < S.fixed_step_iters()) sweeping++;
        int chunk = S.chunk > 0 ? S.chunk : std::max(8, std::min(128, sweeping > 0 ? 262144 / sweeping : 128));
        for (auto& c : chains) {
            // find_eigenray gives up after `iterations` Newton steps
            if (c.phase == Chain::kNewton && c.n >= S.iterations) search_continue(c, S);
            c.sweep.clear();
            c.sweep_req.clear();
            if (c.phase == Chain::kEst) {
                // with a fixed step the next inclinations are known: submit a chunk
                const int m = c.iterations < S.fixed_step_iters() ? chunk : 1;
                double th = c.th;
                for (int j = 0; j < m && S.in_sweep(th, c.th_max); j++) {
                    c.sweep.push_back(th);
                    const std::array<double, 4> key{c.sx, c.sy, th, c.phi};
                    auto it = uniq.find(key);
                    if (it == uniq.end()) {
                        uniq.emplace(key, (int)req6.size());
                        c.sweep_req.push_back((int)req6.size());
                        req6.push_back({c.sx, c.sy, th, c.phi, c.nb + 1, kStopOnEscape});
                    } else {
                        c.sweep_req.push_back(it->second);
                        req6[it->second].n_seg = std::max(req6[it->second].n_seg, c.nb + 1);
                    }
                    th += c.dth;
                }
            } else if (c.phase == Chain::kNewton) {
                c.req0 = (int)req18.size();
                // the 3D find_eigenray follows one reflection at most while iterating
                // (geoac.eigenray.3d.cpp:206); the spherical one all of them
                req18.push_back({c.sx, c.sy, c.theta, c.phi_n, sph ? c.nb + 1 : 1 + std::min(c.nb, 1), kStopOnEscape});
            } else if (c.phase == Chain::kRecordTrace) {
                c.req0 = (int)req18.size();
                req18.push_back({c.sx, c.sy, c.theta, c.phi_n, c.nb + 1, kRecord});
            }
        }
        if (req6.empty() && req18.empty()) break;
        const auto t_round = std::chrono::steady_clock::now();
        const size_t need = std::max(req6.size(), req18.size());
        if (need > cap_req) {
            release();
            cap_req = std::max(need, cap_req * 2);
            cudaError_t e1 = cudaMallocAsync(&d_req, 2 * cap_req * sizeof(TraceReq), st);
            cudaError_t e2 = e1 == cudaSuccess ? cudaMallocAsync(&d_res, 2 * cap_req * res_bytes, st) : e1;
            cudaError_t e3 = e2 == cudaSuccess ? cudaMallocAsync(&d_seg, cap_req * max_seg * sizeof(SegRes), st) : e2;
            if (e3 == cudaSuccess) e3 = cudaMallocAsync(&d_q, 2 * sizeof(unsigned int), st);
            if (e3 != cudaSuccess) return fail(cuda_fail(e3, "cudaMallocAsync(eigen traces)"));
        }
        TraceReq* d_req18 = d_req + cap_req;
        unsigned char* d_res18 = d_res + cap_req * res_bytes;
        cudaError_t e = cudaSuccess;
        // sweep traces go out longest first (more segments first), so the
        // persistent kernel's last requests are short ones
        order6.resize(req6.size());
        for (size_t i = 0; i < order6.size(); i++) order6[i] = (int)i;
        std::stable_sort(order6.begin(), order6.end(), [&](int x, int y) { return req6[x].n_seg > req6[y].n_seg; });
        sorted6.resize(req6.size());
        for (size_t i = 0; i < order6.size(); i++) sorted6[i] = req6[order6[i]];
        if (!req6.empty()) {
            e = cudaMemcpyAsync(d_req, sorted6.data(), sorted6.size() * sizeof(TraceReq), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = h->kind == 1 ? launch_trace_sphr(a, d_req, reinterpret_cast<TraceRes18*>(d_res), (int)req6.size(), false,
                                                     st, d_seg, max_seg, d_q)
                    : h->kind == 2 ? launch_trace_3dr(a, d_req, reinterpret_cast<TraceRes18*>(d_res), (int)req6.size(), false,
                                                      st, d_seg, max_seg, d_q)
                    : sph ? launch_trace_sph(a, d_req, reinterpret_cast<TraceRes18*>(d_res), (int)req6.size(), false, st,
                                           d_seg, max_seg, c_incl_src, d_q)
                    : f32 ? launch_trace_fp32c(a, d_req, reinterpret_cast<TraceRes*>(d_res), (int)req6.size(), false, st,
                                               d_q, d_seg, max_seg)
                          : launch_trace<false>(a, d_req, reinterpret_cast<TraceRes*>(d_res), (int)req6.size(), st, d_q,
                                                d_seg, max_seg);
        }
        if (e == cudaSuccess && !req18.empty()) {
            e = cudaMemcpyAsync(d_req18, req18.data(), req18.size() * sizeof(TraceReq), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = h->kind == 1 ? launch_trace_sphr(a, d_req18, reinterpret_cast<TraceRes18*>(d_res18), (int)req18.size(),
                                                     true, st, nullptr, 0, d_q + 1)
                    : h->kind == 2 ? launch_trace_3dr(a, d_req18, reinterpret_cast<TraceRes18*>(d_res18), (int)req18.size(),
                                                      true, st, nullptr, 0, d_q + 1)
                    : sph ? launch_trace_sph(a, d_req18, reinterpret_cast<TraceRes18*>(d_res18), (int)req18.size(), true,
                                           st, nullptr, 0, c_incl_src, d_q + 1)
                    : f32 ? launch_trace_fp32c(a, d_req18, reinterpret_cast<TraceRes*>(d_res18), (int)req18.size(), true, st,
                                               d_q + 1)
                          : launch_trace<true>(a, d_req18, reinterpret_cast<TraceRes*>(d_res18), (int)req18.size(), st,
                                               d_q + 1);
        }
        seg6.resize(req6.size() * max_seg);
        seg6s.resize(req6.size() * max_seg);
        res18.resize(wide ? 0 : req18.size());
        res18s.resize(wide ? req18.size() : 0);
        if (e == cudaSuccess && !req6.empty())
            e = cudaMemcpyAsync(seg6s.data(), d_seg, seg6s.size() * sizeof(SegRes), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && !req18.empty())
            e = wide ? cudaMemcpyAsync(res18s.data(), d_res18, res18s.size() * sizeof(TraceRes18), cudaMemcpyDeviceToHost, st)
                    : cudaMemcpyAsync(res18.data(), d_res18, res18.size() * sizeof(TraceRes), cudaMemcpyDeviceToHost, st);
        // wait on a blocking-sync event: the host thread sleeps instead of
        // spinning, so concurrent searches (pair groups, server workers) leave
        // the host cores to each other and to the driver
        if (e == cudaSuccess) e = cudaEventRecord(round_done, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(round_done);
        if (e != cudaSuccess) return fail(cuda_fail(e, "eigen trace round"));
        for (size_t i = 0; i < order6.size(); i++)
            std::copy(&seg6s[i * max_seg], &seg6s[i * max_seg] + max_seg, &seg6[(size_t)order6[i] * max_seg]);
        // each search's view of its sweep traces: the entry of its own
        // segment count, or the earlier entry where the trace escaped
        auto sweep_view = [&](int idx, int m, TraceRes& t) {
            const SegRes* g = &seg6[(size_t)idx * max_seg];
            int j = 0;
            while (j < m - 1 && !g[j].escaped) j++;
            t.y[0] = g[j].x; t.y[1] = g[j].y; t.escaped = g[j].escaped; t.steps = g[j].steps;
        };
        long long m6 = 0;
        for (auto& c : chains) {
            if (c.phase != Chain::kEst) continue;
            for (size_t j = 0; j < c.sweep_req.size(); j++) {
                TraceRes t;
                sweep_view(c.sweep_req[j], c.nb + 1, t);
                steps_tot += t.steps; st6 += t.steps;
                m6 = std::max(m6, t.steps);
            }
        }
        for (auto& r : res18) { steps_tot += r.steps; st18 += r.steps; }
        for (auto& r : res18s) { steps_tot += r.steps; st18 += r.steps; }
        n_rounds++; n6 += (long long)req6.size(); n18 += (long long)req18.size();
        if (per_round) {
            long long m18 = 0;
            for (auto& r : res18) m18 = std::max(m18, r.steps);
            for (auto& r : res18s) m18 = std::max(m18, r.steps);
            int n_est = 0, n_newt = 0, n_rec = 0;
            for (auto& c : chains) {
                n_est += c.phase == Chain::kEst;
                n_newt += c.phase == Chain::kNewton;
                n_rec += c.phase == Chain::kRecordTrace;
            }
            fprintf(stderr, "round %lld: sweep %zu (max %lld steps) newton/record %zu (max %lld) chains est %d newton %d "
                            "record %d chunk %d %.4f s\n",
                    n_rounds, req6.size(), m6, req18.size(), m18, n_est, n_newt, n_rec, chunk,
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - t_round).count());
        }

        for (auto& c : chains) {
            if (c.phase == Chain::kEst && !c.sweep.empty()) {
                for (size_t j = 0; j < c.sweep.size(); j++) {
                    TraceRes t;
                    sweep_view(c.sweep_req[j], c.nb + 1, t);
                    if (est_step(c, S, t)) break;
                }
            } else if (c.phase == Chain::kNewton) {
                if (sph) newton_step_sph(c, S, res18s[c.req0]);
                else if (rngdep) newton_step_3dr(c, S, res18s[c.req0]);
                else newton_step(c, S, a, res18[c.req0]);
            } else if (c.phase == Chain::kRecordTrace && sph) {
                // eig_results row of geoac.eigenray.sph.cpp:303-315
                const TraceRes18& t = res18s[c.req0];
                std::vector<double> row(IGA_ARRIVAL_COLS);
                row[0] = c.theta * (180.0 / kPi);
                row[1] = 90.0 - c.phi_n * (180.0 / kPi);
                row[2] = c.nb;
                row[3] = t.y[1] * 180.0 / kPi;
                row[4] = t.y[2] * 180.0 / kPi;
                row[5] = t.tt;
                row[6] = gc_dist_h(t.y[1], t.y[2], c.sx, c.sy) / t.tt;
                row[7] = t.zmax;
                row[8] = t.incl;
                row[9] = t.baz;
                row[10] = t.amp_db;
                row[11] = -2.0 * t.att;
                c.rows.push_back(std::move(row));
                search_continue(c, S);
            } else if (c.phase == Chain::kRecordTrace && rngdep) {
                // eig_results row of geoac.eigenray.3d.cpp:296-308, 18-state layout
                const TraceRes18& t = res18s[c.req0];
                std::vector<double> row(IGA_ARRIVAL_COLS);
                row[0] = c.theta * (180.0 / kPi);
                row[1] = 90.0 - c.phi_n * (180.0 / kPi);
                row[2] = c.nb;
                row[3] = t.y[0];
                row[4] = t.y[1];
                row[5] = t.tt;
                row[6] = sqrt(pow(t.y[0] - c.sx, 2) + pow(t.y[1] - c.sy, 2)) / t.tt;
                row[7] = t.zmax;
                row[8] = t.incl;
                row[9] = t.baz;
                row[10] = t.amp_db;
                row[11] = -2.0 * t.att;
                c.rows.push_back(std::move(row));
                search_continue(c, S);
            } else if (c.phase == Chain::kRecordTrace) {
                const TraceRes& t = res18[c.req0];
                std::vector<double> row(IGA_ARRIVAL_COLS);
                row[0] = c.theta * (180.0 / kPi);
                row[1] = 90.0 - c.phi_n * (180.0 / kPi);
                row[2] = c.nb;
                row[3] = t.y[0];
                row[4] = t.y[1];
                row[5] = t.tt;
                row[6] = sqrt(pow(t.y[0] - c.sx, 2) + pow(t.y[1] - c.sy, 2)) / t.tt;
                row[7] = t.zmax;
                row[8] = t.incl;
                row[9] = t.baz;
                row[10] = t.amp_db;
                row[11] = -2.0 * t.att;
                c.rows.push_back(std::move(row));
                search_continue(c, S);
            }
        }
    }
    release();
    cudaEventDestroy(round_done);
    if (verbose) {
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_begin).count();
        fprintf(stderr, "eig_search: %zu chains, %lld rounds, sweep traces %lld (%lld steps), "
                        "newton/record traces %lld (%lld steps), %.3f s\n",
                chains.size(), n_rounds, n6, st6, n18, st18, secs);
    }
    for (auto& c : chains) {
        for (auto& row : c.rows) {
            out_rows.insert(out_rows.end(), row.begin(), row.end());
            out_pair.push_back(c.pair);
        }
    }
    steps_out = steps_tot;
    return IGA_OK;
}

}  // namespace iga_internal

extern "C" int iga_eig_direct(iga_atmo_t h, const iga_eig_params* P, const iga_eig_pair* pair, double incl_est,
                              double az_est, int bounces, double* eigenray, int* found, long long* total_steps) {
    if (!h || !P || !pair || !found || bounces < 0) return IGA_E_INVALID;
    *found = 0;
    if (total_steps) *total_steps = 0;
    iga_eig_params q = *P;
    q.bnc_min = q.bnc_max = bounces;
    EigDirect d{incl_est * (kPi / 180.0), kPi / 2.0 - az_est * (kPi / 180.0)};
    std::vector<double> rows;
    std::vector<int> pidx;
    long long steps = 0;
    int rc = eig_search(h, &q, pair, 1, h->stream, rows, pidx, steps, &d);
    if (rc) return rc;
    if (!pidx.empty()) {
        *found = 1;
        if (eigenray) memcpy(eigenray, rows.data(), IGA_ARRIVAL_COLS * sizeof(double));
    }
    if (total_steps) *total_steps = steps;
    return IGA_OK;
}

namespace {

// Searches of different pairs are independent: pair groups can run
// concurrently, each on its own host thread and stream, so that their rounds
// overlap on the GPU.  Pairs are dealt round-robin (uneven pairs spread over
// the groups); the rows are merged back in pair order.
int eig_search_groups(iga_atmo_s* h, const iga_eig_params* P, const iga_eig_pair* pairs, int n_pairs, int groups,
                      std::vector<double>& rows, std::vector<int>& pidx, long long& steps) {
    rows.clear(); pidx.clear(); steps = 0;
    if (groups <= 1) return eig_search(h, P, pairs, n_pairs, h->stream, rows, pidx, steps);
    struct Part {
        std::vector<int> idx;
        std::vector<iga_eig_pair> pairs;
        std::vector<double> rows;
        std::vector<int> pidx;
        long long steps = 0;
        int rc = IGA_OK;
        std::string err;
    };
    std::vector<Part> parts(groups);
    for (int i = 0; i < n_pairs; i++) {
        parts[i % groups].idx.push_back(i);
        parts[i % groups].pairs.push_back(pairs[i]);
    }
    std::vector<std::thread> threads;
    for (int g = 0; g < groups; g++) {
        threads.emplace_back([&, g]() {
            Part& pt = parts[g];
            cudaStream_t s = nullptr;
            cudaError_t e = cudaSetDevice(h->device);
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (e != cudaSuccess) {
                pt.rc = cuda_fail(e, "eigen search stream");
            } else {
                pt.rc = eig_search(h, P, pt.pairs.data(), (int)pt.pairs.size(), s, pt.rows, pt.pidx, pt.steps);
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
            if (pt.rc) pt.err = g_cuda_err;
        });
    }
    for (auto& t : threads) t.join();
    for (auto& pt : parts)
        if (pt.rc) {
            g_cuda_err = pt.err;
            return pt.rc;
        }
    // merge in pair order (within a pair the group kept the search order)
    std::vector<std::vector<std::pair<int, int>>> by_pair(n_pairs);   // (group, row)
    for (int g = 0; g < groups; g++) {
        steps += parts[g].steps;
        for (size_t r = 0; r < parts[g].pidx.size(); r++) by_pair[parts[g].idx[parts[g].pidx[r]]].push_back({g, (int)r});
    }
    for (int i = 0; i < n_pairs; i++)
        for (auto& gr : by_pair[i]) {
            const double* src = &parts[gr.first].rows[(size_t)gr.second * IGA_ARRIVAL_COLS];
            rows.insert(rows.end(), src, src + IGA_ARRIVAL_COLS);
            pidx.push_back(i);
        }
    return IGA_OK;
}

}  // namespace

extern "C" int iga_eig_run(iga_atmo_t h, const iga_eig_params* P, const iga_eig_pair* pairs, int n_pairs,
                           double* eigenrays, int cap, int* n_out, int* pair_index, long long* total_steps) {
    if (!h || !P || !n_out || n_pairs < 0 || (n_pairs > 0 && !pairs) || (cap > 0 && !eigenrays)) return IGA_E_INVALID;
    *n_out = 0;
    if (total_steps) *total_steps = 0;
    if (P->streams < 0) return IGA_E_INVALID;
    std::vector<double> rows;
    std::vector<int> pidx;
    long long steps = 0;
    // automatic: one group.  Measured on a config-3 seed (128 pairs, 0-8 bounces),
    // 4 and 16 concurrent groups took 1.8x and 3.8x longer than one: the rounds'
    // big sweep launches already fill the GPU, and concurrent launches only
    // stretch each other's longest trace
    int groups = P->streams > 0 ? P->streams : 1;
    groups = std::max(1, std::min(groups, n_pairs));
    int rc = eig_search_groups(h, P, pairs, n_pairs, groups, rows, pidx, steps);
    if (rc) return rc;
    const int w = (int)pidx.size();
    for (int i = 0; i < w && i < cap; i++) {
        memcpy(eigenrays + (size_t)i * IGA_ARRIVAL_COLS, &rows[(size_t)i * IGA_ARRIVAL_COLS], IGA_ARRIVAL_COLS * sizeof(double));
        if (pair_index) pair_index[i] = pidx[i];
    }
    *n_out = w;
    if (total_steps) *total_steps = steps;
    return w > cap ? IGA_E_TRUNCATED : IGA_OK;
}
