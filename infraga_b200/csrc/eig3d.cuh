// Ray-trace requests of the eigenray search (eig3d.cu) and the trace kernels
// that serve them: FP64 (eig3d.cu) and FP32-compensated (fan3d_fp32c.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

#include "fan3d.cuh"

namespace iga {

// Grid of a persistent trace launch: every SM filled at the kernel's
// occupancy, fewer CTAs when the requests do not need them.  The trace
// kernels take requests from a device counter (queue, zeroed on the stream
// before the launch), so each thread traces until the requests run out.
template <class Kern>
inline cudaError_t trace_grid(Kern kern, int threads, size_t smem, int n, int& grid) {
    int dev = 0, n_sm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess) return e;
    const long long want = ((long long)n + threads - 1) / threads;
    const long long cap = (long long)n_sm * (per_sm > 0 ? per_sm : 1);
    grid = (int)std::max(1LL, std::min(want, cap));
    return cudaSuccess;
}

struct TraceReq {
    double x0, y0;       // source position
    double theta, phi;   // launch angles [rad] (geoac::theta, geoac::phi)
    int n_seg;           // prop_rk4 segments to trace (bounces + 1)
    int flags;
};
enum : int { kStopOnEscape = 1, kRecord = 2 };

struct TraceRes {
    double y[12];        // state at the last row (12-state layout)
    double rc[6];        // nu_x, nu_y, mu_th_x, mu_th_y, mu_ph_x, mu_ph_y
    double tt, att, zmax, amp_db, incl, baz;
    long long steps;
    int escaped;         // the last traced segment left the region
    int pad;
};

// Per-segment result of a sweep trace: the last row of segment j (or the
// row where the trace escaped), the steps so far and whether it escaped.
// Sweep requests of several searches that share a launch (same source and
// launch angles, different bounce counts) are traced once with the largest
// segment count; each search reads the entry of its own count.
struct SegRes {
    double x, y;
    long long steps;
    int escaped;
    int pad;
};

// Result of a trace in the full 18-state layout (spherical: r, lat, lon,
// nu, X_th, mu_th, X_ph, mu_ph; 3D range-dependent: x, y, z, nu, ...): the
// last row; in record mode the arrival columns find_eigenray forms on the
// device; after an amplitude trace the ground under the last row that
// find_eigenray's Newton derivatives use (sound speeds at the source and on
// the ground, the ground height -- a radius in the spherical layout -- and
// its gradient).
struct TraceRes18 {
    double y[18];
    double tt, att, zmax, amp_db, incl, baz;
    double c_src, c_grnd, z_grnd, dzg[2];
    double pad_d;
    long long steps;
    int escaped;
    int pad;
};

// Spherical stratified traces (eigsph.cu); source latitude/longitude per
// request (x0, y0, radians), altitude from the launch arguments.
// c_incl_src is the sound speed find_eigenray divides by in its arrival
// inclination.
cudaError_t launch_trace_sph(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                             cudaStream_t st, SegRes* seg_out, int seg_stride, double c_incl_src,
                             unsigned int* d_queue);

// Range-dependent traces with terrain (fan3dr_fp64.cu, fansphr_fp64.cu): the
// source is the launch arguments' (all requests of a launch share it).
cudaError_t launch_trace_3dr(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                             cudaStream_t st, SegRes* seg_out, int seg_stride, unsigned int* d_queue);
cudaError_t launch_trace_sphr(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                              cudaStream_t st, SegRes* seg_out, int seg_stride, unsigned int* d_queue);

// FP32-compensated traces (same contract as the FP64 trace kernel).  With
// seg_out != null, segment j of request r also writes seg_out[r * seg_stride + j].
cudaError_t launch_trace_fp32c(const Fan3DArgs& a, const TraceReq* d_req, TraceRes* d_res, int n, bool amp,
                               cudaStream_t st, unsigned int* d_queue, SegRes* seg_out = nullptr, int seg_stride = 0);

}  // namespace iga
