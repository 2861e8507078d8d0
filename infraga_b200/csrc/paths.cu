// iga_fan_paths: sampled per-step rows (raypaths, terrain samples) and
// caustic points of a fan, the output of run_prop's write_rays, write_topo
// and write_caustics branches (src/main.infraga.3d.cpp:443-497 and the
// same blocks of the spherical and range-dependent mains).
//
// The fan kernels write a ray's sampled rows into a row range reserved from
// its step count (one step-count pass first when the caller has none), so
// rows land in ray order without a sort; caustic points are rare and are
// appended through one counter, then put in ray / step order on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "handle.h"

using namespace iga_internal;

namespace {

// cudaMalloc'd scratch freed on scope exit (this entry point serves the
// command-line front ends, not the hot path).
struct DevMem {
    std::vector<void*> ptrs;
    ~DevMem() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    int get(T** out, size_t count) {
        void* p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(paths)");
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return IGA_OK;
    }
};

struct StreamGuard {
    cudaStream_t st = nullptr;
    ~StreamGuard() {
        if (st) cudaStreamDestroy(st);
    }
};

}  // namespace

extern "C" int iga_fan_paths(iga_atmo_t h, const iga_fan_params* p, const double* theta_deg, const double* phi_deg,
                             int n_rays, int path_mode, const long long* ray_steps, double* path_rows,
                             long long path_cap, long long* n_path, long long* path_start, double* caustic_rows,
                             long long caustic_cap, long long* n_caustic, int* caustic_ray) {
    if (!h || !p) return IGA_E_INVALID;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    if (path_mode != IGA_PATH_RAYS && path_mode != IGA_PATH_TERRAIN && path_mode != IGA_PATH_PROJ &&
        path_mode != IGA_PATH_RESID)
        return IGA_E_INVALID;
    if (n_rays > 0 && (!theta_deg || !phi_deg)) return IGA_E_INVALID;
    const bool want_path = path_rows != nullptr || n_path != nullptr;
    const bool want_caus = caustic_rows != nullptr || n_caustic != nullptr;
    if ((path_rows && !n_path) || (caustic_rows && !n_caustic)) return IGA_E_INVALID;
    if (path_cap < 0 || caustic_cap < 0 || (path_cap > 0 && !path_rows) || (caustic_cap > 0 && !caustic_rows))
        return IGA_E_INVALID;
    if (want_caus && !p->calc_amp) {
        g_err = "caustics need calc_amp = 1";
        return IGA_E_INVALID;
    }
    if (p->precision != IGA_FP64) return IGA_E_UNSUPPORTED;
    if (path_mode == IGA_PATH_PROJ) {   // run_back_proj of infraga-3d (flat ground) and infraga-3d-rngdep
        if (want_caus || !p->calc_amp) return IGA_E_INVALID;
        if (!(h->kind == 0 || h->kind == 2) || p->geometry != IGA_GEOM_3D || (h->kind == 0 && h->has_topo)) {
            g_err = "back projection rows: 3D stratified flat-ground or 3D range-dependent atmospheres only";
            return IGA_E_UNSUPPORTED;
        }
    }
    if (path_mode == IGA_PATH_RESID) {   // print_resid exists here for the 3D stratified flat-ground solver
        if (want_caus) return IGA_E_INVALID;
        if (h->kind != 0 || p->geometry != IGA_GEOM_3D) {
            g_err = "residual rows: 3D stratified flat-ground atmospheres only";
            return IGA_E_UNSUPPORTED;
        }
    }
    const int pcols = iga::path_cols(path_mode);           // device row width
    const int ucols = path_mode == IGA_PATH_PROJ ? IGA_PROJ_COLS : IGA_PATH_COLS;   // caller's row width
    if (n_path) *n_path = 0;
    if (n_caustic) *n_caustic = 0;
    if (path_start) std::fill(path_start, path_start + n_rays + 1, 0LL);
    if (n_rays == 0 || (!want_path && !want_caus)) return IGA_OK;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");

    iga_fan_params q = *p;
    q.write_rays = 1;
    const int nb = q.bounces + 1;
    const size_t n = (size_t)n_rays;
    StreamGuard sg;
    IGA_CUDA(cudaStreamCreateWithFlags(&sg.st, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaStream_t st = sg.st;

    DevMem mem;
    double *d_th, *d_ph, *d_arr;
    int *d_n;
    long long* d_steps;
    void* d_ws;
    if ((rc = mem.get(&d_th, n)) || (rc = mem.get(&d_ph, n)) || (rc = mem.get(&d_arr, n * nb * IGA_ARRIVAL_COLS)) ||
        (rc = mem.get(&d_n, n)) || (rc = mem.get(&d_steps, n)) ||
        (rc = mem.get(reinterpret_cast<unsigned char**>(&d_ws), iga_fan_workspace_bytes())))
        return rc;
    IGA_CUDA(cudaMemcpyAsync(d_th, theta_deg, sizeof(double) * n, cudaMemcpyHostToDevice, st), "H2D theta");
    IGA_CUDA(cudaMemcpyAsync(d_ph, phi_deg, sizeof(double) * n, cudaMemcpyHostToDevice, st), "H2D phi");

    // step counts (the 6 ray equations do not depend on the auxiliaries, so
    // the count pass runs without them)
    std::vector<long long> steps(n);
    if (ray_steps) {
        std::copy(ray_steps, ray_steps + n, steps.begin());
    } else {
        iga_fan_params c = q;
        c.calc_amp = 0;
        rc = fan_device(h, &c, d_th, d_ph, n_rays, d_arr, d_n, d_steps, nullptr, nullptr, d_ws, st, 0);
        if (rc) return rc;
        IGA_CUDA(cudaMemcpyAsync(steps.data(), d_steps, sizeof(long long) * n, cudaMemcpyDeviceToHost, st), "D2H steps");
        IGA_CUDA(cudaStreamSynchronize(st), "step-count pass");
    }

    std::vector<long long> off(n + 1, 0);
    long long total_steps = 0;
    for (size_t i = 0; i < n; i++) {
        if (steps[i] < 0) return IGA_E_INVALID;
        off[i + 1] = off[i] + (want_path ? iga::path_rows_bound(path_mode, steps[i], nb) : 0);
        total_steps += steps[i];
    }
    iga_internal::PathSpec ps;
    ps.mode = path_mode;
    long long* d_off = nullptr;
    if (want_path) {
        if ((rc = mem.get(&ps.rows, (size_t)off[n] * pcols)) || (rc = mem.get(&d_off, n + 1)) ||
            (rc = mem.get(&ps.n, n)))
            return rc;
        ps.off = d_off;
        IGA_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice, st), "H2D offsets");
    }
    double* d_caus = nullptr;
    unsigned long long* d_cc = nullptr;
    long long ccap = 0;
    auto run = [&]() -> int {
        if (want_caus) {
            ps.caus = d_caus; ps.caus_count = d_cc; ps.caus_cap = ccap;
            IGA_CUDA(cudaMemsetAsync(d_cc, 0, sizeof(unsigned long long), st), "memset caustic counter");
        }
        return fan_device(h, &q, d_th, d_ph, n_rays, d_arr, d_n, d_steps, nullptr, nullptr, d_ws, st, 0, &ps);
    };
    if (want_caus) {
        ccap = std::max<long long>(4096, std::min<long long>(total_steps, 16LL * nb * n_rays));
        if ((rc = mem.get(&d_caus, (size_t)ccap * iga::kCausCols)) || (rc = mem.get(&d_cc, 1))) return rc;
    }
    if ((rc = run())) return rc;
    unsigned long long caus_total = 0;
    if (want_caus) {
        IGA_CUDA(cudaMemcpyAsync(&caus_total, d_cc, sizeof(caus_total), cudaMemcpyDeviceToHost, st), "D2H caustic count");
        IGA_CUDA(cudaStreamSynchronize(st), "paths kernel");
        if ((long long)caus_total > ccap) {   // rare: rerun with room for all of them
            ccap = (long long)caus_total;
            if ((rc = mem.get(&d_caus, (size_t)ccap * iga::kCausCols))) return rc;
            if ((rc = run())) return rc;
        }
    }

    std::vector<long long> pn;
    std::vector<double> rows;
    if (want_path) {
        pn.resize(n);
        rows.resize((size_t)off[n] * pcols);
        IGA_CUDA(cudaMemcpyAsync(pn.data(), ps.n, sizeof(long long) * n, cudaMemcpyDeviceToHost, st), "D2H path counts");
        IGA_CUDA(cudaMemcpyAsync(rows.data(), ps.rows, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "D2H path rows");
    }
    std::vector<double> crows(want_caus ? (size_t)caus_total * iga::kCausCols : 0);
    if (!crows.empty())
        IGA_CUDA(cudaMemcpyAsync(crows.data(), d_caus, crows.size() * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "D2H caustic rows");
    IGA_CUDA(cudaStreamSynchronize(st), "paths kernel");

    bool trunc = false;
    if (want_path) {
        long long w = 0;
        for (size_t i = 0; i < n; i++) {
            if (pn[i] > off[i + 1] - off[i]) {
                g_err = "path rows exceeded the bound from the step count (ray_steps from another fan?)";
                return IGA_E_INVALID;
            }
            if (path_start) path_start[i] = w;
            for (long long j = 0; j < pn[i]; j++, w++)
                if (w < path_cap)
                    memcpy(path_rows + (size_t)w * ucols, &rows[(size_t)(off[i] + j) * pcols], sizeof(double) * ucols);
        }
        if (path_start) path_start[n] = w;
        *n_path = w;
        trunc |= w > path_cap;
    }
    if (want_caus) {
        std::vector<size_t> ord(caus_total);
        std::iota(ord.begin(), ord.end(), size_t(0));
        auto key = [&](size_t r, int c) { return crows[r * iga::kCausCols + c]; };
        std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
            if (key(x, 5) != key(y, 5)) return key(x, 5) < key(y, 5);
            return key(x, 6) < key(y, 6);
        });
        for (size_t w = 0; w < ord.size(); w++) {
            if ((long long)w >= caustic_cap) break;
            const double* r = &crows[ord[w] * iga::kCausCols];
            memcpy(caustic_rows + w * IGA_CAUSTIC_COLS, r, sizeof(double) * IGA_CAUSTIC_COLS);
            if (caustic_ray) caustic_ray[w] = (int)r[5];
        }
        *n_caustic = (long long)caus_total;
        trunc |= (long long)caus_total > caustic_cap;
    }
    return trunc ? IGA_E_TRUNCATED : IGA_OK;
}
