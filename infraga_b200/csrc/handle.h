// Internal (not part of the C ABI): the atmosphere handle and helpers shared
// by the C ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/infraga_gpu.h"
#include "atmo_host.h"
#include "atmo_rngdep.h"
#include "fan3d.cuh"

using iga::StratProfile;

struct iga_atmo_s {
    int device = 0;
    // 0: stratified profile (prof); 1: spherical range-dependent grid (grid,
    // optional topo); 2: 3D range-dependent grid (grid, optional topo), or with
    // strat_topo a stratified profile (prof, d_knots) over terrain (topo)
    int kind = 0;
    bool strat_topo = false;
    StratProfile prof;        // range-dependent: z only (knot altitudes)
    iga::RngdepGrid grid;
    iga::Terrain topo;
    bool has_topo = false;
    double* d_hyb = nullptr;  // hybrid node records, then node lat, lon, z
    float* d_hyb_x32 = nullptr;   // FP32 second-derivative blocks of the hybrid records (FP32C)
    double* d_topo = nullptr; // terrain node records, then node lat, lon
    double* d_knots = nullptr;
    // stream of the host-buffer entry points: one per handle, so calls on
    // different atmospheres from different host threads overlap on the GPU
    cudaStream_t stream = nullptr;
    // reusable device buffers of the host-buffer entry points
    std::mutex mu;
    void* d_buf = nullptr;
    size_t d_buf_bytes = 0;
    // FP32-compensated path: FP32 knot table and alpha(z) tables per frequency
    double* d_knots_c = nullptr;   // power-basis FP64 table of the FP32-compensated kernels
    std::mutex alpha_mu;
    struct AlphaTab { float* d = nullptr; int n = 0; double z0 = 0.0, inv_h = 0.0; };
    std::map<double, AlphaTab> alpha;   // kept until destroy (launches may still read them)
};

namespace iga_internal {
extern thread_local std::string g_cuda_err;
extern thread_local std::string g_err;
int cuda_fail(cudaError_t e, const char* what);
int validate(const iga_fan_params* p, int n_rays);
int build_args(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a);
// Device buffers of the sampled per-step output (Fan3DArgs path_* / caus_*).
struct PathSpec {
    double* rows = nullptr;
    const long long* off = nullptr;
    long long* n = nullptr;
    int mode = 0;
    double* caus = nullptr;
    unsigned long long* caus_count = nullptr;
    long long caus_cap = 0;
};
// iga_fan_run_device with an optional CTA cap (0 = none), for the request
// server, and optional sampled per-step output (paths.cu)
int fan_device(iga_atmo_s* h, const iga_fan_params* p, const double* d_th, const double* d_ph, int n_rays,
               double* d_arr, int* d_n, long long* d_steps, int* d_status, double* d_aux, void* d_ws,
               cudaStream_t st, int grid_cap, const PathSpec* paths = nullptr);
// FP32 knot table and alpha(z) table of `freq` into the launch arguments
int fp32c_setup(iga_atmo_s* h, double freq, iga::Fan3DArgs& a);
// Launch estimate of find_eigenray alone (run_eig_direct): radians, the
// reference's internal azimuth convention (phi = pi/2 - azimuth).
struct EigDirect {
    double theta, phi;
};
// the eigenray search on one stream (eig3d.cu); with `direct` (one entry per
// pair) only the Newton refinement runs, for bounce count P->bnc_min
int eig_search(iga_atmo_s* h, const iga_eig_params* P, const iga_eig_pair* pairs, int n_pairs, cudaStream_t st,
               std::vector<double>& out_rows, std::vector<int>& out_pair, long long& steps_out,
               const EigDirect* direct = nullptr);
}  // namespace iga_internal

#define IGA_CUDA(call, what)                                                  \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return iga_internal::cuda_fail(e_, what);      \
    } while (0)
