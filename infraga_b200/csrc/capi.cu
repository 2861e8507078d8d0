// C ABI of libinfraga_gpu.so (declared in include/infraga_gpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/infraga_gpu.h"
#include "atmo_host.h"
#include "fan3d.cuh"

using iga::StratProfile;

#include "handle.h"
#include "nvtx.h"

namespace iga_internal {
thread_local std::string g_cuda_err;
thread_local std::string g_err;

int cuda_fail(cudaError_t e, const char* what) {
    g_cuda_err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return IGA_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return IGA_E_NODEVICE;
    return IGA_E_CUDA;
}
}  // namespace iga_internal

using namespace iga_internal;

namespace {

int upload(iga_atmo_s* h) {
    int dev;
    IGA_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    h->device = dev;
    const size_t bytes = h->prof.table.size() * sizeof(double);
    IGA_CUDA(cudaMalloc(&h->d_knots, bytes), "cudaMalloc(knots)");
    IGA_CUDA(cudaMemcpy(h->d_knots, h->prof.table.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(knots)");
    IGA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    // Power-basis segment rows of the FP32-compensated kernels: z_k, 1/dz,
    // then for c, u, v the coefficients of the Hermite cubic written as
    // f = a0 + a1 X + a2 X^2 + a3 X^3 (X = (z - z_k)/dz).  With
    // A = s0 dx - df and B = -s1 dx + df (interpolation.cpp:213-221):
    // a1 = df + A = s0 dx, a2 = B - 2A, a3 = A - B; one row per evaluation
    // instead of the two knot rows the Hermite form reads.
    const StratProfile& P = h->prof;
    const size_t n = P.z.size();
    std::vector<double> tc(n * iga::kStrideC, 0.0);
    const std::vector<double>* fv[3] = {&P.c, &P.u, &P.v};
    const std::vector<double>* sv[3] = {&P.cs, &P.us, &P.vs};
    for (size_t k = 0; k < n; k++) {
        double* o = &tc[k * iga::kStrideC];
        o[0] = P.z[k];
        if (k + 1 == n) break;
        const double dx = P.z[k + 1] - P.z[k];
        o[1] = 1.0 / dx;
        for (int f = 0; f < 3; f++) {
            const double f0 = (*fv[f])[k], f1 = (*fv[f])[k + 1];
            const double s0 = (*sv[f])[k], s1 = (*sv[f])[k + 1];
            const double df = f1 - f0, A = s0 * dx - df, B = -s1 * dx + df;
            o[2 + 4 * f] = f0;
            o[3 + 4 * f] = s0 * dx;
            o[4 + 4 * f] = B - 2.0 * A;
            o[5 + 4 * f] = A - B;
        }
    }
    IGA_CUDA(cudaMalloc(&h->d_knots_c, tc.size() * sizeof(double)), "cudaMalloc(knots_c)");
    IGA_CUDA(cudaMemcpy(h->d_knots_c, tc.data(), tc.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(knots_c)");
    return IGA_OK;
}

// terrain node records, then node x (lat), y (lon)
int upload_terrain(iga_atmo_s* h) {
    if (!h->has_topo) return IGA_OK;
    const iga::Terrain& t = h->topo;
    std::vector<double> tb(t.table);
    tb.insert(tb.end(), t.x.begin(), t.x.end());
    tb.insert(tb.end(), t.y.begin(), t.y.end());
    IGA_CUDA(cudaMalloc(&h->d_topo, tb.size() * sizeof(double)), "cudaMalloc(terrain)");
    IGA_CUDA(cudaMemcpy(h->d_topo, tb.data(), tb.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(terrain)");
    return IGA_OK;
}

int upload_rngdep(iga_atmo_s* h) {
    int dev;
    IGA_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    h->device = dev;
    const iga::RngdepGrid& g = h->grid;
    h->prof.z = g.z;   // knot altitudes (limits and defaults)
    std::vector<double> buf(g.table);
    buf.insert(buf.end(), g.x.begin(), g.x.end());
    buf.insert(buf.end(), g.y.begin(), g.y.end());
    buf.insert(buf.end(), g.z.begin(), g.z.end());
    IGA_CUDA(cudaMalloc(&h->d_hyb, buf.size() * sizeof(double)), "cudaMalloc(hybrid tables)");
    IGA_CUDA(cudaMemcpy(h->d_hyb, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy(hybrid)");
    {   // FP32 copies of the second-derivative blocks (c, u, v) for the FP32C kernel
        const size_t n_rec = (size_t)g.nx * g.ny * g.nz;
        std::vector<float> x32(n_rec * iga::kHybX32, 0.0f);
        for (size_t r = 0; r < n_rec; r++)
            for (int k = 0; k < 3 * iga::kHybX; k++)
                x32[r * iga::kHybX32 + k] = (float)g.table[r * iga::kHybRec + iga::kHybXOff + k];
        IGA_CUDA(cudaMalloc(&h->d_hyb_x32, x32.size() * sizeof(float)), "cudaMalloc(hybrid FP32 blocks)");
        IGA_CUDA(cudaMemcpy(h->d_hyb_x32, x32.data(), x32.size() * sizeof(float), cudaMemcpyHostToDevice),
                 "cudaMemcpy(hybrid FP32 blocks)");
    }
    int rc = upload_terrain(h);
    if (rc) return rc;
    IGA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    return IGA_OK;
}

// Sutherland-Bass alpha(z) for one frequency on a 10 m grid spanning the
// profile plus 2 km either side, evaluated in FP64 with the reference's model
// (c and rho from the profile splines, clamped like atmo::c/rho; the gas
// polynomials at the unclamped z) and stored as FP32 for the FP32C kernel.
constexpr double kAlphaStepKm = 0.01;

int ensure_alpha(iga_atmo_s* h, double freq, iga_atmo_s::AlphaTab& out) {
    std::lock_guard<std::mutex> lock(h->alpha_mu);
    auto it = h->alpha.find(freq);
    if (it != h->alpha.end()) { out = it->second; return IGA_OK; }
    const StratProfile& P = h->prof;
    const double z0 = P.z.front() - 2.0, z1 = P.z.back() + 2.0;
    const int n = (int)std::ceil((z1 - z0) / kAlphaStepKm) + 1;
    iga::SBConst sb{std::pow(10.0, -0.67887), std::pow(10.0, -0.10744), std::pow(10.0, -3.3979)};
    std::vector<float> tab(n);
    for (int i = 0; i < n; i++) {
        const double z = z0 + i * kAlphaStepKm;
        double c, rho, d1, d2;
        iga::spline_eval(P.z, P.c, P.cs, z, c, d1, d2);
        iga::spline_eval(P.z, P.rho, P.rhos, z, rho, d1, d2);
        tab[i] = (float)iga::sb_alpha_cart(c, rho, z, freq, 1.0, sb);
    }
    iga_atmo_s::AlphaTab t;
    t.n = n; t.z0 = z0; t.inv_h = 1.0 / kAlphaStepKm;
    IGA_CUDA(cudaMalloc(&t.d, n * sizeof(float)), "cudaMalloc(alpha)");
    const cudaError_t ce = cudaMemcpy(t.d, tab.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) {
        cudaFree(t.d);   // not yet owned by the handle
        return cuda_fail(ce, "cudaMemcpy(alpha)");
    }
    h->alpha[freq] = t;
    out = t;
    return IGA_OK;
}

// Boundary-layer scaling and its z-derivative at altitude z over flat ground
// z0 (topo::bndlyr_sc / bndlyr_dsc, atmo_state.3d.strat.cpp:85-109).
void bl_host(double z, double z0, double bl, double& sc, double& dsc_z) {
    sc = 1.0; dsc_z = 0.0;
    if (z < z0 + 2.0) {
        const double X = std::exp(-(z - z0) / bl);
        sc = (1.0 - X) / (1.0 + X);
        dsc_z = -2.0 * (-X / bl) / std::pow(1.0 + X, 2);
    }
}

}  // namespace

namespace iga_internal {

int validate(const iga_fan_params* p, int n_rays) {
    if (!p || n_rays < 0) return IGA_E_INVALID;
    if (p->geometry != IGA_GEOM_3D && p->geometry != IGA_GEOM_SPH) return IGA_E_INVALID;
    if (p->precision != IGA_FP64 && p->precision != IGA_FP32C && p->precision != IGA_FP32C_FLAGGED)
        return IGA_E_INVALID;
    if (p->geometry == IGA_GEOM_SPH) {
        if (!(std::fabs(p->src[0]) < 90.0) || !std::isfinite(p->src[1])) return IGA_E_INVALID;
        if (!(p->time_max > 0.0)) return IGA_E_INVALID;
    }
    if (p->bounces < 0 || !(p->ds_min > 0.0) || !(p->ds_max >= p->ds_min) || !(p->s_max > 0.0)) return IGA_E_INVALID;
    if (!std::isfinite(p->s_max / p->ds_min) || p->s_max / p->ds_min > 2.0e9) return IGA_E_INVALID;
    if (!(p->freq > 0.0) || !(p->tweak_abs >= 0.0)) return IGA_E_INVALID;
    for (int i = 0; i < 3; i++) if (!std::isfinite(p->src[i])) return IGA_E_INVALID;
    if (p->block != 0 && (p->block < 32 || p->block > 128 || p->block % 32 != 0)) return IGA_E_INVALID;
    return IGA_OK;
}

// Spherical launch constants (set_initial, set_refl, break_check and the
// atmo:: accessors of atmo_state.sph.strat.cpp evaluated at the source and the
// ground point with the reference's own r -> z arithmetic).
int build_args_sph(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    const StratProfile& P = h->prof;
    const double d2r = iga::kPi / 180.0;
    a.r_earth = iga::kEarthRadiusKm;
    a.z0 = p->z_grnd;
    a.r_grnd = a.r_earth + a.z0;
    // main.infraga.sph.cpp:318-320: angles to radians, z_src = max(z_src, topo::z - r0)
    a.src_x = p->src[0] * d2r;
    a.src_y = p->src[1] * d2r;
    a.src_z = std::max(p->src[2], a.r_grnd - a.r_earth);
    a.cos_lat_src = std::cos(a.src_x);
    a.lat_min = p->lat_min * d2r; a.lat_max = p->lat_max * d2r;
    a.lon_min = p->lon_min * d2r; a.lon_max = p->lon_max * d2r;
    a.time_max_h = p->time_max;
    const double half_ang = p->rng_max / (2.0 * a.r_earth);
    if (half_ang > 0.0 && half_ang < 0.5 * iga::kPi - 1e-6) {
        const double sh = std::sin(half_ang);
        a.hav_rng = sh * sh;
        a.rng_exact_only = 0;
    } else {
        a.hav_rng = 0.0;
        a.rng_exact_only = 1;
    }
    // values at the source radius r0 + z_src and the ground radius r_grnd
    const double r_src = a.r_earth + a.src_z;
    const double zs = r_src - a.r_earth, zg = a.r_grnd - a.r_earth;
    auto bl_sc = [&](double r, double& sc, double& dsc) {   // bndlyr_sc / bndlyr_dsc(n = 0)
        sc = 1.0; dsc = 0.0;
        if (r - a.r_earth < a.z0 + 2.0) {
            const double X = std::exp(-(r - a.r_grnd) / 0.1);
            sc = (1.0 - X) / (1.0 + X);
            dsc = -2.0 * (-X / 0.1) / std::pow(1.0 + X, 2);
        }
    };
    double f, d1, d2, sc, dsc;
    iga::spline_eval(P.z, P.c, P.cs, zs, f, d1, d2); a.c0 = f;
    bl_sc(r_src, sc, dsc);
    iga::spline_eval(P.z, P.u, P.us, zs, f, d1, d2); a.u0s = f * sc;
    iga::spline_eval(P.z, P.v, P.vs, zs, f, d1, d2); a.v0s = f * sc;
    iga::spline_eval(P.z, P.rho, P.rhos, zs, f, d1, d2); a.rho0 = f;
    double dcg;
    iga::spline_eval(P.z, P.c, P.cs, zg, f, d1, d2); a.c_gnd = f; dcg = d1; a.dcz_g = d1;
    bl_sc(a.r_grnd, sc, dsc);
    iga::spline_eval(P.z, P.u, P.us, zg, f, d1, d2); a.duz_g = f * dsc + d1 * sc;
    iga::spline_eval(P.z, P.v, P.vs, zg, f, d1, d2); a.dvz_g = f * dsc + d1 * sc;
    a.c_ratio = a.c_gnd / a.c0;
    // set_refl (geoac.eqset.sph.strat.cpp:184-194) factors of dnu_r/ds and ds0
    a.refl_k1 = a.c0 / a.c_gnd * dcg;
    a.refl_k2 = std::pow(a.c_gnd, 2) / a.c0 * 1.0 / a.r_grnd;
    a.refl_k3 = -1.0 / a.c_gnd;
    a.refl_mcr = -a.c0 / a.c_gnd;
    return IGA_OK;
}

// Range-dependent spherical launch constants (run_prop of infraga-sph-rngdep,
// main.infraga.sph.rngdep.cpp:310-320; set_initial; topo::set_bndlyr
// atmo_state.sph.rngdep.cpp:22-33).
int build_args_spht(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a);

int build_args_sphr(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    if (h->strat_topo) return build_args_spht(h, p, a);
    const iga::RngdepGrid& g = h->grid;
    const double d2r = iga::kPi / 180.0;
    a.r_earth = iga::kEarthRadiusKm;
    a.src_x = p->src[0] * d2r;
    a.src_y = p->src[1] * d2r;
    a.cos_lat_src = std::cos(a.src_x);
    a.lat_min = p->lat_min * d2r; a.lat_max = p->lat_max * d2r;
    a.lon_min = p->lon_min * d2r; a.lon_max = p->lon_max * d2r;
    a.time_max_h = p->time_max;
    const double half_ang = p->rng_max / (2.0 * a.r_earth);
    a.rng_exact_only = (half_ang > 0.0 && half_ang < 0.5 * iga::kPi - 1e-6) ? 0 : 1;
    a.hav_rng = a.rng_exact_only ? 0.0 : std::pow(std::sin(half_ang), 2);
    // ground: terrain (z_max = max(0, terrain) + 0.01, z_bndlyr = max + 2) or flat z0
    a.z0 = p->z_grnd;
    a.r_grnd = a.r_earth + a.z0;
    auto topo_r = [&](double lat, double lon) {
        if (!h->has_topo) return a.r_grnd;
        double z, dz[2];
        iga::terrain_eval1(h->topo, lat, lon, z, dz);
        return a.r_earth + z;
    };
    if (h->has_topo) {
        a.topo_zmax = h->topo.z_max + 0.01;
        a.z_bl = h->topo.z_max + 2.0;
        a.x_cut = h->topo.z_max + 40.0;
    } else {
        a.topo_zmax = a.z0;
        a.z_bl = a.z0 + 2.0;
        a.x_cut = a.z0 + 40.0;
    }
    a.src_z = std::max(p->src[2], topo_r(a.src_x, a.src_y) - a.r_earth);
    const double r_src = a.r_earth + a.src_z;
    double sc = 1.0;
    if (r_src - a.r_earth < a.z_bl) {
        const double X = std::exp(-(r_src - topo_r(a.src_x, a.src_y)) / 0.1);
        sc = (1.0 - X) / (1.0 + X);
    }
    double f, df[3];
    const double zs = r_src - a.r_earth;
    iga::hybrid_eval1(g, 0, a.src_x, a.src_y, zs, f, df); a.c0 = f;
    iga::hybrid_eval1(g, 1, a.src_x, a.src_y, zs, f, df); a.u0s = f * sc;
    iga::hybrid_eval1(g, 2, a.src_x, a.src_y, zs, f, df); a.v0s = f * sc;
    iga::hybrid_eval1(g, 3, a.src_x, a.src_y, zs, f, df); a.rho0 = f;
    a.refl_mcr = 0.0;   // position dependent here: formed in the kernel
    a.hyb_tab = h->d_hyb;
    const size_t n_rec = (size_t)g.nx * g.ny * g.nz * iga::kHybRec;
    a.hyb_x = h->d_hyb + n_rec;
    a.hyb_y = a.hyb_x + g.nx;
    a.hyb_z = a.hyb_y + g.ny;
    a.hyb_nx = g.nx; a.hyb_ny = g.ny; a.hyb_nz = g.nz;
    if (h->has_topo) {
        const iga::Terrain& t = h->topo;
        a.topo_tab = h->d_topo;
        a.topo_x = h->d_topo + (size_t)t.nx * t.ny * 4;
        a.topo_y = a.topo_x + t.nx;
        a.topo_nx = t.nx; a.topo_ny = t.ny;
    } else {
        a.topo_tab = nullptr; a.topo_x = a.topo_y = nullptr; a.topo_nx = a.topo_ny = 0;
    }
    return IGA_OK;
}

int set_terrain_args(iga_atmo_s* h, iga::Fan3DArgs& a) {
    const iga::Terrain& t = h->topo;
    a.topo_tab = h->d_topo;
    a.topo_x = h->d_topo + (size_t)t.nx * t.ny * 4;
    a.topo_y = a.topo_x + t.nx;
    a.topo_nx = t.nx; a.topo_ny = t.ny;
    return IGA_OK;
}

// infraga-3d over terrain: run_prop of main.infraga.3d.cpp:199-357 with a
// topo_file, set_initial (eqset.3d.strat.cpp:58-105) at the source raised to
// the ground, topo::set_bndlyr (atmo_state.3d.strat.cpp:36-49: the terrain
// maximum, from 0, plus 0.1 km is the ground-check ceiling, 2 km above it the
// boundary-layer top), topo::z0 = the first profile altitude (set_limits,
// atmo_io.3d.strat.cpp:24-37).  The fan runs the 3D terrain kernel with the
// 1D knot table in place of the hybrid grid.
int build_args_3dt(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    const StratProfile& P = h->prof;
    a.knots = h->d_knots;
    a.n_knots = (int)P.z.size();
    a.uniform = P.uniform ? 1 : 0;
    a.z_lo = P.z.front(); a.z_hi = P.z.back(); a.inv_dz = P.inv_dz;
    a.src_x = p->src[0]; a.src_y = p->src[1];
    a.x_min = p->x_min; a.x_max = p->x_max; a.y_min = p->y_min; a.y_max = p->y_max;
    a.z0 = P.z.front();
    a.topo_zmax = h->topo.z_max + 0.1;
    a.z_bl = a.topo_zmax + 2.0;
    a.x_cut = a.topo_zmax + 40.0;
    double zt = 0.0, dz[2];
    iga::terrain_eval1(h->topo, a.src_x, a.src_y, zt, dz);
    a.src_z = std::max(p->src[2], zt);
    double sc = 1.0;
    if (a.src_z < a.z_bl) {
        const double X = std::exp(-(a.src_z - zt) / 0.1);
        sc = (1.0 - X) / (1.0 + X);
    }
    double f, d1, d2;
    iga::spline_eval(P.z, P.c, P.cs, a.src_z, f, d1, d2); a.c0 = f;
    iga::spline_eval(P.z, P.u, P.us, a.src_z, f, d1, d2); a.u0s = f * sc;
    iga::spline_eval(P.z, P.v, P.vs, a.src_z, f, d1, d2); a.v0s = f * sc;
    iga::spline_eval(P.z, P.rho, P.rhos, a.src_z, f, d1, d2); a.rho0 = f;
    a.hyb_tab = nullptr; a.hyb_x = a.hyb_y = a.hyb_z = nullptr;
    a.hyb_nx = a.hyb_ny = a.hyb_nz = 0;
    return set_terrain_args(h, a);
}

// infraga-sph over terrain: run_prop of main.infraga.sph.cpp:200-360 with a
// topo_file, set_initial at the source raised to the ground, topo::set_bndlyr
// (atmo_state.sph.strat.cpp:41-54: ground-check ceiling = terrain maximum,
// from 0, plus 0.01 km; boundary-layer top 2 km above that ceiling),
// topo::z0 = the first profile altitude (set_limits, atmo_io.sph.strat.cpp:27-39).
// The fan runs the spherical terrain kernel with the 1D knot table.
int build_args_spht(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    const StratProfile& P = h->prof;
    const double d2r = iga::kPi / 180.0;
    a.knots = h->d_knots;
    a.n_knots = (int)P.z.size();
    a.uniform = P.uniform ? 1 : 0;
    a.z_lo = P.z.front(); a.z_hi = P.z.back(); a.inv_dz = P.inv_dz;
    a.r_earth = iga::kEarthRadiusKm;
    a.src_x = p->src[0] * d2r;
    a.src_y = p->src[1] * d2r;
    a.cos_lat_src = std::cos(a.src_x);
    a.lat_min = p->lat_min * d2r; a.lat_max = p->lat_max * d2r;
    a.lon_min = p->lon_min * d2r; a.lon_max = p->lon_max * d2r;
    a.time_max_h = p->time_max;
    const double half_ang = p->rng_max / (2.0 * a.r_earth);
    a.rng_exact_only = (half_ang > 0.0 && half_ang < 0.5 * iga::kPi - 1e-6) ? 0 : 1;
    a.hav_rng = a.rng_exact_only ? 0.0 : std::pow(std::sin(half_ang), 2);
    a.z0 = P.z.front();
    a.r_grnd = a.r_earth + a.z0;
    a.topo_zmax = h->topo.z_max + 0.01;
    a.z_bl = a.topo_zmax + 2.0;
    a.x_cut = a.topo_zmax + 40.0;
    double zt = 0.0, dz[2];
    iga::terrain_eval1(h->topo, a.src_x, a.src_y, zt, dz);
    a.src_z = std::max(p->src[2], zt);
    double sc = 1.0;
    if (a.src_z < a.z_bl) {
        const double X = std::exp(-((a.r_earth + a.src_z) - (a.r_earth + zt)) / 0.1);
        sc = (1.0 - X) / (1.0 + X);
    }
    double f, d1, d2;
    iga::spline_eval(P.z, P.c, P.cs, a.src_z, f, d1, d2); a.c0 = f;
    iga::spline_eval(P.z, P.u, P.us, a.src_z, f, d1, d2); a.u0s = f * sc;
    iga::spline_eval(P.z, P.v, P.vs, a.src_z, f, d1, d2); a.v0s = f * sc;
    iga::spline_eval(P.z, P.rho, P.rhos, a.src_z, f, d1, d2); a.rho0 = f;
    a.refl_mcr = 0.0;   // position dependent: formed in the kernel
    a.hyb_tab = nullptr; a.hyb_x = a.hyb_y = a.hyb_z = nullptr;
    a.hyb_nx = a.hyb_ny = a.hyb_nz = 0;
    return set_terrain_args(h, a);
}

// 3D range-dependent launch constants (run_prop of infraga-3d-rngdep,
// main.infraga.3d.rngdep.cpp:235-309; set_initial; topo::set_bndlyr).
// Without terrain topo::z is 0 in this solver (atmo_state.3d.rngdep.cpp:45-51).
int build_args_3dr(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    const iga::RngdepGrid& g = h->grid;
    if (h->strat_topo) return build_args_3dt(h, p, a);
    a.src_x = p->src[0]; a.src_y = p->src[1];
    a.x_min = p->x_min; a.x_max = p->x_max; a.y_min = p->y_min; a.y_max = p->y_max;
    a.z0 = p->z_grnd;
    auto topo_z = [&](double x, double y) {
        if (!h->has_topo) return 0.0;
        double z, dz[2];
        iga::terrain_eval1(h->topo, x, y, z, dz);
        return z;
    };
    if (h->has_topo) {
        a.topo_zmax = h->topo.z_max + 0.01;
        a.z_bl = h->topo.z_max + 2.0;
        a.x_cut = h->topo.z_max + 40.0;
    } else {
        a.topo_zmax = a.z0;
        a.z_bl = a.z0 + 2.0;
        a.x_cut = 40.0;
    }
    a.src_z = std::max(p->src[2], topo_z(a.src_x, a.src_y));
    double sc = 1.0;
    if (a.src_z < a.z_bl) {
        const double X = std::exp(-(a.src_z - topo_z(a.src_x, a.src_y)) / 0.1);
        sc = (1.0 - X) / (1.0 + X);
    }
    double f, df[3];
    iga::hybrid_eval1(g, 0, a.src_x, a.src_y, a.src_z, f, df); a.c0 = f;
    iga::hybrid_eval1(g, 1, a.src_x, a.src_y, a.src_z, f, df); a.u0s = f * sc;
    iga::hybrid_eval1(g, 2, a.src_x, a.src_y, a.src_z, f, df); a.v0s = f * sc;
    iga::hybrid_eval1(g, 3, a.src_x, a.src_y, a.src_z, f, df); a.rho0 = f;
    a.hyb_tab = h->d_hyb;
    const size_t n_rec = (size_t)g.nx * g.ny * g.nz * iga::kHybRec;
    a.hyb_x = h->d_hyb + n_rec;
    a.hyb_y = a.hyb_x + g.nx;
    a.hyb_z = a.hyb_y + g.ny;
    a.hyb_nx = g.nx; a.hyb_ny = g.ny; a.hyb_nz = g.nz;
    if (h->has_topo) {
        const iga::Terrain& t = h->topo;
        a.topo_tab = h->d_topo;
        a.topo_x = h->d_topo + (size_t)t.nx * t.ny * 4;
        a.topo_y = a.topo_x + t.nx;
        a.topo_nx = t.nx; a.topo_ny = t.ny;
    } else {
        a.topo_tab = nullptr; a.topo_x = a.topo_y = nullptr; a.topo_nx = a.topo_ny = 0;
    }
    return IGA_OK;
}

int build_args(iga_atmo_s* h, const iga_fan_params* p, iga::Fan3DArgs& a) {
    const StratProfile& P = h->prof;
    memset(&a, 0, sizeof(a));
    if (h->kind != 0) {
        a.bounces = p->bounces;
        a.write_rays = p->write_rays ? 1 : 0;
        a.length = (int)(p->s_max / p->ds_min);
        a.ds_min = p->ds_min; a.ds_max = p->ds_max; a.s_max = p->s_max;
        a.alt_max = p->alt_max; a.rng_max = p->rng_max;
        a.bl = 0.1;
        a.inv_bl = 1.0 / a.bl;
        a.freq = p->freq; a.tweak_abs = p->tweak_abs; a.turn_ht_min = p->turn_ht_min;
        a.sb.x0_low = std::pow(10.0, -0.67887);
        a.sb.x1_low = std::pow(10.0, -0.10744);
        a.sb.x2 = std::pow(10.0, -3.3979);
        return h->kind == 1 ? build_args_sphr(h, p, a) : build_args_3dr(h, p, a);
    }
    a.knots = h->d_knots;
    a.n_knots = (int)P.z.size();
    a.uniform = P.uniform ? 1 : 0;
    a.z_lo = P.z.front();
    a.z_hi = P.z.back();
    a.inv_dz = P.inv_dz;
    a.bounces = p->bounces;
    a.write_rays = p->write_rays ? 1 : 0;
    a.length = (int)(p->s_max / p->ds_min);
    a.src_x = p->src[0];
    a.src_y = p->src[1];
    a.z0 = p->z_grnd;
    a.src_z = std::max(p->src[2], a.z0);   // z_src = max(z_src, topo::z) (main.infraga.3d.cpp:306)
    a.ds_min = p->ds_min; a.ds_max = p->ds_max; a.s_max = p->s_max;
    a.alt_max = p->alt_max; a.rng_max = p->rng_max;
    a.x_min = p->x_min; a.x_max = p->x_max; a.y_min = p->y_min; a.y_max = p->y_max;
    a.z_bl = a.z0 + 2.0;
    a.bl = 0.1;
    a.inv_bl = 1.0 / a.bl;
    a.freq = p->freq; a.tweak_abs = p->tweak_abs; a.turn_ht_min = p->turn_ht_min;
    double f, d1, d2, sc, dsc;
    iga::spline_eval(P.z, P.c, P.cs, a.src_z, f, d1, d2); a.c0 = f;
    bl_host(a.src_z, a.z0, a.bl, sc, dsc);
    iga::spline_eval(P.z, P.u, P.us, a.src_z, f, d1, d2); a.u0s = f * sc;
    iga::spline_eval(P.z, P.v, P.vs, a.src_z, f, d1, d2); a.v0s = f * sc;
    iga::spline_eval(P.z, P.rho, P.rhos, a.src_z, f, d1, d2); a.rho0 = f;
    iga::spline_eval(P.z, P.c, P.cs, a.z0, f, d1, d2); a.c_gnd = f; a.dcz_g = d1;
    bl_host(a.z0, a.z0, a.bl, sc, dsc);
    iga::spline_eval(P.z, P.u, P.us, a.z0, f, d1, d2); a.duz_g = f * dsc + d1 * sc;
    iga::spline_eval(P.z, P.v, P.vs, a.z0, f, d1, d2); a.dvz_g = f * dsc + d1 * sc;
    a.c_ratio = a.c_gnd / a.c0;
    a.sb.x0_low = std::pow(10.0, -0.67887);
    a.sb.x1_low = std::pow(10.0, -0.10744);
    a.sb.x2 = std::pow(10.0, -3.3979);
    if (p->geometry == IGA_GEOM_SPH) return build_args_sph(h, p, a);
    return IGA_OK;
}

}  // namespace iga_internal

namespace {

int run_device(iga_atmo_s* h, const iga_fan_params* p, const double* d_th, const double* d_ph, int n_rays,
               double* d_arr, int* d_n, long long* d_steps, int* d_status, double* d_aux, void* d_ws,
               cudaStream_t st, int grid_cap = 0, const PathSpec* ps = nullptr) {
    const bool f32c = p->precision == IGA_FP32C || p->precision == IGA_FP32C_FLAGGED;
    const bool sph_grid = h->kind == 1 && !h->strat_topo;   // a spherical node grid (not a profile over terrain)
    if (h->kind != 0 && (p->geometry != (h->kind == 1 ? IGA_GEOM_SPH : IGA_GEOM_3D) ||
                         (p->precision != IGA_FP64 && !(sph_grid && f32c)))) {
        g_cuda_err = "range-dependent or terrain atmosphere: the geometry it was loaded for; FP32C on a spherical "
                     "node grid only";
        return IGA_E_UNSUPPORTED;
    }
    if (p->geometry == IGA_GEOM_SPH && f32c && !sph_grid) {
        g_cuda_err = "spherical geometry: FP32C on range-dependent node grids only";
        return IGA_E_UNSUPPORTED;
    }
    NvtxRange nv(ps ? "iga_fan_paths launch" : "iga_fan launch");
    iga::Fan3DArgs a;
    int rc = build_args(h, p, a);
    if (rc) return rc;
    a.theta_deg = d_th; a.phi_deg = d_ph; a.n_rays = n_rays;
    a.arrivals = d_arr; a.n_arr = d_n; a.ray_steps = d_steps; a.ray_status = d_status; a.aux = d_aux;
    a.queue = static_cast<unsigned int*>(d_ws);
    a.grid_cap = grid_cap;
    a.block = p->block;
    if (ps) {
        if (p->precision != IGA_FP64) {
            g_cuda_err = "sampled ray paths: FP64 only";
            return IGA_E_UNSUPPORTED;
        }
        a.path_rows = ps->rows; a.path_off = ps->off; a.path_n = ps->n; a.path_mode = ps->mode;
        a.caus_rows = ps->caus; a.caus_count = ps->caus_count; a.caus_cap = ps->caus_cap;
    }
    a.retrace = p->precision == IGA_FP32C ? 1 : 0;
    if (f32c && h->kind == 0) {
        iga_atmo_s::AlphaTab t;
        rc = ensure_alpha(h, p->freq, t);
        if (rc) return rc;
        a.knots_c = h->d_knots_c;
        a.alpha_tab = t.d; a.alpha_n = t.n; a.alpha_z0 = t.z0; a.alpha_inv_h = t.inv_h;
    }
    if (f32c && sph_grid) a.hyb_x32 = h->d_hyb_x32;
    IGA_CUDA(cudaMemsetAsync(d_ws, 0, iga_fan_workspace_bytes(), st), "cudaMemsetAsync(workspace)");
    if (n_rays == 0) return IGA_OK;
    if (sph_grid && f32c)
        IGA_CUDA(iga::launch_fansphr_fp32c(a, p->calc_amp != 0, st, nullptr), "fansphr fp32c kernel launch");
    else if (h->kind == 1)
        IGA_CUDA(iga::launch_fansphr_fp64(a, p->calc_amp != 0, st, nullptr), "fansphr kernel launch");
    else if (h->kind == 2)
        IGA_CUDA(iga::launch_fan3dr_fp64(a, p->calc_amp != 0, st, nullptr), "fan3dr kernel launch");
    else if (p->geometry == IGA_GEOM_SPH)
        IGA_CUDA(iga::launch_fansph_fp64(a, p->calc_amp != 0, st, nullptr), "fansph kernel launch");
    else if (f32c)
        IGA_CUDA(iga::launch_fan3d_fp32c(a, p->calc_amp != 0, st, nullptr), "fan3d fp32c kernel launch");
    else
        IGA_CUDA(iga::launch_fan3d_fp64(a, p->calc_amp != 0, st, nullptr), "fan3d kernel launch");
    return IGA_OK;
}

}  // namespace

namespace iga_internal {
int fp32c_setup(iga_atmo_s* h, double freq, iga::Fan3DArgs& a) {
    iga_atmo_s::AlphaTab t;
    int rc = ensure_alpha(h, freq, t);
    if (rc) return rc;
    a.knots_c = h->d_knots_c;
    a.alpha_tab = t.d; a.alpha_n = t.n; a.alpha_z0 = t.z0; a.alpha_inv_h = t.inv_h;
    return IGA_OK;
}

int fan_device(iga_atmo_s* h, const iga_fan_params* p, const double* d_th, const double* d_ph, int n_rays,
               double* d_arr, int* d_n, long long* d_steps, int* d_status, double* d_aux, void* d_ws,
               cudaStream_t st, int grid_cap, const PathSpec* paths) {
    int rc = validate(p, n_rays);
    if (rc) return rc;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    return run_device(h, p, d_th, d_ph, n_rays, d_arr, d_n, d_steps, d_status, d_aux, d_ws, st, grid_cap, paths);
}
}  // namespace iga_internal

extern "C" {

const char* iga_strerror(int status) {
    switch (status) {
        case IGA_OK: return "ok";
        case IGA_E_INVALID: return "invalid argument";
        case IGA_E_IO: return g_err.empty() ? "profile or terrain file error" : g_err.c_str();
        case IGA_E_NOMEM: return "out of memory";
        case IGA_E_CUDA: return "CUDA error";
        case IGA_E_NODEVICE: return "no usable CUDA device";
        case IGA_E_TRUNCATED: return "output capacity too small";
        case IGA_E_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

const char* iga_last_cuda_error(void) { return g_cuda_err.c_str(); }

int iga_version(void) { return IGA_ABI_VERSION; }

int iga_device_count(int* count) {
    if (!count) return IGA_E_INVALID;
    *count = 0;
    IGA_CUDA(cudaGetDeviceCount(count), "cudaGetDeviceCount");
    return IGA_OK;
}

int iga_atmo_load(const char* met_path, const char* format, int reverse_winds, iga_atmo_t* out) {
    if (!met_path || !out) return IGA_E_INVALID;
    *out = nullptr;
    iga_atmo_s* h = new (std::nothrow) iga_atmo_s();
    if (!h) return IGA_E_NOMEM;
    int rc = iga::load_met(met_path, format ? format : "zTuvdp", reverse_winds != 0, h->prof, g_err);
    if (rc == IGA_OK) rc = upload(h);
    if (rc != IGA_OK) { iga_atmo_destroy(h); return rc; }
    *out = h;
    return IGA_OK;
}

int iga_atmo_load_rngdep(const char* prefix, const char* x_file, const char* y_file, const char* topo_file,
                         const char* format, int reverse_winds, int geometry, iga_atmo_t* out) {
    if (!prefix || !x_file || !y_file || !out) return IGA_E_INVALID;
    if (geometry != IGA_GEOM_3D && geometry != IGA_GEOM_SPH) return IGA_E_INVALID;
    *out = nullptr;
    iga_atmo_s* h = new (std::nothrow) iga_atmo_s();
    if (!h) return IGA_E_NOMEM;
    const bool sph = geometry == IGA_GEOM_SPH;
    h->kind = sph ? 1 : 2;
    int rc = iga::load_rngdep(prefix, x_file, y_file, format ? format : "zTuvdp", reverse_winds != 0, sph, h->grid, g_err);
    if (rc == IGA_OK && topo_file && topo_file[0]) {
        rc = iga::load_terrain(topo_file, sph, h->topo, g_err);
        h->has_topo = (rc == IGA_OK);
    }
    if (rc == IGA_OK) rc = upload_rngdep(h);
    if (rc != IGA_OK) { iga_atmo_destroy(h); return rc; }
    *out = h;
    return IGA_OK;
}

int iga_atmo_load_topo(const char* met_path, const char* topo_file, const char* format, int reverse_winds,
                       int geometry, iga_atmo_t* out) {
    if (!met_path || !topo_file || !out) return IGA_E_INVALID;
    if (geometry != IGA_GEOM_3D && geometry != IGA_GEOM_SPH) return IGA_E_INVALID;
    *out = nullptr;
    iga_atmo_s* h = new (std::nothrow) iga_atmo_s();
    if (!h) return IGA_E_NOMEM;
    const bool sph = geometry == IGA_GEOM_SPH;
    h->kind = sph ? 1 : 2;
    h->strat_topo = true;
    int rc = iga::load_terrain(topo_file, sph, h->topo, g_err);
    h->has_topo = (rc == IGA_OK);
    if (rc == IGA_OK) rc = iga::load_met(met_path, format ? format : "zTuvdp", reverse_winds != 0, h->prof, g_err);
    if (rc == IGA_OK) rc = upload(h);
    if (rc == IGA_OK) rc = upload_terrain(h);
    if (rc != IGA_OK) { iga_atmo_destroy(h); return rc; }
    *out = h;
    return IGA_OK;
}

int iga_atmo_terrain(iga_atmo_t h, double x, double y, double* z, double* dz_dx, double* dz_dy) {
    if (!h) return IGA_E_INVALID;
    if (!h->has_topo) return IGA_E_UNSUPPORTED;
    double zz = 0.0, d[2] = {0.0, 0.0};
    iga::terrain_eval1(h->topo, x, y, zz, d);
    if (z) *z = zz;
    if (dz_dx) *dz_dx = d[0];
    if (dz_dy) *dz_dy = d[1];
    return IGA_OK;
}

int iga_atmo_sample(iga_atmo_t h, const iga_fan_params* p, double x, double y, const double* z, int n, double* out) {
    if (!h || !p || n < 0 || (n > 0 && (!z || !out))) return IGA_E_INVALID;
    const bool sph = p->geometry == IGA_GEOM_SPH;
    if (h->kind != 0 && sph != (h->kind == 1)) return IGA_E_UNSUPPORTED;
    iga::Fan3DArgs a;   // host-side launch constants: ground, boundary-layer top
    int rc = build_args(h, p, a);
    if (rc) return rc;
    const double d2r = iga::kPi / 180.0;
    const double hx = sph ? x * d2r : x, hy = sph ? y * d2r : y;   // grid / terrain units
    // topo::z under the point (an altitude): terrain, else the flat ground (0 for
    // the 3D range-dependent solver without terrain, atmo_state.3d.rngdep.cpp:45-51)
    double zg = a.z0;
    if (h->has_topo) {
        double dz[2];
        iga::terrain_eval1(h->topo, hx, hy, zg, dz);
    } else if (h->kind == 2) {
        zg = 0.0;
    }
    const bool hybrid = h->kind != 0 && !h->strat_topo;
    const StratProfile& P = h->prof;
    for (int i = 0; i < n; i++) {
        double sc = 1.0;   // topo::bndlyr_sc
        if (z[i] < a.z_bl) {
            const double X = std::exp(-(z[i] - zg) / a.bl);
            sc = (1.0 - X) / (1.0 + X);
        }
        double f[4];
        if (hybrid) {
            double df[3];
            for (int k = 0; k < 4; k++) iga::hybrid_eval1(h->grid, k, hx, hy, z[i], f[k], df);
        } else {
            double d1, d2;
            iga::spline_eval(P.z, P.c, P.cs, z[i], f[0], d1, d2);
            iga::spline_eval(P.z, P.u, P.us, z[i], f[1], d1, d2);
            iga::spline_eval(P.z, P.v, P.vs, z[i], f[2], d1, d2);
            iga::spline_eval(P.z, P.rho, P.rhos, z[i], f[3], d1, d2);
        }
        out[4 * i + 0] = f[0];
        out[4 * i + 1] = f[1] * sc;
        out[4 * i + 2] = f[2] * sc;
        out[4 * i + 3] = f[3];
    }
    return IGA_OK;
}

int iga_atmo_region(iga_atmo_t h, double* lat_min, double* lat_max, double* lon_min, double* lon_max) {
    if (!h) return IGA_E_INVALID;
    double r[4] = {-90.0, 90.0, -180.0, 180.0};
    if (h->kind == 2 && h->strat_topo) {
        // geoac::set_limits with terrain (atmo_io.3d.strat.cpp:24-30): terrain extent less 0.001 km
        const double buf = 0.001;
        r[0] = h->topo.x.front() + buf; r[1] = h->topo.x.back() - buf;
        r[2] = h->topo.y.front() + buf; r[3] = h->topo.y.back() - buf;
    } else if (h->kind == 2) {
        // geoac::set_limits (atmo_io.3d.rngdep.cpp:25-40): grid (and terrain) extent less 0.001 km
        const double buf = 0.001;
        double a0 = h->grid.x.front() + buf, a1 = h->grid.x.back() - buf;
        double b0 = h->grid.y.front() + buf, b1 = h->grid.y.back() - buf;
        if (h->has_topo) {
            a0 = std::max(a0, h->topo.x.front() + buf); a1 = std::min(a1, h->topo.x.back() - buf);
            b0 = std::max(b0, h->topo.y.front() + buf); b1 = std::min(b1, h->topo.y.back() - buf);
        }
        r[0] = a0; r[1] = a1; r[2] = b0; r[3] = b1;
    } else if (h->kind == 1 && h->strat_topo) {
        // geoac::set_limits with terrain (atmo_io.sph.strat.cpp:27-31): terrain extent less 1e-3 deg
        const double buf = 1.0e-3 * (iga::kPi / 180.0), r2d = 180.0 / iga::kPi;
        r[0] = (h->topo.x.front() + buf) * r2d; r[1] = (h->topo.x.back() - buf) * r2d;
        r[2] = (h->topo.y.front() + buf) * r2d; r[3] = (h->topo.y.back() - buf) * r2d;
    } else if (h->kind == 1) {
        // geoac::set_limits (atmo_io.sph.rngdep.cpp:27-43): grid (and terrain) extent less 1e-3 deg
        const double buf = 1.0e-3 * (iga::kPi / 180.0);
        double a0 = h->grid.x.front() + buf, a1 = h->grid.x.back() - buf;
        double b0 = h->grid.y.front() + buf, b1 = h->grid.y.back() - buf;
        if (h->has_topo) {
            a0 = std::max(a0, h->topo.x.front() + buf); a1 = std::min(a1, h->topo.x.back() - buf);
            b0 = std::max(b0, h->topo.y.front() + buf); b1 = std::min(b1, h->topo.y.back() - buf);
        }
        const double r2d = 180.0 / iga::kPi;
        r[0] = a0 * r2d; r[1] = a1 * r2d; r[2] = b0 * r2d; r[3] = b1 * r2d;
    }
    if (lat_min) *lat_min = r[0];
    if (lat_max) *lat_max = r[1];
    if (lon_min) *lon_min = r[2];
    if (lon_max) *lon_max = r[3];
    return IGA_OK;
}

int iga_atmo_create(const iga_profile* pr, iga_atmo_t* out) {
    if (!pr || !out || pr->n < 3 || !pr->z || !pr->c || !pr->u || !pr->v || !pr->rho) return IGA_E_INVALID;
    *out = nullptr;
    iga_atmo_s* h = new (std::nothrow) iga_atmo_s();
    if (!h) return IGA_E_NOMEM;
    h->prof.z.assign(pr->z, pr->z + pr->n);
    h->prof.c.assign(pr->c, pr->c + pr->n);
    h->prof.u.assign(pr->u, pr->u + pr->n);
    h->prof.v.assign(pr->v, pr->v + pr->n);
    h->prof.rho.assign(pr->rho, pr->rho + pr->n);
    int rc = iga::finalize_profile(h->prof, g_err);
    if (rc == IGA_OK) rc = upload(h);
    if (rc != IGA_OK) { iga_atmo_destroy(h); return rc; }
    *out = h;
    return IGA_OK;
}

int iga_atmo_limits(iga_atmo_t h, double* z_ground, double* z_top) {
    if (!h) return IGA_E_INVALID;
    if (z_ground) *z_ground = h->prof.z.front();
    if (z_top) *z_top = h->prof.z.back();
    return IGA_OK;
}

int iga_atmo_destroy(iga_atmo_t h) {
    if (!h) return IGA_OK;
    if (h->d_knots) cudaFree(h->d_knots);
    if (h->d_buf) cudaFree(h->d_buf);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->d_knots_c) cudaFree(h->d_knots_c);
    if (h->d_hyb) cudaFree(h->d_hyb);
    if (h->d_hyb_x32) cudaFree(h->d_hyb_x32);
    if (h->d_topo) cudaFree(h->d_topo);
    for (auto& kv : h->alpha) cudaFree(kv.second.d);
    delete h;
    return IGA_OK;
}

int iga_fan_params_default(iga_atmo_t h, iga_fan_params* p) {
    if (!h || !p) return IGA_E_INVALID;
    memset(p, 0, sizeof(*p));
    p->geometry = IGA_GEOM_3D;
    p->precision = IGA_FP64;
    p->bounces = 10;
    p->calc_amp = 1;
    p->write_rays = 0;
    p->ds_min = 0.001; p->ds_max = 0.05; p->s_max = 1000.0;
    p->alt_max = h->prof.z.back();
    p->rng_max = 2000.0;
    p->x_min = -2000.0; p->x_max = 2000.0; p->y_min = -2000.0; p->y_max = 2000.0;
    p->z_grnd = h->prof.z.front();
    p->freq = 0.1; p->tweak_abs = 1.0; p->turn_ht_min = 0.2;
    p->lat_min = -90.0; p->lat_max = 90.0; p->lon_min = -180.0; p->lon_max = 180.0;
    p->time_max = 10.0;
    return IGA_OK;
}

int iga_fan_params_init(iga_atmo_t h, int geometry, iga_fan_params* p) {
    if (geometry != IGA_GEOM_3D && geometry != IGA_GEOM_SPH) return IGA_E_INVALID;
    int rc = iga_fan_params_default(h, p);
    if (rc) return rc;
    if (h->kind == 2 && geometry == IGA_GEOM_3D) {
        // run_prop of infraga-3d-rngdep (main.infraga.3d.rngdep.cpp:210-242): the
        // set_limits region and the source at its centre; rng_max keeps the
        // 1000 km of geoac.params.3d.cpp (set_limits here does not reset it)
        iga_atmo_region(h, &p->x_min, &p->x_max, &p->y_min, &p->y_max);
        p->src[0] = (p->x_max + p->x_min) / 2.0;
        p->src[1] = (p->y_max + p->y_min) / 2.0;
        p->rng_max = 1000.0;
    }
    if (geometry == IGA_GEOM_SPH) {
        p->geometry = IGA_GEOM_SPH;
        p->src[0] = 30.0; p->src[1] = 0.0; p->src[2] = 0.0;
        p->rng_max = 1000.0;
        if (h->kind == 1) {
            // run_prop of infraga-sph-rngdep (main.infraga.sph.rngdep.cpp:209, 238-239):
            // 2 bounces, source at the centre of the set_limits region
            iga_atmo_region(h, &p->lat_min, &p->lat_max, &p->lon_min, &p->lon_max);
            const double d2r = iga::kPi / 180.0, r2d = 180.0 / iga::kPi;
            p->src[0] = (p->lat_max * d2r + p->lat_min * d2r) / 2.0 * r2d;
            p->src[1] = (p->lon_max * d2r + p->lon_min * d2r) / 2.0 * r2d;
            // infraga-sph over terrain keeps its 10 bounces (main.infraga.sph.cpp:209)
            p->bounces = h->strat_topo ? 10 : 2;
        }
    }
    return IGA_OK;
}

size_t iga_fan_workspace_bytes(void) { return 256; }

// Launch-shape autotuner: the persistent fan kernels keep every resident
// thread busy with one ray at a time, so a fan with fewer rays than resident
// thread slots leaves SMs idle at the kernel's largest CTA size, while
// smaller CTAs spread the same rays over more SMs (and fit more CTAs per SM
// where registers limit occupancy).  Which wins depends on the fan (rays,
// ray lengths, kernel), so each candidate CTA size is timed on the fan itself.
int iga_fan_tune(iga_atmo_t h, const iga_fan_params* p, const double* theta_deg, const double* phi_deg, int n_rays,
                 int* best_block, double* seconds) {
    if (!h || !p || !best_block || n_rays <= 0 || !theta_deg || !phi_deg) return IGA_E_INVALID;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    const int nb = p->bounces + 1;
    const size_t n = (size_t)n_rays;
    double *d_th = nullptr, *d_ph = nullptr, *d_arr = nullptr;
    int* d_n = nullptr;
    long long* d_steps = nullptr;
    void* d_ws = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_th); cudaFree(d_ph); cudaFree(d_arr); cudaFree(d_n); cudaFree(d_steps); cudaFree(d_ws);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
    };
    cudaError_t e = cudaMalloc(&d_th, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_ph, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_arr, n * nb * IGA_ARRIVAL_COLS * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_n, n * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_steps, n * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&d_ws, iga_fan_workspace_bytes());
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_th, theta_deg, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ph, phi_deg, n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "iga_fan_tune set-up"); }
    const int cand[4] = {32, 64, 96, 128};
    double best_t = 1e300;
    int best = 0;
    for (int k = -1; k < 4; k++) {   // k = -1: untimed warm-up (module load)
        iga_fan_params q = *p;
        q.block = k < 0 ? 0 : cand[k];
        if ((e = cudaEventRecord(e0, st)) != cudaSuccess) break;
        rc = run_device(h, &q, d_th, d_ph, n_rays, d_arr, d_n, d_steps, nullptr, nullptr, d_ws, st);
        if (rc) { cleanup(); return rc; }
        if ((e = cudaEventRecord(e1, st)) != cudaSuccess) break;
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.0f;
        if ((e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) break;
        if (k < 0) continue;
        if (seconds) seconds[k] = 1e-3 * ms;
        if (1e-3 * ms < best_t) { best_t = 1e-3 * ms; best = cand[k]; }
    }
    cleanup();
    if (e != cudaSuccess) return cuda_fail(e, "iga_fan_tune");
    *best_block = best;
    return IGA_OK;
}

int iga_fan_run_device(iga_atmo_t h, const iga_fan_params* p, const double* d_th, const double* d_ph, int n_rays,
                       double* d_arr, int* d_n, long long* d_steps, int* d_status, double* d_aux, void* d_ws,
                       void* stream) {
    if (!h) return IGA_E_INVALID;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    if (n_rays > 0 && (!d_th || !d_ph || !d_arr || !d_n || !d_steps)) return IGA_E_INVALID;
    if (!d_ws || (reinterpret_cast<uintptr_t>(d_ws) & 15)) return IGA_E_INVALID;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    return run_device(h, p, d_th, d_ph, n_rays, d_arr, d_n, d_steps, d_status, d_aux, d_ws,
                      static_cast<cudaStream_t>(stream));
}

int iga_fan_run(iga_atmo_t h, const iga_fan_params* p, const double* theta_deg, const double* phi_deg, int n_rays,
                double* arrivals, int cap, int* n_out, int* ray_index, long long* ray_steps, int* ray_status,
                long long* total_steps, double* arrival_aux) {
    if (!h || !n_out) return IGA_E_INVALID;
    *n_out = 0;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    if (n_rays > 0 && (!theta_deg || !phi_deg)) return IGA_E_INVALID;
    if (cap > 0 && !arrivals) return IGA_E_INVALID;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    if (total_steps) *total_steps = 0;
    if (n_rays == 0) return IGA_OK;

    const int nb = p->bounces + 1;
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_ws = align(iga_fan_workspace_bytes());
    const size_t b_ang = align(sizeof(double) * (size_t)n_rays);
    const size_t b_arr = align(sizeof(double) * 12 * (size_t)nb * n_rays);
    const size_t b_n = align(sizeof(int) * (size_t)n_rays);
    const size_t b_st = align(sizeof(long long) * (size_t)n_rays);
    const size_t b_aux = arrival_aux ? align(sizeof(double) * 4 * (size_t)nb * n_rays) : 0;
    const size_t need = b_ws + 2 * b_ang + b_arr + 2 * b_n + b_st + b_aux;

    std::lock_guard<std::mutex> lock(h->mu);
    if (h->d_buf_bytes < need) {
        if (h->d_buf) cudaFree(h->d_buf);
        h->d_buf = nullptr;
        h->d_buf_bytes = 0;
        IGA_CUDA(cudaMalloc(&h->d_buf, need), "cudaMalloc(fan buffers)");
        h->d_buf_bytes = need;
    }
    char* base = static_cast<char*>(h->d_buf);
    void* d_ws = base; base += b_ws;
    double* d_th = reinterpret_cast<double*>(base); base += b_ang;
    double* d_ph = reinterpret_cast<double*>(base); base += b_ang;
    double* d_arr = reinterpret_cast<double*>(base); base += b_arr;
    int* d_n = reinterpret_cast<int*>(base); base += b_n;
    int* d_stat = reinterpret_cast<int*>(base); base += b_n;
    long long* d_steps = reinterpret_cast<long long*>(base); base += b_st;
    double* d_aux = arrival_aux ? reinterpret_cast<double*>(base) : nullptr;

    cudaStream_t st = h->stream;
    IGA_CUDA(cudaMemcpyAsync(d_th, theta_deg, sizeof(double) * n_rays, cudaMemcpyHostToDevice, st), "H2D theta");
    IGA_CUDA(cudaMemcpyAsync(d_ph, phi_deg, sizeof(double) * n_rays, cudaMemcpyHostToDevice, st), "H2D phi");
    rc = run_device(h, p, d_th, d_ph, n_rays, d_arr, d_n, d_steps, d_stat, d_aux, d_ws, st);
    if (rc) return rc;
    std::vector<int> n_arr(n_rays), stat(n_rays);
    std::vector<long long> steps(n_rays);
    std::vector<double> rows((size_t)12 * nb * n_rays);
    IGA_CUDA(cudaMemcpyAsync(n_arr.data(), d_n, sizeof(int) * n_rays, cudaMemcpyDeviceToHost, st), "D2H n_arr");
    IGA_CUDA(cudaMemcpyAsync(stat.data(), d_stat, sizeof(int) * n_rays, cudaMemcpyDeviceToHost, st), "D2H status");
    IGA_CUDA(cudaMemcpyAsync(steps.data(), d_steps, sizeof(long long) * n_rays, cudaMemcpyDeviceToHost, st), "D2H steps");
    IGA_CUDA(cudaMemcpyAsync(rows.data(), d_arr, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H arrivals");
    std::vector<double> aux_rows(arrival_aux ? (size_t)4 * nb * n_rays : 0);
    if (arrival_aux)
        IGA_CUDA(cudaMemcpyAsync(aux_rows.data(), d_aux, aux_rows.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H aux");
    IGA_CUDA(cudaStreamSynchronize(st), "fan kernel");

    long long tot = 0;
    int w = 0;
    for (int i = 0; i < n_rays; i++) {
        tot += steps[i];
        if (ray_steps) ray_steps[i] = steps[i];
        if (ray_status) ray_status[i] = stat[i];
        for (int j = 0; j < n_arr[i]; j++, w++) {
            if (w < cap) {
                memcpy(arrivals + (size_t)w * 12, &rows[((size_t)i * nb + j) * 12], 12 * sizeof(double));
                if (ray_index) ray_index[w] = i;
                if (arrival_aux) memcpy(arrival_aux + (size_t)w * 4, &aux_rows[((size_t)i * nb + j) * 4], 4 * sizeof(double));
            }
        }
    }
    *n_out = w;
    if (total_steps) *total_steps = tot;
    return w > cap ? IGA_E_TRUNCATED : IGA_OK;
}

}  // extern "C"

// ---- allocation-free fan entry (iga_fan_run_device_noalloc) ----
namespace {
constexpr int kMaxStaticDevices = 64;
// Ray-queue scratch for iga_fan_run_device_noalloc.  Host code must not use
// this name as an address (on the host it only stands in for the symbol):
// the per-device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_fan_static_scratch[IGA_FAN_STATIC_SCRATCH_BYTES];
std::mutex g_static_mu;
void* g_static_addr[kMaxStaticDevices] = {};
}  // namespace

extern "C" int iga_fan_run_device_noalloc(iga_atmo_t h, const iga_fan_params* p, const double* d_th,
                                          const double* d_ph, int n_rays, double* d_arr, int* d_n,
                                          long long* d_steps, int* d_status, double* d_aux, void* stream) {
    if (!h) return IGA_E_INVALID;
    int rc = validate(p, n_rays);
    if (rc) return rc;
    if (n_rays > 0 && (!d_th || !d_ph || !d_arr || !d_n || !d_steps)) return IGA_E_INVALID;
    if (p->precision != IGA_FP64) {
        g_cuda_err = "iga_fan_run_device_noalloc: FP64 only (FP32C builds its absorption table on first use)";
        return IGA_E_UNSUPPORTED;
    }
    if (iga_fan_workspace_bytes() > IGA_FAN_STATIC_SCRATCH_BYTES) {
        g_cuda_err = "iga_fan_run_device_noalloc: scratch need " + std::to_string(iga_fan_workspace_bytes()) +
                     " bytes exceeds the static " + std::to_string(IGA_FAN_STATIC_SCRATCH_BYTES) + "-byte array";
        return IGA_E_INVALID;
    }
    if (h->device < 0 || h->device >= kMaxStaticDevices) return IGA_E_UNSUPPORTED;
    IGA_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    void* ws = nullptr;
    {
        // one-time, per device, with that device current
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_addr[h->device]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_fan_static_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fan_static_scratch)");
            g_static_addr[h->device] = ptr;
        }
        ws = g_static_addr[h->device];
    }
    // run_device clears the queue counter on `stream` before the launch
    return run_device(h, p, d_th, d_ph, n_rays, d_arr, d_n, d_steps, d_status, d_aux, ws,
                      static_cast<cudaStream_t>(stream));
}
