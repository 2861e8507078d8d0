// Host-side stratified atmosphere: .met parsing and FP64 spline tables.
//
// The device kernels read one interleaved row per altitude knot (see
// kKnotStride); the slopes are the natural-cubic-spline knot derivatives the
// reference solves with the Thomas algorithm (interp::set,
// src/util/interpolation.cpp:103-136), built here in FP64 on the host.
#pragma once
#include <string>
#include <vector>

namespace iga {

// Row layout of the device knot table (doubles):
//   0 z, 1 1/(z[i+1]-z[i]) (0 on the last knot),
//   2 c, 3 c', 4 u, 5 u', 6 v, 7 v', 8 rho, 9 rho'
constexpr int kKnotStride = 10;
enum KnotCol { kZ = 0, kInvDz = 1, kC = 2, kCs = 3, kU = 4, kUs = 5, kV = 6, kVs = 7, kRho = 8, kRhos = 9 };

struct StratProfile {
    std::vector<double> z, c, u, v, rho;       // solver units (km, km/s, g/cm^3)
    std::vector<double> cs, us, vs, rhos;      // spline slopes
    std::vector<double> table;                 // n * kKnotStride
    bool uniform = false;                      // equal knot spacing
    double inv_dz = 0.0;                       // 1 / spacing when uniform
};

// Natural cubic spline knot slopes (tridiagonal solve, natural ends).
void natural_spline_slopes(const std::vector<double>& x, const std::vector<double>& f, std::vector<double>& s);

// Hermite evaluation of f, f', f'' at x inside segment k (host copy of the
// device evaluator; used for per-launch constants).
void spline_eval(const std::vector<double>& x, const std::vector<double>& f, const std::vector<double>& s,
                 double z, double& val, double& d1, double& d2);

// Reads a .met profile like set_region (atmo_io.3d.strat.cpp:55-143):
// formats zTuvdp / zuvwTdp / zcuvd, '#' comment lines, pressure and density
// converted to c = sqrt(0.1 gamma p / rho) / 1000 km/s, winds m/s -> km/s
// (negated when reverse_winds).  Returns 0 or a negative iga_status.
int load_met(const char* path, const char* format, bool reverse_winds, StratProfile& out, std::string& err);

// Builds slopes and the device table from z/c/u/v/rho already set.
int finalize_profile(StratProfile& p, std::string& err);

}  // namespace iga
