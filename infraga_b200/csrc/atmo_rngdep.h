// Host-side range-dependent atmosphere and terrain: file loading and the
// device node tables.
//
// Range-dependent atmosphere (interp::hybrid_spline_3D,
// src/util/interpolation.cpp:886-1788).  The reference evaluates, at a point
// (lat, lon, z), natural cubic splines in z at the nodes of a 4x4..6x6
// horizontal stencil, forms central finite differences across nodes and
// feeds corner values and differences into a bicubic patch, separately for
// f, df/dz, d2f/dz2, df/dx (for d2f/dx2) and df/dy (for d2f/dy2).  Every one
// of those node quantities is a linear combination of node splines, so it is
// itself a cubic Hermite spline in z whose knot values and slopes are the
// same linear combination of the node knot values and slopes.  The tables
// below store those combined knots per node, so that an evaluation reads
// only the 4 corner nodes of its cell (two z knots each) instead of the
// 36-node stencil, with the reference's arithmetic up to rounding order.
//
// Terrain (interp::natural_cubic_spline_2D, interpolation.cpp:266-680) is a
// natural spline in lon per lat row followed, per evaluation, by a natural
// spline in lat through the row values.  That is the tensor-product natural
// bicubic spline, fixed by f, f_lat, f_lon and f_lat,lon at the nodes; those
// are precomputed here and evaluated as a bicubic Hermite patch.
#pragma once
#include <string>
#include <vector>

namespace iga {

// Per (lat node, lon node, z knot) record of the hybrid table (doubles).
// Value/slope pairs of node splines in z, for fields c, u, v, rho:
//   P0 = f, P1 = FDx f, P2 = FDy f, P3 = FDxy f      (all four fields)
// and, for c, u, v only (second derivatives):
//   D  = dfdx_slopes (slope of the node's df/dx spline; the reference's
//        eval_node_dfdy uses the same slopes, interpolation.cpp:1118-1119)
//   Q1 = FDx Q, Q3 = FDxy Q   with Q = (FDx f values, D slopes)
//   R2 = FDy R, R3 = FDxy R   with R = (FDy f values, D slopes)
// FD* are the reference's clamped central differences across nodes.
constexpr int kHybP = 8;                 // P0v P0s P1v P1s P2v P2s P3v P3s
constexpr int kHybX = 9;                 // D Q1v Q1s Q3v Q3s R2v R2s R3v R3s
constexpr int kHybRec = 64;              // 4 * kHybP (c u v rho) + 3 * kHybX, padded
constexpr int kHybXOff = 4 * kHybP;      // first extra block (c), then u, v

struct RngdepGrid {
    int nx = 0, ny = 0, nz = 0;                 // latitude, longitude, altitude counts
    std::vector<double> x, y, z;                // lat, lon [rad] (or x, y [km]), z [km]
    std::vector<double> f[4];                   // c, u, v, rho at [(ix * ny + iy) * nz + iz]
    std::vector<double> table;                  // nx * ny * nz * kHybRec
};

struct Terrain {
    int nx = 0, ny = 0;
    std::vector<double> x, y;                   // lat, lon [rad] (or x, y [km])
    std::vector<double> f;                      // [ix * ny + iy] km
    std::vector<double> table;                  // nx * ny * 4: f, f_x, f_y, f_xy
    double z_max = 0.0;                         // max node height
};

// set_region for the range-dependent solvers (atmo_io.sph.rngdep.cpp:61-188,
// atmo_io.3d.rngdep.cpp:58-190): node coordinate lists (latitude/longitude in
// degrees when `degrees`, else x/y in km), node profiles {prefix}{n}.met with
// n = i_x * n_y + i_y, same columns and conversions as the 1D loader.
int load_rngdep(const char* prefix, const char* lat_file, const char* lon_file, const char* format,
                bool reverse_winds, bool degrees, RngdepGrid& g, std::string& err);

// Terrain file of rows "lat lon z" (deg, deg, km; or "x y z" in km when not
// `degrees`), first coordinate major (atmo_io.sph.rngdep.cpp:205-225,
// atmo_io.3d.rngdep.cpp:205-223, file_2d_dims fileIO.cpp:64-85).
int load_terrain(const char* path, bool degrees, Terrain& t, std::string& err);

void build_hybrid_table(RngdepGrid& g);
void build_terrain_table(Terrain& t);

// Host evaluation (per-launch constants at the source and the ground):
// f and first derivatives (d/dlat, d/dlon, d/dz) of field `fld` (0 c, 1 u,
// 2 v, 3 rho) with the reference's clamping of lat, lon, z.
void hybrid_eval1(const RngdepGrid& g, int fld, double lat, double lon, double z, double& f, double df[3]);
// terrain height and gradient (d/dlat, d/dlon) at (lat, lon)
void terrain_eval1(const Terrain& t, double lat, double lon, double& z, double dz[2]);

}  // namespace iga
