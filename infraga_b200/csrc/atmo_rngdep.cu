// Host side of the range-dependent atmosphere and terrain (atmo_rngdep.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/infraga_gpu.h"
#include "atmo_host.h"
#include "atmo_rngdep.h"
#include "device_common.cuh"
#include "rngdep_eval.cuh"

namespace iga {

namespace {

// file_length (fileIO.cpp:18-35): lines not starting with '#', counting the
// empty read after a final newline, minus one.
int file_length(const char* path) {
    std::ifstream in(path);
    if (!in.is_open()) return -1;
    std::string line;
    int n = 0;
    while (!in.eof()) {
        std::getline(in, line);
        if (line.find('#') != 0) n++;
    }
    return n - 1;
}

int read_list(const char* path, int n, bool degrees, std::vector<double>& out, std::string& err) {
    std::ifstream in(path);
    if (!in.is_open()) { err = std::string("cannot open '") + path + "'"; return IGA_E_IO; }
    out.resize(n);
    for (int i = 0; i < n; i++) {
        if (!(in >> out[i])) { err = std::string("'") + path + "': expected " + std::to_string(n) + " values"; return IGA_E_IO; }
        if (degrees) out[i] *= kPi / 180.0;
    }
    for (int i = 0; i + 1 < n; i++)
        if (!(out[i + 1] > out[i])) { err = std::string("'") + path + "': node coordinates must increase"; return IGA_E_IO; }
    return IGA_OK;
}

// clamped central-difference neighbours (interp::set and finite_diff_*,
// interpolation.cpp:976-980, 1188-1196)
inline int up(int i, int n) { return i + 1 < n ? i + 1 : n - 1; }
inline int dn(int i) { return i > 0 ? i - 1 : 0; }

}  // namespace

int load_rngdep(const char* prefix, const char* lat_file, const char* lon_file, const char* format,
                bool reverse_winds, bool degrees, RngdepGrid& g, std::string& err) {
    const int nx = file_length(lat_file), ny = file_length(lon_file);
    if (nx < 2 || ny < 2) { err = "latitude/longitude node lists need at least 2 entries each"; return IGA_E_IO; }
    g = RngdepGrid();
    int rc = read_list(lat_file, nx, degrees, g.x, err);
    if (rc) return rc;
    if ((rc = read_list(lon_file, ny, degrees, g.y, err))) return rc;
    g.nx = nx; g.ny = ny;
    for (int ix = 0; ix < nx; ix++) {
        for (int iy = 0; iy < ny; iy++) {
            const std::string path = std::string(prefix) + std::to_string(ix * ny + iy) + ".met";
            StratProfile p;
            rc = load_met(path.c_str(), format, reverse_winds, p, err);
            if (rc) return rc;
            if (ix == 0 && iy == 0) {
                g.nz = (int)p.z.size();
                g.z = p.z;
                for (auto& f : g.f) f.assign((size_t)nx * ny * g.nz, 0.0);
            } else if ((int)p.z.size() != g.nz || p.z != g.z) {
                err = "node profile '" + path + "' has altitudes different from node 0";
                return IGA_E_IO;
            }
            const size_t o = ((size_t)ix * ny + iy) * g.nz;
            for (int k = 0; k < g.nz; k++) {
                g.f[0][o + k] = p.c[k]; g.f[1][o + k] = p.u[k];
                g.f[2][o + k] = p.v[k]; g.f[3][o + k] = p.rho[k];
            }
        }
    }
    build_hybrid_table(g);
    return IGA_OK;
}

void build_hybrid_table(RngdepGrid& g) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const size_t nn = (size_t)nx * ny;
    auto at = [&](int ix, int iy) { return ((size_t)ix * ny + iy) * nz; };
    g.table.assign(nn * nz * kHybRec, 0.0);
    std::vector<double> col(nz), sl(nz);
    for (int fld = 0; fld < 4; fld++) {
        const std::vector<double>& F = g.f[fld];
        // vertical slopes of f at every node (set, interpolation.cpp:920-955)
        std::vector<double> FS(nn * nz), P1v(nn * nz), P2v(nn * nz), D(nn * nz);
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                std::vector<double> fcol(F.begin() + at(ix, iy), F.begin() + at(ix, iy) + nz);
                natural_spline_slopes(g.z, fcol, sl);
                std::copy(sl.begin(), sl.end(), FS.begin() + at(ix, iy));
            }
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int xu = up(ix, nx), xd = dn(ix), yu = up(iy, ny), yd = dn(iy);
                const double hx = g.x[xu] - g.x[xd], hy = g.y[yu] - g.y[yd];
                for (int k = 0; k < nz; k++) {
                    P1v[at(ix, iy) + k] = (F[at(xu, iy) + k] - F[at(xd, iy) + k]) / hx;
                    P2v[at(ix, iy) + k] = (F[at(ix, yu) + k] - F[at(ix, yd) + k]) / hy;
                }
                // dfdx_slopes: natural spline in z of the x-difference (interpolation.cpp:968-1005)
                for (int k = 0; k < nz; k++) col[k] = P1v[at(ix, iy) + k];
                natural_spline_slopes(g.z, col, sl);
                std::copy(sl.begin(), sl.end(), D.begin() + at(ix, iy));
            }
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                const int xu = up(ix, nx), xd = dn(ix), yu = up(iy, ny), yd = dn(iy);
                const double hx = g.x[xu] - g.x[xd], hy = g.y[yu] - g.y[yd], hxy = hx * hy;
                for (int k = 0; k < nz; k++) {
                    double* r = &g.table[(at(ix, iy) + k) * kHybRec];
                    const size_t c = at(ix, iy) + k;
                    const size_t uu = at(xu, yu) + k, ud = at(xu, yd) + k, du = at(xd, yu) + k, dd = at(xd, yd) + k;
                    double* p = r + fld * kHybP;
                    p[0] = F[c];
                    p[1] = FS[c];
                    p[2] = P1v[c];
                    p[3] = (FS[at(xu, iy) + k] - FS[at(xd, iy) + k]) / hx;
                    p[4] = P2v[c];
                    p[5] = (FS[at(ix, yu) + k] - FS[at(ix, yd) + k]) / hy;
                    p[6] = (F[uu] - F[ud] - F[du] + F[dd]) / hxy;
                    p[7] = (FS[uu] - FS[ud] - FS[du] + FS[dd]) / hxy;
                    if (fld < 3) {
                        double* x = r + kHybXOff + fld * kHybX;
                        x[0] = D[c];
                        // Q = (P1v, D): FDx Q and FDxy Q
                        x[1] = (P1v[at(xu, iy) + k] - P1v[at(xd, iy) + k]) / hx;
                        x[2] = (D[at(xu, iy) + k] - D[at(xd, iy) + k]) / hx;
                        x[3] = (P1v[uu] - P1v[ud] - P1v[du] + P1v[dd]) / hxy;
                        x[4] = (D[uu] - D[ud] - D[du] + D[dd]) / hxy;
                        // R = (P2v, D): FDy R and FDxy R
                        x[5] = (P2v[at(ix, yu) + k] - P2v[at(ix, yd) + k]) / hy;
                        x[6] = (D[at(ix, yu) + k] - D[at(ix, yd) + k]) / hy;
                        x[7] = (P2v[uu] - P2v[ud] - P2v[du] + P2v[dd]) / hxy;
                        x[8] = (D[uu] - D[ud] - D[du] + D[dd]) / hxy;
                    }
                }
            }
    }
}

int load_terrain(const char* path, bool degrees, Terrain& t, std::string& err) {
    // file_2d_dims: N rows; n_lon = index of the first row whose lon decreases
    const int N = file_length(path);
    std::ifstream in(path);
    if (N < 4 || !in.is_open()) { err = std::string("cannot read terrain file '") + path + "'"; return IGA_E_IO; }
    std::vector<double> a((size_t)N * 3);
    for (int i = 0; i < N; i++) {
        if (!(in >> a[3 * i] >> a[3 * i + 1] >> a[3 * i + 2])) {
            err = std::string("terrain file '") + path + "': expected lat lon z rows";
            return IGA_E_IO;
        }
    }
    int ny = N;
    for (int n = 1; n < N; n++)
        if (a[3 * n + 1] < a[3 * (n - 1) + 1]) { ny = n; break; }
    const int nx = N / ny;
    if (nx < 2 || ny < 2 || nx * ny != N) { err = std::string("terrain file '") + path + "' is not a full lat x lon grid"; return IGA_E_IO; }
    t = Terrain();
    t.nx = nx; t.ny = ny;
    t.x.resize(nx); t.y.resize(ny); t.f.resize((size_t)N);
    // set_region reads x, y and f row by row (atmo_io.sph.rngdep.cpp:217-223)
    for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny; iy++) {
            const double* r = &a[3 * ((size_t)ix * ny + iy)];
            t.x[ix] = degrees ? r[0] * (kPi / 180.0) : r[0];
            t.y[iy] = degrees ? r[1] * (kPi / 180.0) : r[1];
            t.f[(size_t)ix * ny + iy] = r[2];
        }
    for (int i = 0; i + 1 < nx; i++) if (!(t.x[i + 1] > t.x[i])) { err = "terrain latitudes must increase"; return IGA_E_IO; }
    for (int i = 0; i + 1 < ny; i++) if (!(t.y[i + 1] > t.y[i])) { err = "terrain longitudes must increase"; return IGA_E_IO; }
    t.z_max = 0.0;   // topo::set_bndlyr starts from 0 (atmo_state.sph.rngdep.cpp:24-31)
    for (double v : t.f) t.z_max = std::max(t.z_max, v);
    build_terrain_table(t);
    return IGA_OK;
}

void build_terrain_table(Terrain& t) {
    const int nx = t.nx, ny = t.ny;
    std::vector<double> fy((size_t)nx * ny), fx((size_t)nx * ny), fxy((size_t)nx * ny);
    std::vector<double> row(ny), rs(ny), col(nx), cs(nx);
    for (int ix = 0; ix < nx; ix++) {   // natural spline in lon per lat row (interp::set 2D)
        for (int iy = 0; iy < ny; iy++) row[iy] = t.f[(size_t)ix * ny + iy];
        natural_spline_slopes(t.y, row, rs);
        for (int iy = 0; iy < ny; iy++) fy[(size_t)ix * ny + iy] = rs[iy];
    }
    for (int iy = 0; iy < ny; iy++) {   // natural splines in lat of f and of f_lon (set_node_slopes)
        for (int ix = 0; ix < nx; ix++) col[ix] = t.f[(size_t)ix * ny + iy];
        natural_spline_slopes(t.x, col, cs);
        for (int ix = 0; ix < nx; ix++) fx[(size_t)ix * ny + iy] = cs[ix];
        for (int ix = 0; ix < nx; ix++) col[ix] = fy[(size_t)ix * ny + iy];
        natural_spline_slopes(t.x, col, cs);
        for (int ix = 0; ix < nx; ix++) fxy[(size_t)ix * ny + iy] = cs[ix];
    }
    t.table.resize((size_t)nx * ny * 4);
    for (size_t i = 0; i < (size_t)nx * ny; i++) {
        t.table[4 * i] = t.f[i]; t.table[4 * i + 1] = fx[i];
        t.table[4 * i + 2] = fy[i]; t.table[4 * i + 3] = fxy[i];
    }
}

void hybrid_eval1(const RngdepGrid& g, int fld, double lat, double lon, double z, double& f, double df[3]) {
    HybView v{g.table.data(), g.x.data(), g.y.data(), g.z.data(), g.nx, g.ny, g.nz};
    HybLoc L;
    int cx = 0, cy = 0, cz = 0;
    hyb_locate(v, lat, lon, z, L, cx, cy, cz);
    HybF1 o;
    hyb_f1(v, L, fld, o);
    f = o.f;
    df[0] = o.d[0]; df[1] = o.d[1]; df[2] = o.d[2];
}

void terrain_eval1(const Terrain& t, double lat, double lon, double& z, double dz[2]) {
    TopoView v{t.table.data(), t.x.data(), t.y.data(), t.nx, t.ny};
    TopoVal o;
    int cx = 0, cy = 0;
    topo_eval(v, lat, lon, 1, o, cx, cy);
    z = o.z;
    dz[0] = o.d[0]; dz[1] = o.d[1];
}

}  // namespace iga
