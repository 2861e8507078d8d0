// CPU oracle (test infrastructure only; never linked into the product).
//
// Restatement of the reference's stratified profile reader:
//   file_length      src/util/fileIO.cpp:18-35
//   set_region       src/atmo/atmo_io.3d.strat.cpp:55-143 (same parser in
//                    atmo_io.sph.strat.cpp for the spherical solver)
#pragma once
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include "oracle_spline.h"

namespace orc {

constexpr double kPi = 3.141592653589793238462643;   // geoac.params.3d.cpp:10
constexpr double kGam = 1.4;                         // atmo_state.3d.strat.cpp:25
constexpr double kR = 287.058;                       // atmo_state.3d.strat.cpp:26

// file_length (fileIO.cpp:18-35): lines not starting with '#', minus one.
inline int file_length(const char* path) {
    std::ifstream in(path);
    if (!in.is_open()) return 0;
    int count = 0;
    std::string line;
    while (!in.eof()) {
        std::getline(in, line);
        if (line.find("#") != 0) count++;
    }
    return count - 1;
}

struct Profile {
    Spline1D c, u, v, rho;
};

// set_region (atmo_io.3d.strat.cpp:55-143) without the terrain branch.
// Returns 0 on error, like the reference.
inline int load_profile(const char* path, const char* fmt, bool invert_winds, Profile& P) {
    const int L = file_length(path);
    if (L < 2) return 0;
    Spline1D* all[4] = {&P.c, &P.u, &P.v, &P.rho};
    for (auto* s : all) { s->n = L; s->x.assign(L, 0.0); s->f.assign(L, 0.0); }
    std::ifstream in(path);
    if (!in.is_open()) return 0;
    int n = 0;
    double temp;
    std::string line;
    while (!in.eof() && n < L) {
        std::getline(in, line);
        if (line.find("#") == 0) continue;
        std::stringstream ss(line);
        if (strncmp(fmt, "zTuvdp", 6) == 0) {
            ss >> P.c.x[n] >> temp >> P.u.f[n] >> P.v.f[n] >> P.rho.f[n] >> P.c.f[n];
        } else if (strncmp(fmt, "zuvwTdp", 7) == 0) {
            ss >> P.c.x[n] >> P.u.f[n] >> P.v.f[n] >> temp >> temp >> P.rho.f[n] >> P.c.f[n];
        } else if (strncmp(fmt, "zcuvd", 5) == 0) {
            ss >> P.c.x[n] >> P.c.f[n] >> P.u.f[n] >> P.v.f[n] >> P.rho.f[n];
        } else {
            return 0;
        }
        P.u.x[n] = P.c.x[n]; P.v.x[n] = P.c.x[n]; P.rho.x[n] = P.c.x[n];
        if (strncmp(fmt, "zTuvdp", 6) == 0 || strncmp(fmt, "zuvwTdp", 7) == 0)
            P.c.f[n] = sqrt(0.1 * kGam * P.c.f[n] / P.rho.f[n]) / 1000.0;
        else
            P.c.f[n] /= 1000.0;
        if (invert_winds) { P.u.f[n] /= -1000.0; P.v.f[n] /= -1000.0; }
        else { P.u.f[n] /= 1000.0; P.v.f[n] /= 1000.0; }
        n++;
    }
    spline_set(P.c); spline_set(P.u); spline_set(P.rho); spline_set(P.v);
    return 1;
}

}  // namespace orc
