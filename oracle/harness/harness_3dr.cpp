// Full-precision driver around the reference's own 3D Cartesian range-
// dependent solver (hybrid 3D atmosphere splines, optional terrain).
//
// Test infrastructure only (oracle): compiled together with the reference's
// unmodified sources for infraga-3d-rngdep (see oracle/Makefile) and replaces
// only its command-line front end (src/main.infraga.3d.rngdep.cpp), so that
// arrivals come out with 17 significant digits and every RK4 step is counted.
//
//   prop mode  follows run_prop  (src/main.infraga.3d.rngdep.cpp:204-535)
//
//   iga_ref_3dr prop <prefix> <x_file> <y_file> key=value...
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <iostream>
#include <fstream>
#include <algorithm>

#include "atmo/atmo_state.h"
#include "atmo/atmo_io.3d.rngdep.h"
#include "geoac/geoac.params.h"
#include "geoac/geoac.eqset.h"
#include "geoac/geoac.interface.h"
#include "util/fileIO.h"
#include "util/rk4solver.h"
#include "util/interpolation.h"

using namespace std;

static long long g_steps = 0;
extern "C" int __real__ZN5geoac8prop_rk4ERPPdRbi(double**& sol, bool& check, int length);
extern "C" int __wrap__ZN5geoac8prop_rk4ERPPdRbi(double**& sol, bool& check, int length) {
    int k = __real__ZN5geoac8prop_rk4ERPPdRbi(sol, check, length);
    g_steps += k;
    return k;
}

static double now_s() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static bool key(const char* arg, const char* k, const char** val) {
    size_t n = strlen(k);
    if (strncmp(arg, k, n) == 0) { *val = arg + n; return true; }
    return false;
}

static int run_prop(int argc, char** argv) {
    double theta_min = 0.5, theta_max = 45.0, theta_step = 0.5;
    double phi_min = -90.0, phi_max = -90.0, phi_step = 1.0;
    int bounces = 10;
    double x_src, y_src, z_src = 0.0;
    bool write_rays = true;   // only selects the per-step (k-1 segment) accumulation
    double freq = 0.1, turn_ht_min = 0.2;
    const char* prof_format = "zTuvdp";
    const char* topo_file = "None";
    const char* v;

    topo::z0 = 0.0;
    atmo::tweak_abs = 1.0;
    geoac::calc_amp = true;
    geoac::is_topo = false;

    for (int i = 5; i < argc; i++) {
        if (key(argv[i], "prof_format=", &v)) prof_format = v;
        else if (key(argv[i], "z_grnd=", &v)) topo::z0 = atof(v);
        else if (key(argv[i], "topo_file=", &v)) { topo_file = v; geoac::is_topo = true; }
    }
    int ok = geoac::is_topo ? set_region(argv[2], argv[3], argv[4], (char*)topo_file, (char*)prof_format, false)
                            : set_region(argv[2], argv[3], argv[4], (char*)prof_format, false);
    if (!ok) return 1;
    x_src = (geoac::x_max + geoac::x_min) / 2.0;
    y_src = (geoac::y_max + geoac::y_min) / 2.0;

    for (int i = 5; i < argc; i++) {
        const char* a = argv[i];
        if (key(a, "incl_min=", &v)) theta_min = atof(v);
        else if (key(a, "incl_max=", &v)) theta_max = atof(v);
        else if (key(a, "incl_step=", &v)) theta_step = atof(v);
        else if (key(a, "az_min=", &v)) phi_min = atof(v);
        else if (key(a, "az_max=", &v)) phi_max = atof(v);
        else if (key(a, "az_step=", &v)) phi_step = atof(v);
        else if (key(a, "inclination=", &v)) { theta_min = theta_max = atof(v); theta_step = 1.0; }
        else if (key(a, "azimuth=", &v)) { phi_min = phi_max = atof(v); phi_step = 1.0; }
        else if (key(a, "bounces=", &v)) bounces = atoi(v);
        else if (key(a, "src_x=", &v)) x_src = atof(v);
        else if (key(a, "src_y=", &v)) y_src = atof(v);
        else if (key(a, "src_alt=", &v)) z_src = atof(v);
        else if (key(a, "turn_ht_min=", &v)) turn_ht_min = atof(v);
        else if (key(a, "write_rays=", &v)) write_rays = string2bool(v);
        else if (key(a, "freq=", &v)) freq = atof(v);
        else if (key(a, "abs_coeff=", &v)) atmo::tweak_abs = max(0.0, atof(v));
        else if (key(a, "calc_amp=", &v)) geoac::calc_amp = string2bool(v);
        else if (key(a, "max_alt=", &v)) geoac::alt_max = atof(v);
        else if (key(a, "max_rng=", &v)) geoac::rng_max = atof(v);
        else if (key(a, "min_x=", &v)) geoac::x_min = atof(v);
        else if (key(a, "max_x=", &v)) geoac::x_max = atof(v);
        else if (key(a, "min_y=", &v)) geoac::y_min = atof(v);
        else if (key(a, "max_y=", &v)) geoac::y_max = atof(v);
        else if (key(a, "min_ds=", &v)) geoac::ds_min = atof(v);
        else if (key(a, "max_ds=", &v)) geoac::ds_max = atof(v);
        else if (key(a, "max_s=", &v)) geoac::s_max = atof(v);
        else if (key(a, "z_grnd=", &v)) {
            if (!geoac::is_topo) { topo::z0 = atof(v); topo::z_max = topo::z0; topo::z_bndlyr = topo::z0 + 2.0; }
        }
        else if (key(a, "prof_format=", &v) || key(a, "topo_file=", &v)) {}
        else { fprintf(stderr, "harness: unknown key %s\n", a); return 2; }
    }
    z_src = max(z_src, topo::z(x_src, y_src));
    geoac::configure();

    double travel_time_sum, attenuation, z_max;
    int k, length = int(geoac::s_max / geoac::ds_min);
    bool break_check;
    double** solution;
    geoac::build_solution(solution, length);
    long long n_rays = 0;
    double t0 = now_s();

    for (double phi = phi_min; phi <= phi_max; phi += phi_step) {
        geoac::phi = Pi / 2.0 - phi * Pi / 180.0;
        double theta_grnd;
        if (z_src - topo::z(x_src, y_src) < 0.01) {
            if (geoac::is_topo)
                theta_grnd = atan(topo::dz(x_src, y_src, 0) * sin(phi * Pi / 180.0) + topo::dz(x_src, y_src, 1) * cos(phi * Pi / 180.0)) * (180.0 / Pi) + 0.1;
            else
                theta_grnd = 0.1;
        } else {
            theta_grnd = -89.9;
        }
        for (double theta = max(theta_min, theta_grnd); theta <= max(theta_max, theta_grnd); theta += theta_step) {
            geoac::theta = theta * Pi / 180.0;
            geoac::set_initial(solution, x_src, y_src, z_src);
            travel_time_sum = 0.0;
            attenuation = 0.0;
            z_max = 0.0;
            long long steps_before = g_steps;
            n_rays++;
            for (int bnc_cnt = 0; bnc_cnt <= bounces; bnc_cnt++) {
                k = geoac::prop_rk4(solution, break_check, length);
                if (write_rays) {
                    for (int m = 1; m < k; m++) {
                        geoac::travel_time(travel_time_sum, solution, m - 1, m);
                        geoac::atten(attenuation, solution, m - 1, m, freq);
                    }
                } else {
                    travel_time_sum += geoac::travel_time(solution, k);
                    attenuation += geoac::atten(solution, k, freq);
                }
                for (int m = 0; m < k; m++) z_max = max(z_max, solution[m][2]);
                if (!geoac::is_topo && z_max < (topo::z0 + turn_ht_min)) break;
                if (break_check || k < 2) break;

                double inclination = -asin(atmo::c(solution[k][0], solution[k][1], topo::z(solution[k][0], solution[k][1])) / atmo::c(x_src, y_src, z_src) * solution[k][5]) * 180.0 / Pi;
                double back_az = 90.0 - atan2(-solution[k][4], -solution[k][3]) * 180.0 / Pi;
                if (back_az < -180.0) back_az += 360.0;
                else if (back_az > 180.0) back_az -= 360.0;

                printf("%.17g\t%.17g\t%d\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\t%.17g\n",
                       theta, phi, bnc_cnt, solution[k][0], solution[k][1], travel_time_sum,
                       sqrt(pow(solution[k][0] - x_src, 2) + pow(solution[k][1] - y_src, 2)) / travel_time_sum,
                       z_max, inclination, back_az,
                       geoac::calc_amp ? 20.0 * log10(geoac::amp(solution, k)) : 0.0,
                       -2.0 * attenuation);
                geoac::set_refl(solution, k);
            }
            printf("R\t%.17g\t%.17g\t%lld\n", theta, phi, g_steps - steps_before);
            geoac::clear_solution(solution, k);
        }
    }
    double t1 = now_s();
    printf("# rays %lld steps %lld elapsed_s %.6f\n", n_rays, g_steps, t1 - t0);
    printf("# src %.17g %.17g %.17g\n", x_src, y_src, z_src);
    geoac::delete_solution(solution, length);
    clear_region();
    return 0;
}

int main(int argc, char** argv) {
    cout.setstate(ios::failbit);   // silence the reference's progress banners on stdout
    if (argc < 5) { fprintf(stderr, "usage: %s prop <prefix> <x_file> <y_file> key=value...\n", argv[0]); return 2; }
    if (strcmp(argv[1], "prop") == 0) return run_prop(argc, argv);
    fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
}
