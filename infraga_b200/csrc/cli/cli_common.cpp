// Drop-in command-line front ends over libinfraga_gpu.so (see cli_common.h).
//
// Output formats follow the reference mains line for line, because files
// written by these binaries are read by the same downstream tools
// (infraga/run_infraga.py, plotting scripts): header text and column order
// of run_prop (src/main.infraga.3d.cpp:348-402, main.infraga.sph.cpp:357-411,
// main.infraga.3d.rngdep.cpp:141-197, main.infraga.sph.rngdep.cpp:149-205)
// and of run_eig_search / find_eigenray (main.infraga.3d.cpp:893-936,
// src/geoac/geoac.eigenray.3d.cpp:220-318), written through std::ofstream
// with the same precision manipulators so numbers print identically
// (spherical rows switch their stream to 8 significant digits at the first
// latitude and keep it, as the reference streams do).
#include "cli_common.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <algorithm>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "infraga_gpu.h"

namespace cli {
namespace {

constexpr double Pi = 3.141592653589793238462643;   // geoac.params.3d.cpp:9
constexpr double kR0 = 6370.0;                       // globe::r0 (util/globe.cpp:10)

// strncmp(arg, key, n) == 0, value at arg + off (the reference's matching,
// including its few keys whose compare length or value offset is off by some
// characters).
bool match(const char* a, const char* k, size_t n, size_t off, const char** v) {
    if (strncmp(a, k, n) != 0) return false;
    *v = a + off;
    return true;
}
bool key(const char* a, const char* k, const char** v) { return match(a, k, strlen(k), strlen(k), v); }
bool key2(const char* a, const char* k1, const char* k2, const char** v) { return key(a, k1, v) || key(a, k2, v); }

// util/fileIO.cpp:87-90
bool str2bool(const char* s) { return s[0] != '\0' && (strcasecmp(s, "true") == 0 || atoi(s) != 0); }

bool confirm_unknown(const char* arg, bool leading_newline) {
    if (leading_newline) std::cout << '\n';
    std::cout << "***WARNING*** Unrecognized parameter entry: " << arg << '\n';
    std::cout << "Continue? (y/n):";
    char c = 0;
    std::cin >> c;
    return c == 'y' || c == 'Y';
}

// The reference cuts the profile argument at its last '.' in place, so the
// ".arrivals.dat" header's "profile:" line shows the shortened text too.
void strip_extension(char* s) {
    for (int m = (int)strlen(s); m >= 0; m--)
        if (s[m] == '.') {
            s[m] = '\0';
            break;
        }
}

// How the binary was started: its reference name (the serial one or the MPI
// build's infraga-accel-* name) and, under mpirun, the process count the
// reference's MPI summaries print as "threads".
struct Launch {
    bool accel = false;
    int threads = 1;
};
Launch g_launch;

// Rank and size of an MPI launch, from the variables the common launchers set
// (Open MPI, MPICH / Hydra, PMIx, Slurm); 0 and 1 without one.
int env_int(const char* const* names, int dflt) {
    for (const char* const* n = names; *n; n++) {
        const char* v = getenv(*n);
        if (v && v[0]) return atoi(v);
    }
    return dflt;
}
int launch_rank() {
    static const char* const k[] = {"OMPI_COMM_WORLD_RANK", "PMI_RANK", "PMIX_RANK", "MV2_COMM_WORLD_RANK", "SLURM_PROCID", nullptr};
    return env_int(k, 0);
}
int launch_size() {
    static const char* const k[] = {"OMPI_COMM_WORLD_SIZE", "PMI_SIZE", "MV2_COMM_WORLD_SIZE", "SLURM_NTASKS", nullptr};
    return std::max(1, env_int(k, 1));
}

const char* variant_name(Variant v) {
    if (g_launch.accel) {
        switch (v) {
            case Variant::k3D: return "infraga-accel-3d";
            case Variant::kSph: return "infraga-accel-sph";
            case Variant::k3DRngdep: return "infraga-accel-3d-rngdep";
            default: return "infraga-accel-sph-rngdep";
        }
    }
    switch (v) {
        case Variant::k3D: return "infraga-3d";
        case Variant::kSph: return "infraga-sph";
        case Variant::k3DRngdep: return "infraga-3d-rngdep";
        default: return "infraga-sph-rngdep";
    }
}

// The MPI builds' summaries end with the process count (main.infraga.3d.mpi.cpp:322, :868).
void threads_line(std::ostream& f, const char* lead) {
    if (g_launch.accel) f << lead << '\t' << "threads: " << g_launch.threads << '\n';
}

bool is_sph(Variant v) { return v == Variant::kSph || v == Variant::kSphRngdep; }
bool is_rngdep(Variant v) { return v == Variant::k3DRngdep || v == Variant::kSphRngdep; }

int fail(const char* what, int rc) {
    std::cout << '\t' << "ERROR: " << what << ": " << iga_strerror(rc);
    const char* ce = iga_last_cuda_error();
    if (ce && ce[0]) std::cout << " (" << ce << ")";
    std::cout << '\n';
    return 0;   // the reference exits 0 after its error messages
}

void banner(Variant v, const char* mode) {
    const std::string name = std::string("Running ") + variant_name(v);
    const int w = (int)std::max(name.size(), strlen(mode)) + 10;
    auto line = [&](const std::string& t) {
        const int pad = w - 8 - (int)t.size();
        std::cout << '\t' << "####" << std::string(pad / 2, ' ') << t << std::string(pad - pad / 2, ' ') << "####" << '\n';
    };
    std::cout << '\n' << '\t' << std::string(w, '#') << '\n';
    line(name);
    line(mode);
    std::cout << '\t' << std::string(w, '#') << '\n' << '\n';
}

void usage(Variant v) {
    const char* n = variant_name(v);
    const bool sph = is_sph(v), rd = is_rngdep(v);
    std::cout << '\n' << "Usage: " << n << " [option] " << (rd ? "prefix x_or_lat_file y_or_lon_file" : "profile.met")
              << " [parameters]" << '\n';
    std::cout << '\t' << "GPU (B200) ray tracing through "
              << (rd ? "a range-dependent" : "a stratified") << ", moving medium"
              << (sph ? " on the globe" : " (3D Cartesian)") << "; output files match the reference " << n << ".\n\n";
    std::cout << "Options:" << '\n';
    std::cout << '\t' << "-prop        ray fan over inclination/azimuth ranges (incl_min, incl_max, incl_step, az_min, az_max,"
              << '\n' << '\t' << "             az_step, inclination, azimuth, bounces, " << (sph ? "src_lat, src_lon" : "src_x, src_y")
              << ", src_alt, turn_ht_min, write_rays, write_caustics, write_topo)" << '\n';
    std::cout << '\t' << "-eig_search  eigenrays from " << (sph ? "(src_lat, src_lon, src_alt) to (rcvr_lat, rcvr_lon)"
                                                                   : "(src_x, src_y, src_alt) to (rcvr_x, rcvr_y)")
              << " (incl_min, incl_max, bnc_min,"
              << '\n' << '\t' << "             bnc_max, bounces, verbose, iterations, damping, tolerance, az_dev_lim, incl_step_min,"
              << '\n' << '\t' << "             incl_step_max)" << '\n';
    std::cout << '\t' << "-eig_direct  one eigenray near (incl_est, az_est) with a given bounce count" << '\n';
    std::cout << '\t' << "Common: freq, abs_coeff, z_grnd, prof_format, reverse_winds, output_id, calc_amp, max_alt, max_rng,"
              << '\n' << '\t' << "        " << (sph ? "min_lat, max_lat, min_lon, max_lon, max_time" : "min_x, max_x, min_y, max_y")
              << ", min_ds, max_ds, max_s, topo_file" << '\n';
    const bool back = v == Variant::k3D || v == Variant::k3DRngdep;
    if (back)
        std::cout << '\t' << "-back_proj   one ray from (rcvr_x, rcvr_y) at (inclination, azimuth) through the reversed"
                  << " winds (bounces)" << '\n';
    std::cout << '\t' << (back ? "" : "-back_proj, ")
              << (v == Variant::k3D || v == Variant::kSph ? "" : "-wnl_wvfrm, ")
              << "the reference's MPI builds are not provided by the GPU front end." << '\n' << '\n';
}

void version() {
    std::cout << '\n' << '\t' << "infraga-gpu: B200 ray-fan and eigenray solver with the infraga 1.0.3 command-line interface"
              << '\n' << '\t' << "C ABI version " << iga_version() << '\n' << '\n';
}

// ------------------------------------------------------------------------
// -prop
// ------------------------------------------------------------------------

struct PropOpts {
    double theta_min = 0.5, theta_max = 45.0, theta_step = 0.5;
    double phi_min = -90.0, phi_max = -90.0, phi_step = 1.0;
    bool write_atmo = false, write_rays = true, write_caustics = false, write_topo = false;
    bool print_resid = false, use_blw = false;
    const char* output_id = nullptr;
    const char* topo_file = nullptr;
};

// Loads the atmosphere of argv (first pass: prof_format, reverse_winds,
// topo_file; z_grnd there is overwritten by set_limits) and prints set_region's
// messages.  Returns null on failure (messages printed).
iga_atmo_t load_atmosphere(Variant v, int argc, char** argv, const char** topo_out, bool force_rev = false) {
    const int first = is_rngdep(v) ? 5 : 3;
    const char* fmt = "zTuvdp";
    const char* topo = nullptr;
    bool rev = force_rev;
    const char* val;
    for (int i = first; i < argc; i++) {
        if (key(argv[i], "prof_format=", &val)) fmt = val;
        else if (key(argv[i], "z_grnd=", &val)) {}
        else if (key(argv[i], "reverse_winds=", &val)) rev = str2bool(val);
        else if (key(argv[i], "topo_file=", &val)) topo = val;
    }
    *topo_out = topo;
    iga_atmo_t a = nullptr;
    int rc;
    if (!is_rngdep(v) && topo) {
        // set_region(atmo_file, topo_file, ...) (atmo_io.3d.strat.cpp:146-258, atmo_io.sph.strat.cpp)
        std::cout << "Interpolating atmosphere data in '" << argv[2] << "' and topography data in '" << topo << "'..."
                  << '\n';
        if (rev) std::cout << '\t' << "Inverting wind fields for back projection analysis..." << '\n';
        rc = iga_atmo_load_topo(argv[2], topo, fmt, rev ? 1 : 0, is_sph(v) ? IGA_GEOM_SPH : IGA_GEOM_3D, &a);
        if (rc == IGA_E_IO) {
            std::cout << '\t' << "ERROR: Invalid terrain file or atmospheric specification (" << topo << ", " << argv[2]
                      << ")" << '\n' << '\t' << iga_strerror(rc) << '\n' << '\n';
            return nullptr;
        }
    } else if (!is_rngdep(v)) {
        std::cout << "Interpolating atmosphere data in '" << argv[2] << "' using format '" << fmt << "'..." << '\n';
        if (rev) std::cout << '\t' << "Inverting wind fields for back projection analysis..." << '\n';
        rc = iga_atmo_load(argv[2], fmt, rev ? 1 : 0, &a);
        if (rc == IGA_E_IO) {
            std::cout << '\t' << "ERROR: Invalid atmospheric specification (" << argv[2] << ")" << '\n' << '\t'
                      << iga_strerror(rc) << '\n' << '\n';
            return nullptr;
        }
    } else {
        if (topo)
            std::cout << "Interpolating atmosphere data in '" << argv[2] << "*' and topography data in '" << topo << "'..."
                      << '\n';
        else
            std::cout << "Interpolating atmosphere data in '" << argv[2] << "'* using format '" << fmt << "'..." << '\n';
        if (rev) std::cout << '\t' << "Inverting wind fields for back projection analysis..." << '\n';
        rc = iga_atmo_load_rngdep(argv[2], argv[3], argv[4], topo, fmt, rev ? 1 : 0,
                                  is_sph(v) ? IGA_GEOM_SPH : IGA_GEOM_3D, &a);
        if (rc == IGA_E_IO) {
            std::cout << '\t' << "ERROR: Invalid grid, profile or terrain files (" << argv[2] << "*, " << argv[3] << ", "
                      << argv[4] << (topo ? ", " : "") << (topo ? topo : "") << ")" << '\n' << '\t' << iga_strerror(rc)
                      << '\n' << '\n';
            return nullptr;
        }
    }
    if (rc) {
        fail("loading the atmosphere", rc);
        return nullptr;
    }
    return a;
}

void print_region(Variant v, const iga_fan_params& p) {
    std::cout << '\t' << "Propagation region limits:" << '\n';
    if (is_sph(v)) {
        std::cout << '\t' << '\t' << "latitude = " << p.lat_min << ", " << p.lat_max << '\n';
        std::cout << '\t' << '\t' << "longitude = " << p.lon_min << ", " << p.lon_max << '\n';
        std::cout << '\t' << '\t' << "altitude = " << p.z_grnd << ", " << p.alt_max << '\n' << '\n';
    } else {
        std::cout << '\t' << '\t' << "x = " << p.x_min << ", " << p.x_max << '\n';
        std::cout << '\t' << '\t' << "y = " << p.y_min << ", " << p.y_max << '\n';
        std::cout << '\t' << '\t' << "z = " << p.z_grnd << ", " << p.alt_max << '\n';
    }
}

// Keys shared by every mode's second pass (propagation limits, absorption,
// output naming).  Returns true when `a` was one of them.
bool common_key(Variant v, const char* a, iga_fan_params& p, PropOpts& o, bool has_topo, double& freq) {
    const char* val;
    const bool sph = is_sph(v);
    if (key(a, "freq=", &val)) freq = atof(val);
    else if (key(a, "abs_coeff=", &val)) p.tweak_abs = std::max(0.0, atof(val));
    else if (key2(a, "max_alt=", "alt_max=", &val)) {
        p.alt_max = atof(val);
        std::cout << '\t' << "User selected altitude maximum = " << p.alt_max << '\n';
    } else if (key2(a, "max_rng=", "rng_max=", &val)) {
        p.rng_max = atof(val);
        std::cout << '\t' << "User selected range maximum = " << p.rng_max << '\n';
    } else if (sph && key2(a, "max_time=", "time_max=", &val)) {
        p.time_max = atof(val);
        std::cout << '\t' << "User selected propagation time maximum = " << p.time_max << '\n';
    } else if (sph && key2(a, "min_lat=", "lat_min=", &val)) {
        p.lat_min = atof(val);
        std::cout << '\t' << "User selected latitude minimum = " << p.lat_min * (Pi / 180.0) * (180.0 / Pi) << '\n';
    } else if (sph && key2(a, "max_lat=", "lat_max=", &val)) {
        p.lat_max = atof(val);
        std::cout << '\t' << "User selected latitude maximum = " << p.lat_max * (Pi / 180.0) * (180.0 / Pi) << '\n';
    } else if (sph && key2(a, "min_lon=", "lon_min=", &val)) {
        p.lon_min = atof(val);
        std::cout << '\t' << "User selected longitude minimum = " << p.lon_min * (Pi / 180.0) * (180.0 / Pi) << '\n';
    } else if (sph && key2(a, "max_lon=", "lon_max=", &val)) {
        p.lon_max = atof(val);
        std::cout << '\t' << "User selected longitude maximum = " << p.lon_max * (Pi / 180.0) * (180.0 / Pi) << '\n';
    } else if (!sph && key2(a, "min_x=", "x_min=", &val)) {
        p.x_min = atof(val);
        std::cout << '\t' << "User selected x minimum = " << p.x_min << '\n';
    } else if (!sph && key2(a, "max_x=", "x_max=", &val)) {
        p.x_max = atof(val);
        std::cout << '\t' << "User selected x maximum = " << p.x_max << '\n';
    } else if (!sph && key2(a, "min_y=", "y_min=", &val)) {
        p.y_min = atof(val);
        std::cout << '\t' << "User selected y minimum = " << p.y_min << '\n';
    } else if (!sph && key2(a, "max_y=", "y_max=", &val)) {
        p.y_max = atof(val);
        std::cout << '\t' << "User selected y maximum = " << p.y_max << '\n';
    } else if (key2(a, "min_ds=", "ds_min=", &val)) {
        p.ds_min = atof(val);
        std::cout << '\t' << "User selected ds minimum = " << p.ds_min << '\n';
    } else if (key2(a, "max_ds=", "ds_max=", &val)) {
        p.ds_max = atof(val);
        std::cout << '\t' << "User selected ds maximum = " << p.ds_max << '\n';
    } else if (key2(a, "max_s=", "s_max=", &val)) {
        p.s_max = atof(val);
        std::cout << '\t' << "User selected s maximum (path length between reflections) = " << p.s_max << '\n';
    } else if (key(a, "write_atmo=", &val)) o.write_atmo = str2bool(val);
    else if (key(a, "prof_format=", &val) || key(a, "reverse_winds=", &val) || key(a, "topo_file=", &val)) {}
    else if (key(a, "output_id=", &val)) o.output_id = val;
    else if (key(a, "z_grnd=", &val)) {
        if (!has_topo) p.z_grnd = atof(val);
        else std::cout << '\t' << "Note: cannot adjust ground elevation with topography." << '\n';
    } else if (key(a, "topo_use_BLw=", &val)) o.use_blw = str2bool(val);
    else return false;
    return true;
}

// The source height raised to the ground (run_prop: z_src = max(z_src, topo::z(src)))
// and the ground launch limit theta_grnd of one azimuth (main.infraga.3d.cpp:411-419,
// main.infraga.sph.cpp:420-433, 3d.rngdep :205-214, sph.rngdep :212-225).
struct Ground {
    Variant v;
    iga_atmo_t atmo;
    bool topo;
    double z0;
    double z(double x, double y) const {   // topo::z, as an altitude [km]
        if (topo) {
            double zz = 0.0;
            iga_atmo_terrain(atmo, x, y, &zz, nullptr, nullptr);
            return zz;
        }
        return v == Variant::k3DRngdep ? 0.0 : z0;   // 3D range-dependent topo::z is 0 without terrain
    }
    double theta_grnd(double xs, double ys, double zs, double phi_deg) const {
        if (zs - z(xs, ys) < 0.01) {
            if (!topo) return 0.1;
            double zz, d0, d1;
            iga_atmo_terrain(atmo, xs, ys, &zz, &d0, &d1);
            if (is_sph(v)) {
                const double dzgdx = 1.0 / (kR0 * cos(xs)) * d1;
                const double dzgdy = 1.0 / kR0 * d0;
                return atan(dzgdx * sin(phi_deg * Pi / 180.0) + dzgdy * cos(phi_deg * Pi / 180.0)) * (180.0 / Pi) + 0.1;
            }
            return atan(d0 * sin(phi_deg * Pi / 180.0) + d1 * cos(phi_deg * Pi / 180.0)) * (180.0 / Pi) + 0.1;
        }
        return -89.9;
    }
};

// write_atmo=true: geoac::write_prof (geoac.interface.3d.cpp:47-66,
// geoac.interface.sph.cpp:55-73) into ./atmo.dat: for z = m / 10 km, m < alt_max * 10,
// c, u, v [m/s], rho and the effective sound speed c + cos(az) u + sin(az) v [m/s]
// at the source (x, y [km] or lat, lon [deg]); 3D rows end with a tab.
int write_atmo_file(iga_atmo_t atmo, const iga_fan_params& p, double x, double y, double azimuth) {
    const bool sph = p.geometry == IGA_GEOM_SPH;
    std::vector<double> z;
    for (int m = 0; m < p.alt_max * 10.0; m++) z.push_back(sph ? (kR0 + m / 10.0) - kR0 : m / 10.0);
    std::vector<double> v(z.size() * 4);
    const int rc = iga_atmo_sample(atmo, &p, x, y, z.data(), (int)z.size(), v.data());
    if (rc) return rc;
    std::ofstream f("atmo.dat");
    for (size_t m = 0; m < z.size(); m++) {
        const double* q = &v[4 * m];
        f << (double)m / 10.0 << '\t' << q[0] * 1000.0 << '\t' << q[1] * 1000.0 << '\t' << q[2] * 1000.0 << '\t' << q[3]
          << '\t' << (q[0] + cos(azimuth) * q[1] + sin(azimuth) * q[2]) * 1000.0 << (sph ? "\n" : "\t\n");
    }
    return IGA_OK;
}

// Rows of one ray of a fan as the library returned them.
struct FanChunk {
    std::vector<double> arr;     // arrivals
    std::vector<int> arr_ray;
    std::vector<long long> steps;
    std::vector<double> path;
    std::vector<long long> path_start;
    std::vector<double> caus;
    std::vector<int> caus_ray;
};

int run_prop(int argc, char** argv, Variant v) {
    banner(v, "Propagation");
    const bool sph = is_sph(v), rd = is_rngdep(v);
    const char* topo = nullptr;
    iga_atmo_t atmo = load_atmosphere(v, argc, argv, &topo);
    if (!atmo) return 0;
    const bool has_topo = topo != nullptr;

    iga_fan_params p;
    int rc = iga_fan_params_init(atmo, sph ? IGA_GEOM_SPH : IGA_GEOM_3D, &p);
    if (rc) return fail("parameters", rc);
    print_region(v, p);
    PropOpts o;
    int bounces = p.bounces;
    double xs = p.src[0], ys = p.src[1], zs = 0.0;
    double freq = p.freq, turn_ht_min = p.turn_ht_min;
    bool calc_amp = true;
    const char* val;
    for (int i = rd ? 5 : 3; i < argc; i++) {
        const char* a = argv[i];
        if (key2(a, "incl_min=", "min_incl=", &val)) o.theta_min = atof(val);
        else if (key2(a, "incl_max=", "max_incl=", &val)) o.theta_max = atof(val);
        else if (key2(a, "az_min=", "min_az=", &val)) o.phi_min = atof(val);
        else if (key2(a, "az_max=", "max_az=", &val)) o.phi_max = atof(val);
        else if (key(a, "incl_step=", &val)) o.theta_step = atof(val);
        else if (key(a, "az_step=", &val)) o.phi_step = atof(val);
        else if (key(a, "inclination=", &val)) { o.theta_min = o.theta_max = atof(val); o.theta_step = 1.0; }
        else if (key(a, "azimuth=", &val)) { o.phi_min = o.phi_max = atof(val); o.phi_step = 1.0; }
        else if (key(a, "bounces=", &val)) bounces = atoi(val);
        else if (!sph && key2(a, "src_x=", "x_src=", &val)) xs = atof(val);
        else if (!sph && key2(a, "src_y=", "y_src=", &val)) ys = atof(val);
        else if (sph && key2(a, "src_lat=", "lat_src=", &val)) xs = atof(val);
        else if (sph && key2(a, "src_lon=", "lon_src=", &val)) ys = atof(val);
        else if (key(a, "src_alt=", &val) || match(a, "alt_src=", sph ? 8 : 6, 8, &val)) zs = atof(val);
        else if (key(a, "turn_ht_min=", &val)) turn_ht_min = atof(val);
        else if (key(a, "write_rays=", &val)) o.write_rays = str2bool(val);
        else if (key(a, "write_caustics=", &val)) o.write_caustics = str2bool(val);
        // infraga-3d-rngdep compares 8 characters and reads the value from the
        // '=' on (main.infraga.3d.rngdep.cpp:269), so any calc_amp= turns it off
        else if (v == Variant::k3DRngdep && match(a, "calc_amp=", 8, 8, &val)) calc_amp = str2bool(val);
        else if (v != Variant::k3DRngdep && key(a, "calc_amp=", &val)) calc_amp = str2bool(val);
        else if (key(a, "write_topo=", &val)) o.write_topo = str2bool(val);
        else if (key(a, "print_resid=", &val)) o.print_resid = str2bool(val);
        else if (common_key(v, a, p, o, has_topo, freq)) {}
        else if (!confirm_unknown(a, v == Variant::k3DRngdep)) return 0;
    }
    if (o.use_blw) {
        std::cout << '\t' << "ERROR: topo_use_BLw (boundary-layer vertical winds) is not provided by the GPU front end" << '\n';
        return 0;
    }
    // print_resid: residuals of every bounce segment, from the library's
    // residual rows (3D stratified flat ground; the other solvers do not have them)
    const bool resid = o.print_resid && v == Variant::k3D && !has_topo;
    if (o.print_resid && !resid) std::cout << '\t' << "Note: print_resid is not provided by the GPU front end for this solver" << '\n';

    // source: degrees on the command line, radians inside (spherical)
    const double lat_r = xs * (Pi / 180.0), lon_r = ys * (Pi / 180.0);
    Ground g{v, atmo, has_topo, p.z_grnd};
    zs = sph ? std::max(zs, g.z(lat_r, lon_r)) : std::max(zs, g.z(xs, ys));
    if (o.write_atmo && (rc = write_atmo_file(atmo, p, xs, ys, (90.0 - o.phi_min) * Pi / 180.0)))
        return fail("write_atmo", rc);
    if (o.write_caustics) calc_amp = true;

    const char* sum_src = sph ? "source location (lat, lon, alt): " : "source location: ";
    const double sx = sph ? lat_r * (180.0 / Pi) : xs, sy = sph ? lon_r * (180.0 / Pi) : ys;
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << "inclination: " << o.theta_min << ", " << o.theta_max << ", " << o.theta_step << '\n';
    std::cout << '\t' << "azimuth: " << o.phi_min << ", " << o.phi_max << ", " << o.phi_step << '\n';
    std::cout << '\t' << "bounces: " << bounces << '\n';
    std::cout << '\t' << sum_src << sx << ", " << sy << ", " << zs << '\n';
    if (!has_topo) std::cout << '\t' << "ground elevation: " << p.z_grnd << '\n';
    if (v == Variant::kSph) std::cout << '\t' << "turn_ht_min: " << turn_ht_min << '\n';
    std::cout << '\t' << "frequency: " << freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << p.tweak_abs << (sph ? "\n" : "\n\n");
    std::cout << '\t' << "write_atmo: " << (o.write_atmo ? "true" : "false") << '\n';
    std::cout << '\t' << "write_rays: " << (o.write_rays ? "true" : "false") << '\n';
    std::cout << '\t' << "write_topo: " << (o.write_topo ? "true" : "false") << '\n';
    std::cout << '\t' << "write_caustics: " << (o.write_caustics ? "true" : "false") << '\n';
    std::cout << '\t' << "calc_amp: " << (calc_amp ? "true" : "false") << '\n' << '\n';

    if (!o.output_id) {
        strip_extension(argv[2]);
        o.output_id = argv[2];
    }
    const std::string id = o.output_id;

    // launch angles: the reference's FP64-accumulated loops
    if (!(o.theta_step > 0.0) || !(o.phi_step > 0.0)) {
        std::cout << '\t' << "ERROR: incl_step and az_step must be positive" << '\n';
        return 0;
    }
    std::vector<double> th, ph;
    std::vector<size_t> az_end;
    std::vector<char> topo_first;
    const double src_x = sph ? lat_r : xs, src_y = sph ? lon_r : ys;
    for (double phi = o.phi_min; phi <= o.phi_max; phi += o.phi_step) {
        const double tg = g.theta_grnd(src_x, src_y, zs, phi);
        const double t0 = std::max(o.theta_min, tg), t1 = std::max(o.theta_max, tg);
        for (double theta = t0; theta <= t1; theta += o.theta_step) {
            th.push_back(theta);
            ph.push_back(phi);
            topo_first.push_back(fabs(theta - t0) < o.theta_step);
            if (th.size() > (size_t)200000000) {
                std::cout << '\t' << "ERROR: more than 2e8 rays requested" << '\n';
                return 0;
            }
        }
        az_end.push_back(th.size());
    }

    p.bounces = bounces;
    p.calc_amp = calc_amp ? 1 : 0;
    p.write_rays = (o.write_rays || o.write_caustics) ? 1 : 0;
    p.src[0] = xs; p.src[1] = ys; p.src[2] = zs;
    p.freq = freq;
    p.turn_ht_min = turn_ht_min;
    p.precision = IGA_FP64;

    std::ofstream results((id + ".arrivals.dat").c_str());
    results << "# " << variant_name(v) << " -prop summary:" << '\n';
    if (v == Variant::k3DRngdep) {
        results << "#" << '\t' << "profile prefix: " << argv[2] << '\n';
        results << "#" << '\t' << "profile grid files: " << argv[3] << ", " << argv[4] << '\n';
    } else {
        results << "#" << '\t' << "profile: " << argv[2] << '\n';
    }
    results << "#" << '\t' << "inclination: " << o.theta_min << ", " << o.theta_max << ", " << o.theta_step << '\n';
    results << "#" << '\t' << "azimuth: " << o.phi_min << ", " << o.phi_max << ", " << o.phi_step << '\n';
    results << "#" << '\t' << "bounces: " << bounces << '\n';
    results << "#" << '\t' << sum_src << sx << ", " << sy << ", " << zs << '\n';
    if (!has_topo) results << "#" << '\t' << "ground elevation: " << p.z_grnd << '\n';
    else results << "#" << '\t' << "topo file:" << topo << '\n';
    if (v == Variant::kSph) results << "#" << '\t' << "turn_ht_min: " << turn_ht_min << '\n';
    results << "#" << '\t' << "frequency: " << freq << '\n';
    results << "#" << '\t' << "S&B atten coeff: " << p.tweak_abs << '\n';
    threads_line(results, "#");
    results << '\n';
    const char* cols_3d[] = {"x_0 [km]", "y_0 [km]", "arrival incl [deg]", "back az [deg]"};
    const char* cols_sph[] = {"lat_0 [deg]", "lon_0 [deg]", "inclination [deg]", "back azimuth [deg]"};
    const char** cn = sph ? cols_sph : cols_3d;
    results << "# incl [deg]" << '\t' << "az [deg]" << '\t' << "n_b" << '\t' << cn[0] << '\t' << cn[1] << '\t' << "time [s]"
            << '\t' << "cel [km/s]" << '\t' << "turning ht [km]" << '\t' << cn[2] << '\t' << cn[3] << '\t'
            << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\n';

    const char* pos_hdr = sph ? "# lat [deg]\tlon [deg]\tz [km]" : "# x [km]\ty [km]\tz [km]";
    std::ofstream raypath;
    if (o.write_rays) {
        raypath.open((id + ".raypaths.dat").c_str());
        raypath << pos_hdr << '\t' << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\t' << "time [s]" << '\n';
    }
    std::vector<std::ofstream> caustics;
    if (o.write_caustics) {
        caustics.resize(bounces + 1);
        for (int b = 0; b <= bounces; b++) {
            caustics[b].open((id + ".caustics-" + std::to_string(b) + ".dat").c_str());
            caustics[b] << pos_hdr << '\t' << "time [s]" << '\n';
        }
    }

    // trace in chunks of rays (host and device memory stay bounded), write in ray order
    const size_t n = th.size();
    const size_t kChunk = 1u << 20;
    const long long kPathRowsMax = 1LL << 25;
    size_t az = 0;
    bool first_result = true;
    const int nb = bounces + 1;
    for (size_t r0 = 0; r0 < n; r0 += kChunk) {
        const size_t r1 = std::min(n, r0 + kChunk), m = r1 - r0;
        FanChunk c;
        c.arr.resize(m * nb * IGA_ARRIVAL_COLS);
        c.arr_ray.resize(m * nb);
        c.steps.resize(m);
        int n_out = 0;
        long long tot = 0;
        rc = iga_fan_run(atmo, &p, &th[r0], &ph[r0], (int)m, c.arr.data(), (int)(m * nb), &n_out, c.arr_ray.data(),
                         c.steps.data(), nullptr, &tot, nullptr);
        if (rc) return fail("ray fan", rc);
        // sampled paths and caustics, in sub-chunks whose path rows fit kPathRowsMax
        std::vector<std::vector<double>> path_rows(m);
        std::vector<std::vector<double>> caus_rows(m);
        if (o.write_rays || o.write_caustics) {
            size_t s0 = 0;
            while (s0 < m) {
                size_t s1 = s0;
                long long bound = 0;
                while (s1 < m) {
                    const long long b = (long long)nb + c.steps[s1] / 15 + 1;
                    if (s1 > s0 && bound + b > kPathRowsMax) break;
                    bound += b;
                    s1++;
                }
                const int k = (int)(s1 - s0);
                std::vector<double> prow(o.write_rays ? (size_t)bound * IGA_PATH_COLS : 0);
                std::vector<long long> pstart(k + 1);
                long long n_path = 0, n_caus = 0;
                std::vector<double> crow;
                std::vector<int> cray;
                long long ccap = o.write_caustics ? 4096 : 0;
                for (int attempt = 0; attempt < 2; attempt++) {
                    crow.assign((size_t)ccap * IGA_CAUSTIC_COLS, 0.0);
                    cray.assign((size_t)ccap, 0);
                    rc = iga_fan_paths(atmo, &p, &th[r0 + s0], &ph[r0 + s0], k, IGA_PATH_RAYS, &c.steps[s0],
                                       o.write_rays ? prow.data() : nullptr, o.write_rays ? bound : 0,
                                       o.write_rays ? &n_path : nullptr, o.write_rays ? pstart.data() : nullptr,
                                       o.write_caustics ? crow.data() : nullptr, ccap,
                                       o.write_caustics ? &n_caus : nullptr, o.write_caustics ? cray.data() : nullptr);
                    if (rc == IGA_E_TRUNCATED && o.write_caustics && n_caus > ccap && n_path <= bound) {
                        ccap = n_caus;
                        continue;
                    }
                    break;
                }
                if (rc) return fail("ray paths", rc);
                for (int i = 0; i < k && o.write_rays; i++)
                    path_rows[s0 + i].assign(prow.begin() + pstart[i] * IGA_PATH_COLS,
                                             prow.begin() + pstart[i + 1] * IGA_PATH_COLS);
                for (long long j = 0; j < n_caus; j++) {
                    auto& dst = caus_rows[s0 + cray[j]];
                    dst.insert(dst.end(), crow.begin() + j * IGA_CAUSTIC_COLS, crow.begin() + (j + 1) * IGA_CAUSTIC_COLS);
                }
                s0 = s1;
            }
        }
        std::vector<double> res_rows;
        std::vector<long long> res_start;
        if (resid) {
            res_rows.assign(m * nb * IGA_PATH_COLS, 0.0);
            res_start.assign(m + 1, 0);
            long long n_res = 0;
            rc = iga_fan_paths(atmo, &p, &th[r0], &ph[r0], (int)m, IGA_PATH_RESID, c.steps.data(), res_rows.data(),
                               (long long)(m * nb), &n_res, res_start.data(), nullptr, 0, nullptr, nullptr);
            if (rc) return fail("residuals", rc);
        }
        size_t w = 0;   // next arrival row
        for (size_t i = 0; i < m; i++) {
            const size_t r = r0 + i;
            std::cout << "Calculating ray path: " << th[r] << " degrees inclination, " << ph[r] << " degrees azimuth." << '\n';
            for (long long j = resid ? res_start[i] : 0; resid && j < res_start[i + 1]; j++) {
                // after each prop_rk4 call (main.infraga.3d.cpp:437-441)
                const double* q = &res_rows[(size_t)j * IGA_PATH_COLS];
                std::cout << '\t' << "Residuals at Ray Termination (region boundary or reflection):" << '\n';
                std::cout << '\t' << '\t' << "Eikonal residual: " << q[0] << '\n';
                std::cout << '\t' << '\t' << "Aux. param. residual: " << q[1] << '\n';
            }
            for (const double* q = path_rows[i].data(); q < path_rows[i].data() + path_rows[i].size(); q += IGA_PATH_COLS) {
                if (sph) raypath << std::setprecision(8) << q[0] << '\t' << std::setprecision(8) << q[1];
                else raypath << q[0] << '\t' << q[1];
                raypath << '\t' << q[2] << '\t' << q[3] << '\t' << q[4] << '\t' << q[5] << '\n';
            }
            for (const double* q = caus_rows[i].data(); q < caus_rows[i].data() + caus_rows[i].size(); q += IGA_CAUSTIC_COLS) {
                std::ofstream& cs = caustics[(int)q[4]];
                if (sph) cs << std::setprecision(8) << q[0] << '\t' << std::setprecision(8) << q[1];
                else cs << q[0] << '\t' << q[1];
                cs << '\t' << q[2];
                if (v == Variant::k3DRngdep) cs << '\t' << 0.0;
                cs << '\t' << q[3] << '\n';
            }
            for (; w < (size_t)n_out && c.arr_ray[w] == (int)i; w++) {
                const double* q = &c.arr[w * IGA_ARRIVAL_COLS];
                results << q[0] << '\t' << q[1] << '\t' << (int)q[2];
                if (sph) results << '\t' << std::setprecision(8) << q[3] << '\t' << std::setprecision(8) << q[4];
                else results << '\t' << q[3] << '\t' << q[4];
                for (int col = 5; col < IGA_ARRIVAL_COLS; col++) results << '\t' << q[col];
                results << '\n';
                first_result = false;
            }
            if (o.write_rays) raypath << '\n';
            while (az < az_end.size() && az_end[az] == r + 1) {
                results << '\n';
                az++;
            }
        }
    }
    while (az < az_end.size()) {   // azimuths without rays
        results << '\n';
        az++;
    }
    (void)first_result;

    // terrain under the last ray that opened the terrain file (the first
    // inclination of each azimuth by the reference's test; each reopening
    // truncates the file)
    if (o.write_topo) {
        long long last = -1;
        for (size_t r = 0; r < n; r++)
            if (topo_first[r]) last = (long long)r;
        std::ofstream tf;
        if (last >= 0) {
            tf.open((id + ".terrain.dat").c_str());
            std::vector<long long> st(1);
            int n_out = 0;
            std::vector<double> arr((size_t)nb * IGA_ARRIVAL_COLS);
            rc = iga_fan_run(atmo, &p, &th[last], &ph[last], 1, arr.data(), nb, &n_out, nullptr, st.data(), nullptr,
                             nullptr, nullptr);
            if (rc) return fail("terrain samples", rc);
            const long long cap = (long long)nb + st[0] / 10 + 1;
            std::vector<double> rows((size_t)cap * IGA_PATH_COLS);
            long long np = 0;
            rc = iga_fan_paths(atmo, &p, &th[last], &ph[last], 1, IGA_PATH_TERRAIN, st.data(), rows.data(), cap, &np,
                               nullptr, nullptr, 0, nullptr, nullptr);
            if (rc) return fail("terrain samples", rc);
            for (long long j = 0; j < np; j++) {
                const double* q = &rows[(size_t)j * IGA_PATH_COLS];
                if (sph) tf << std::setprecision(8) << q[0] << '\t' << std::setprecision(8) << q[1];
                else tf << q[0] << '\t' << q[1];
                tf << '\t' << q[2] << '\n';
            }
        }
    }
    iga_atmo_destroy(atmo);
    return 0;
}

// ------------------------------------------------------------------------
// -eig_search / -eig_direct (3D and spherical stratified)
// ------------------------------------------------------------------------

// src / rcvr in the library's order: 3D (x, y, alt) / (x, y) [km];
// spherical (lat, lon [deg], alt [km]) / (lat, lon)
struct EigOpts {
    double src[3] = {0.0, 0.0, 0.0};
    double rcvr[2] = {-250.0, 0.0};
    bool verbose = false;
    bool write_atmo = false;
    const char* output_id = nullptr;
    // infraga-accel-* only: source and receiver list files
    // (main.infraga.3d.mpi.cpp:639-640, :720-760)
    const char* srcs_list = nullptr;
    const char* rcvrs_list = nullptr;
};

// Sampled path of one eigenray for {id}.eigenray-N.dat (find_eigenray's
// final trace, geoac.eigenray.3d.cpp:220-279, geoac.eigenray.sph.cpp:230-268):
// 3D rows of the first segment as run_prop writes them, later segments with
// the raw altitude and the absorption sum itself instead of -2 x it; the
// spherical file writes every segment alike, latitude and longitude with
// 8 significant digits.
int write_eigenray_file(const std::string& path, iga_atmo_t atmo, const iga_fan_params& base, const double* src,
                        double theta, double az, int n_b, bool sph) {
    iga_fan_params q = base;
    q.bounces = n_b;
    q.calc_amp = 1;
    q.write_rays = 1;
    q.turn_ht_min = -1.0e30;   // the final trace never stops at a low turning height
    q.time_max = 1.0e30;       // nor at run_prop's travel-time cap
    q.src[0] = src[0]; q.src[1] = src[1]; q.src[2] = src[2];
    long long st = 0;
    int n_out = 0;
    std::vector<double> arr((size_t)(n_b + 1) * IGA_ARRIVAL_COLS);
    int rc = iga_fan_run(atmo, &q, &theta, &az, 1, arr.data(), n_b + 1, &n_out, nullptr, &st, nullptr, nullptr, nullptr);
    if (rc) return rc;
    const long long cap = (long long)n_b + 1 + st / 15 + 1;
    std::vector<double> rows((size_t)cap * IGA_PATH_COLS);
    long long np = 0;
    rc = iga_fan_paths(atmo, &q, &theta, &az, 1, IGA_PATH_RAYS, &st, rows.data(), cap, &np, nullptr, nullptr, 0, nullptr,
                       nullptr);
    if (rc) return rc;
    std::ofstream f(path.c_str());
    f << (sph ? "# lat [deg]\tlon [deg]\tz [km]" : "# x [km]\ty [km]\tz [km]") << '\t' << "trans. coeff. [dB]" << '\t'
      << "absorption [dB]" << '\t' << "time [s]" << '\n';
    for (long long j = 0; j < np; j++) {
        const double* r = &rows[(size_t)j * IGA_PATH_COLS];
        if (sph) {
            f << std::setprecision(8) << r[0] << '\t' << std::setprecision(8) << r[1] << '\t' << r[2] << '\t' << r[3] << '\t'
              << r[4] << '\t' << r[5] << '\n';
        } else {
            const double absorb = r[6] >= 1.0 ? -r[4] / 2.0 : r[4];
            f << r[0] << '\t' << r[1] << '\t' << r[2] << '\t' << r[3] << '\t' << absorb << '\t' << r[5] << '\n';
        }
    }
    return IGA_OK;
}

void print_eigenray(const double* q, const double* src, bool verbose) {
    if (verbose) {
        std::cout << '\t' << '\t' << "Eigenray Identified:" << '\n';
        std::cout << '\t' << '\t' << '\t' << "inclination [deg] = " << std::setprecision(8) << q[0] << '\n';
        std::cout << '\t' << '\t' << '\t' << "azimuth [deg] = " << std::setprecision(8) << q[1] << '\n';
        std::cout << '\t' << '\t' << '\t' << "bounces [-] = " << (int)q[2] << '\n';
        std::cout << '\t' << '\t' << '\t' << "x [km E-W] = " << q[3] << '\n';
        std::cout << '\t' << '\t' << '\t' << "y [km N-S] = " << q[4] << '\n';
        std::cout << '\t' << '\t' << '\t' << "time [s] = " << q[5] << '\n';
        std::cout << '\t' << '\t' << '\t' << "celerity [km/s] = " << q[6] << '\n';
        std::cout << '\t' << '\t' << '\t' << "turning height [km] = " << q[7] << '\n';
        std::cout << '\t' << '\t' << '\t' << "arrival inclination [deg] = " << q[8] << '\n';
        std::cout << '\t' << '\t' << '\t' << "back azimuth = " << q[9] << '\n';
        std::cout << '\t' << '\t' << '\t' << "attenuation (geometric) [dB] = " << q[10] << '\n';
        std::cout << '\t' << '\t' << '\t' << "absorption [dB] = " << q[11] << '\n' << '\n';
    } else {
        std::cout << '\t' << "Eigenray identified:" << '\t' << "theta, phi = " << std::setprecision(8) << q[0] << ", " << q[1]
                  << " degrees." << '\n';
    }
    (void)src;
}

// Second pass of the eigenray modes.  direct = run_eig_direct's key set.
bool parse_eig(int argc, char** argv, Variant v, bool direct, iga_eig_params& ep, EigOpts& o, bool has_topo,
               double& incl_est, double& az_est_deg, bool& az_est_given, int& bounces) {
    const bool sph = is_sph(v);
    PropOpts po;
    double freq = ep.fan.freq;
    const char* val;
    for (int i = is_rngdep(v) ? 5 : 3; i < argc; i++) {
        const char* a = argv[i];
        if (!direct && key2(a, "incl_min=", "min_incl=", &val)) ep.incl_min = atof(val);
        else if (!direct && key2(a, "incl_max=", "max_incl=", &val)) ep.incl_max = atof(val);
        else if (!direct && key2(a, "bnc_min=", "min_bnc=", &val)) ep.bnc_min = atoi(val);
        else if (!direct && key2(a, "bnc_max=", "max_bnc=", &val)) ep.bnc_max = atoi(val);
        else if (!direct && key(a, "bounces=", &val)) ep.bnc_min = ep.bnc_max = atoi(val);
        else if (direct && (key(a, "incl_est=", &val) || (sph && key(a, "est_incl=", &val)))) incl_est = atof(val);
        else if (direct && key2(a, "az_est=", "est_az=", &val)) { az_est_deg = atof(val); az_est_given = true; }
        else if (direct && key(a, "bounces=", &val)) bounces = atoi(val);
        else if (!sph && key2(a, "src_x=", "x_src=", &val)) o.src[0] = atof(val);
        else if (!sph && (key(a, "src_y=", &val) || match(a, "y_src_y=", 6, 6, &val))) o.src[1] = atof(val);
        else if (sph && key2(a, "src_lat=", "lat_src=", &val)) o.src[0] = atof(val);
        else if (sph && key2(a, "src_lon=", "lon_src=", &val)) o.src[1] = atof(val);
        else if (key2(a, "src_alt=", "alt_src=", &val)) o.src[2] = atof(val);
        else if (!sph && key2(a, "rcvr_x=", "x_rcvr=", &val)) o.rcvr[0] = atof(val);
        else if (!sph && key2(a, "rcvr_y=", "y_rcvr=", &val)) o.rcvr[1] = atof(val);
        else if (sph && key2(a, "rcvr_lat=", "lat_rcvr=", &val)) o.rcvr[0] = atof(val);
        else if (sph && key2(a, "rcvr_lon=", "lon_rcvr=", &val)) o.rcvr[1] = atof(val);
        else if (key(a, "verbose=", &val)) o.verbose = str2bool(val);
        else if (g_launch.accel && !direct && key2(a, "srcs_list=", "list_srcs=", &val)) o.srcs_list = val;
        else if (g_launch.accel && !direct && key2(a, "rcvrs_list=", "list_rcvrs=", &val)) o.rcvrs_list = val;
        // the MPI builds' sequential-source reuse and verbose receiver choice:
        // accepted; every source here gets the full search
        else if (g_launch.accel && !direct && key(a, "seq_srcs=", &val)) {}
        else if (g_launch.accel && !direct && key(a, "seq_srcs_dr=", &val)) {}
        else if (g_launch.accel && !direct && key(a, "verbose_rcvr=", &val)) {}
        else if (key(a, "iterations=", &val)) ep.iterations = (int)atof(val);
        else if (key(a, "damping=", &val)) ep.damping = atof(val);
        else if (key(a, "tolerance=", &val)) ep.tolerance = atof(val);
        else if (!direct && key(a, "az_dev_lim=", &val)) ep.az_err_lim = atof(val);
        else if (!direct && key2(a, "incl_step_min=", "min_incl_step=", &val)) ep.incl_step_min = atof(val);
        else if (!direct && key2(a, "incl_step_max=", "max_incl_step=", &val)) ep.incl_step_max = atof(val);
        else if (common_key(v, a, ep.fan, po, has_topo, freq)) {}
        else if (!confirm_unknown(a, false)) return false;
    }
    ep.fan.freq = freq;
    o.output_id = po.output_id;
    if (po.use_blw) {
        std::cout << '\t' << "ERROR: topo_use_BLw (boundary-layer vertical winds) is not provided by the GPU front end" << '\n';
        return false;
    }
    o.write_atmo = po.write_atmo;
    return true;
}

// Rows of a source or receiver list file: file_length lines (those not
// starting with '#', less one), `cols` numbers each (fileIO.cpp:18-35).
bool read_list(const char* path, int cols, std::vector<double>& out) {
    std::ifstream f(path);
    if (!f.is_open()) return false;
    // file_length (util/fileIO.cpp:18-35): read until eof, count the lines
    // not starting with '#', minus one -- the empty read after a final newline
    // (a list without one loses its last entry there too)
    int n = 0;
    std::string line;
    while (!f.eof()) {
        std::getline(f, line);
        if (line.find('#') != 0) n++;
    }
    n -= 1;
    if (n < 1) return false;
    f.clear();
    f.seekg(0);
    out.clear();
    for (int i = 0; i < n * cols; i++) {
        double x;
        if (!(f >> x)) return false;
        out.push_back(x);
    }
    return true;
}

// infraga-accel-* -eig_search with srcs_list= / rcvrs_list=
// (main.infraga.3d.mpi.cpp:556-975): every source against every receiver,
// each source's receivers in one batched search, one arrivals file per
// (source, receiver) named as the MPI build names them, eigenray path files
// numbered per file from 0.  The search itself is the serial one
// (est_eigenray / find_eigenray of geoac.eigenray.3d.cpp), as for the
// single-pair case.
template <class Ground>
int run_eig_lists(Variant v, const char* profile, const char* topo, iga_atmo_t atmo, iga_eig_params& ep,
                  const EigOpts& o, const std::string& id, Ground ground) {
    const bool sph = is_sph(v), has_topo = topo != nullptr;
    std::vector<double> srcs, rcvrs;
    if (o.srcs_list) {
        if (!read_list(o.srcs_list, 3, srcs)) {
            std::cout << '\t' << "ERROR: cannot read source list " << o.srcs_list << '\n';
            return 0;
        }
    } else {
        srcs.assign(o.src, o.src + 3);
    }
    if (o.rcvrs_list) {
        if (!read_list(o.rcvrs_list, 2, rcvrs)) {
            std::cout << '\t' << "ERROR: cannot read receiver list " << o.rcvrs_list << '\n';
            return 0;
        }
    } else {
        rcvrs.assign(o.rcvr, o.rcvr + 2);
    }
    const int n_src = (int)srcs.size() / 3, n_rcv = (int)rcvrs.size() / 2;
    for (int n = 0; n < n_src; n++) srcs[3 * n + 2] = std::max(srcs[3 * n + 2], ground(srcs[3 * n], srcs[3 * n + 1]));
    const char* loc_s = sph ? "source location (lat, lon, alt): " : "source location: ";
    const char* loc_r = sph ? "receiver location (lat, lon, alt): " : "receiver location: ";
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << "source location(s) " << (sph ? "(lat, lon, alt):" : "(x, y, alt):") << '\n';
    for (int n = 0; n < std::min(n_src, 10); n++)
        std::cout << '\t' << '\t' << "(" << srcs[3 * n] << ", " << srcs[3 * n + 1] << ", " << srcs[3 * n + 2] << ")" << '\n';
    if (n_src > 10) std::cout << '\t' << '\t' << "..." << '\n';
    std::cout << '\t' << "receiver location(s) " << (sph ? "(lat, lon, alt):" : "(x, y, alt):") << '\n';
    for (int i = 0; i < std::min(n_rcv, 10); i++)
        std::cout << '\t' << '\t' << "(" << rcvrs[2 * i] << ", " << rcvrs[2 * i + 1] << ", "
                  << ground(rcvrs[2 * i], rcvrs[2 * i + 1]) << ")" << '\n';
    if (n_rcv > 10) std::cout << '\t' << '\t' << "..." << '\n';
    std::cout << '\t' << "inclination range: " << ep.incl_min << ", " << ep.incl_max << '\n';
    std::cout << '\t' << "bounces: " << ep.bnc_min << ", " << ep.bnc_max << '\n';
    if (!has_topo) std::cout << '\t' << "ground elevation: " << ep.fan.z_grnd << '\n';
    std::cout << '\t' << "damping:" << ep.damping << '\n';
    std::cout << '\t' << "frequency: " << ep.fan.freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << ep.fan.tweak_abs << '\n';
    std::cout << '\t' << "threads: " << g_launch.threads << '\n' << '\n';

    for (int n = 0; n < n_src; n++) {
        const double* src = &srcs[3 * n];
        std::cout << '\n' << "Searching for eigenrays from source at " << src[0] << ", " << src[1] << ", " << src[2] << '\n';
        std::vector<iga_eig_pair> pairs(n_rcv);
        for (int i = 0; i < n_rcv; i++) {
            pairs[i].src[0] = src[0]; pairs[i].src[1] = src[1]; pairs[i].src[2] = src[2];
            pairs[i].rcvr[0] = rcvrs[2 * i]; pairs[i].rcvr[1] = rcvrs[2 * i + 1];
        }
        int cap = 256 * n_rcv, n_out = 0;
        std::vector<double> rows((size_t)cap * IGA_ARRIVAL_COLS);
        std::vector<int> pidx(cap);
        long long steps = 0;
        int rc = iga_eig_run(atmo, &ep, pairs.data(), n_rcv, rows.data(), cap, &n_out, pidx.data(), &steps);
        if (rc == IGA_E_TRUNCATED) {
            cap = n_out;
            rows.resize((size_t)cap * IGA_ARRIVAL_COLS);
            pidx.resize(cap);
            rc = iga_eig_run(atmo, &ep, pairs.data(), n_rcv, rows.data(), cap, &n_out, pidx.data(), &steps);
        }
        if (rc) return fail("eigenray search", rc);
        for (int i = 0; i < n_rcv; i++) {
            std::string stem = id;
            if (n_src > 1) stem += ".src-" + std::to_string(n);
            if (n_rcv > 1) stem += ".rcvr-" + std::to_string(i);
            std::ofstream res((stem + ".arrivals.dat").c_str());
            const double zr = ground(rcvrs[2 * i], rcvrs[2 * i + 1]);
            res << "# " << variant_name(v) << " -eig_search summary:" << '\n';
            res << "# " << '\t' << "profile: " << profile << '\n';
            res << "# " << '\t' << loc_s << src[0] << ", " << src[1] << ", " << src[2] << '\n';
            res << "# " << '\t' << loc_r << rcvrs[2 * i] << ", " << rcvrs[2 * i + 1] << ", " << zr << ")." << '\n';
            res << "# " << '\t' << "inclination range: " << ep.incl_min << ", " << ep.incl_max << '\n';
            res << "# " << '\t' << "bounces: " << ep.bnc_min << ", " << ep.bnc_max << '\n';
            if (!has_topo) res << "#" << '\t' << "ground elevation: " << ep.fan.z_grnd << '\n';
            else res << "#" << '\t' << "topo file:" << topo << '\n';
            res << "# " << '\t' << "damping: " << ep.damping << '\n';
            res << "# " << '\t' << "frequency: " << ep.fan.freq << '\n';
            res << "# " << '\t' << "S&B atten coeff: " << ep.fan.tweak_abs << '\n';
            res << "# " << '\t' << "threads: " << g_launch.threads << '\n' << '\n';
            res << "# incl [deg]" << '\t' << "az [deg]" << '\t' << "n_b" << '\t' << (sph ? "lat_0 [deg]" : "x_0 [km]") << '\t'
                << (sph ? "lon_0 [deg]" : "y_0 [km]") << '\t' << "time [s]" << '\t' << "cel [km/s]" << '\t'
                << "turning ht [km]" << '\t' << "arrival incl [deg]" << '\t' << "back az [deg]" << '\t'
                << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\n';
            int cnt = 0;
            for (int j = 0; j < n_out; j++) {
                if (pidx[j] != i) continue;
                const double* q = &rows[(size_t)j * IGA_ARRIVAL_COLS];
                res << std::setprecision(8) << q[0] << '\t' << std::setprecision(8) << q[1] << '\t' << (int)q[2];
                for (int col = 3; col < IGA_ARRIVAL_COLS; col++) res << '\t' << q[col];
                res << '\n';
                print_eigenray(q, src, o.verbose);
                rc = write_eigenray_file(stem + ".eigenray-" + std::to_string(cnt) + ".dat", atmo, ep.fan, src, q[0], q[1],
                                         (int)q[2], sph);
                if (rc) return fail("eigenray path", rc);
                cnt++;
            }
            std::cout << '\t' << "Identified " << cnt << " eigenray(s) to receiver at " << rcvrs[2 * i] << ", "
                      << rcvrs[2 * i + 1] << ", " << zr << '\n';
        }
    }
    return 0;
}

int run_eig(int argc, char** argv, Variant v, bool direct) {
    banner(v, direct ? "Eigenray Direct" : "Eigenray Search");
    const char* topo = nullptr;
    iga_atmo_t atmo = load_atmosphere(v, argc, argv, &topo);
    if (!atmo) return 0;
    const bool sph = is_sph(v), rd = is_rngdep(v), has_topo = topo != nullptr;
    iga_eig_params ep;
    int rc = iga_eig_params_default(atmo, &ep);
    if (!rc && (sph || rd)) rc = iga_fan_params_init(atmo, sph ? IGA_GEOM_SPH : IGA_GEOM_3D, &ep.fan);
    if (rc) return fail("parameters", rc);
    print_region(v, ep.fan);
    EigOpts o;
    o.verbose = direct && !sph;   // the spherical -eig_direct is quiet by default
    double incl_est = 10.0, az_est = 0.0;
    // source and receiver defaults of run_eig_search / run_eig_direct
    if (is_sph(v) && !has_topo) {   // main.infraga.sph.cpp:788-789
        o.src[0] = 30.0; o.src[1] = 0.0; o.src[2] = 0.0;
        o.rcvr[0] = 30.0; o.rcvr[1] = -2.5;
    } else if (v == Variant::k3D && has_topo) {   // main.infraga.3d.cpp:812-815, :992-995
        double a0, a1, b0, b1;
        iga_atmo_region(atmo, &a0, &a1, &b0, &b1);
        o.src[0] = (a1 + a0) / 2.0; o.src[1] = (b1 + b0) / 2.0;
        o.rcvr[0] = o.src[0] - 250.0; o.rcvr[1] = o.src[1];
    } else if (rd || sph) {   // the centre of the region (main.infraga.3d.rngdep.cpp:816-817, sph.rngdep :821-822,
                              // infraga-sph over terrain main.infraga.sph.cpp:825-828 with the receiver 2.5 deg east)
        double a0, a1, b0, b1;
        iga_atmo_region(atmo, &a0, &a1, &b0, &b1);
        o.src[0] = (a1 + a0) / 2.0; o.src[1] = (b1 + b0) / 2.0; o.src[2] = 0.0;
        o.rcvr[0] = sph ? o.src[0] : o.src[0] + 250.0;
        o.rcvr[1] = sph ? o.src[1] + (rd ? 5.0 : 2.5) : o.src[1];
    }
    // the range-dependent -eig_direct keep their inclination estimate in radians
    // when none is given: 0.5 (3D) and 10 (spherical)
    if (v == Variant::k3DRngdep) incl_est = 0.5 * (180.0 / Pi);
    if (v == Variant::kSphRngdep) incl_est = 10.0 * (180.0 / Pi);
    bool az_given = false;
    int bounces = 0;
    if (!parse_eig(argc, argv, v, direct, ep, o, has_topo, incl_est, az_est, az_given, bounces)) return 0;
    // topo::z under the source and the receiver: the flat ground, the terrain,
    // or 0 for the 3D range-dependent solver without terrain
    auto ground = [&](double x, double y) {
        if (has_topo) {
            double zz = 0.0;
            iga_atmo_terrain(atmo, sph ? x * (Pi / 180.0) : x, sph ? y * (Pi / 180.0) : y, &zz, nullptr, nullptr);
            return zz;
        }
        return v == Variant::k3DRngdep ? 0.0 : ep.fan.z_grnd;
    };
    o.src[2] = std::max(ground(o.src[0], o.src[1]), o.src[2]);
    const double z_rcvr = ground(o.rcvr[0], o.rcvr[1]);
    if (o.write_atmo) {   // the azimuth argument of each main's write_prof call
        double az_w;
        if (sph) {        // globe::bearing(src, rcvr), radians (main.infraga.sph.cpp:892, :1097)
            const double la1 = o.src[0] * (Pi / 180.0), lo1 = o.src[1] * (Pi / 180.0);
            const double la2 = o.rcvr[0] * (Pi / 180.0), lo2 = o.rcvr[1] * (Pi / 180.0);
            az_w = atan2(sin(lo2 - lo1), cos(la1) * tan(la2) - sin(la1) * cos(lo2 - lo1));
        } else if (direct && az_given) {   // phi_est (main.infraga.3d.cpp:1050-1056)
            az_w = Pi / 2.0 - az_est * (Pi / 180.0);
        } else {          // atan2(rcvr - src) (main.infraga.3d.cpp:875)
            az_w = atan2(o.rcvr[1] - o.src[1], o.rcvr[0] - o.src[0]);
        }
        if ((rc = write_atmo_file(atmo, ep.fan, o.src[0], o.src[1], az_w))) return fail("write_atmo", rc);
    }
    if (!o.output_id) {
        strip_extension(argv[2]);
        o.output_id = argv[2];
    }
    const std::string id = o.output_id;
    if (!direct && (o.srcs_list || o.rcvrs_list)) {
        rc = run_eig_lists(v, argv[2], topo, atmo, ep, o, id, ground);
        iga_atmo_destroy(atmo);
        return rc;
    }
    iga_eig_pair pair;
    pair.src[0] = o.src[0]; pair.src[1] = o.src[1]; pair.src[2] = o.src[2];
    pair.rcvr[0] = o.rcvr[0]; pair.rcvr[1] = o.rcvr[1];

    // locations as the reference echoes them (spherical: degrees -> radians -> degrees)
    const double d2r = Pi / 180.0, r2d = 180.0 / Pi;
    const double es[3] = {sph ? o.src[0] * d2r * r2d : o.src[0], sph ? o.src[1] * d2r * r2d : o.src[1], o.src[2]};
    const double er[2] = {sph ? o.rcvr[0] * d2r * r2d : o.rcvr[0], sph ? o.rcvr[1] * d2r * r2d : o.rcvr[1]};
    const char* loc_s = sph ? "source location (lat, lon, alt): " : "source location: ";
    const char* loc_r = sph ? "receiver location (lat, lon, alt): " : "receiver location: ";
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << loc_s << es[0] << ", " << es[1] << ", " << es[2] << '\n';
    std::cout << '\t' << loc_r << er[0] << ", " << er[1] << ", " << z_rcvr << '\n';
    if (direct) {
        double phi_est;
        if (az_given) {
            phi_est = Pi / 2.0 - az_est * (Pi / 180.0);
        } else if (sph) {   // Pi/2 - globe::bearing(src, rcvr)
            const double la1 = o.src[0] * d2r, lo1 = o.src[1] * d2r, la2 = o.rcvr[0] * d2r, lo2 = o.rcvr[1] * d2r;
            phi_est = Pi / 2.0 - atan2(sin(lo2 - lo1), cos(la1) * tan(la2) - sin(la1) * cos(lo2 - lo1));
        } else {
            phi_est = atan2(o.rcvr[1] - o.src[1], o.rcvr[0] - o.src[0]);
        }
        az_est = 90.0 - phi_est * 180.0 / Pi;
        std::cout << '\t' << "inclination estimate: " << incl_est << '\n';
        std::cout << '\t' << "azimuth estimate: " << az_est << '\n';
        std::cout << '\t' << "bounces: " << bounces << '\n';
    } else {
        std::cout << '\t' << "inclination range: " << ep.incl_min << ", " << ep.incl_max << '\n';
        std::cout << '\t' << "bounces: " << ep.bnc_min << ", " << ep.bnc_max << '\n';
    }
    if (!has_topo) std::cout << '\t' << "ground elevation: " << ep.fan.z_grnd << '\n';
    std::cout << '\t' << "damping:" << ep.damping << '\n';
    std::cout << '\t' << "frequency: " << ep.fan.freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << ep.fan.tweak_abs << '\n' << '\n';

    std::vector<double> rows;
    int n_out = 0;
    if (direct) {
        rows.resize(IGA_ARRIVAL_COLS);
        rc = iga_eig_direct(atmo, &ep, &pair, incl_est, az_est, bounces, rows.data(), &n_out, nullptr);
        if (rc) return fail("eigenray search", rc);
    } else {
        std::ofstream res((id + ".arrivals.dat").c_str());
        res << "# " << variant_name(v) << " -eig_search summary:" << '\n';
        res << "# " << '\t' << (rd ? "profile prefix: " : "profile: ") << argv[2] << '\n';
        if (v == Variant::k3DRngdep) res << "# " << '\t' << "profile grid files: " << argv[3] << ", " << argv[4] << '\n';
        res << "# " << '\t' << loc_s << es[0] << ", " << es[1] << ", " << es[2] << '\n';
        res << "# " << '\t' << loc_r << er[0] << ", " << er[1] << ", " << z_rcvr << '\n';
        res << "# " << '\t' << "inclination range: " << ep.incl_min * (Pi / 180.0) * (180.0 / Pi) << ", "
            << ep.incl_max * (Pi / 180.0) * (180.0 / Pi) << '\n';
        res << "# " << '\t' << "bounces: " << ep.bnc_min << ", " << ep.bnc_max << '\n';
        if (!has_topo) res << "#" << '\t' << "ground elevation: " << ep.fan.z_grnd << '\n';
        else res << "#" << '\t' << "topo file:" << topo << '\n';
        res << "# " << '\t' << "damping: " << ep.damping << '\n';
        res << "# " << '\t' << "frequency: " << ep.fan.freq << '\n';
        // infraga-sph writes no blank line after the summary (main.infraga.sph.cpp:944)
        res << "# " << '\t' << "S&B atten coeff: " << ep.fan.tweak_abs << '\n';
        threads_line(res, "# ");
        res << (sph ? "" : "\n");
        if (sph)
            res << "# incl [deg]" << '\t' << "az [deg]" << '\t' << "n_b" << '\t' << "lat_0 [deg]" << '\t' << "lon_0 [deg]"
                << '\t' << "time [s]" << '\t' << "cel [km/s]" << '\t' << "turning ht [km]" << '\t' << "inclination [deg]"
                << '\t' << "back azimuth [deg]" << '\t' << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\n';
        else
            res << "# incl [deg]" << '\t' << "az [deg]" << '\t' << "n_b" << '\t' << "x_0 [km]" << '\t' << "y_0 [km]" << '\t'
                << "time [s]" << '\t' << "cel [km/s]" << '\t' << "turning ht [km]" << '\t' << "arrival incl [deg]" << '\t'
                << "back az [deg]" << '\t' << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\n';
        for (int nbc = ep.bnc_min; nbc <= ep.bnc_max; nbc++) {
            if (sph) std::cout << "Searching for " << nbc << " bounce eigenrays." << '\n';
            else std::cout << "Searching for " << nbc << " bounce eigenray(s) with inclination between " << ep.incl_min
                           << " and " << ep.incl_max << "." << '\n';
        }
        const int cap0 = 256;
        rows.resize((size_t)cap0 * IGA_ARRIVAL_COLS);
        long long steps = 0;
        rc = iga_eig_run(atmo, &ep, &pair, 1, rows.data(), cap0, &n_out, nullptr, &steps);
        if (rc == IGA_E_TRUNCATED) {
            rows.resize((size_t)n_out * IGA_ARRIVAL_COLS);
            rc = iga_eig_run(atmo, &ep, &pair, 1, rows.data(), n_out, &n_out, nullptr, &steps);
        }
        if (rc) return fail("eigenray search", rc);
        for (int j = 0; j < n_out; j++) {
            const double* q = &rows[(size_t)j * IGA_ARRIVAL_COLS];
            res << std::setprecision(8) << q[0] << '\t' << std::setprecision(8) << q[1] << '\t' << (int)q[2];
            for (int col = 3; col < IGA_ARRIVAL_COLS; col++) res << '\t' << q[col];
            res << '\n';
        }
    }
    for (int j = 0; j < n_out; j++) {
        const double* q = &rows[(size_t)j * IGA_ARRIVAL_COLS];
        print_eigenray(q, o.src, o.verbose);
        rc = write_eigenray_file(id + ".eigenray-" + std::to_string(j) + ".dat", atmo, ep.fan, o.src, q[0], q[1], (int)q[2],
                                 sph);
        if (rc) return fail("eigenray path", rc);
    }
    if (!direct) std::cout << '\t' << "Identified " << n_out << " eigenray(s)." << '\n';
    iga_atmo_destroy(atmo);
    return 0;
}

// ------------------------------------------------------------------------
// -back_proj (infraga-3d, flat ground): run_back_proj, main.infraga.3d.cpp:559-770
// ------------------------------------------------------------------------

// One ray from the receiver through the reversed winds; {id}.projection.dat
// holds its rows m == 1 and m % 5 == 0 with the inclination / azimuth
// derivatives of position and travel time and the group velocity
// (iga_fan_paths, IGA_PATH_PROJ), the console the arrival at the last bounce.
int run_back_3dr(int argc, char** argv, Variant v);
void write_projection(const std::string& id, const std::vector<double>& rows, long long np);
void print_back_arrival(const std::vector<double>& arr, int n_out, int nb);

int run_back(int argc, char** argv, Variant v) {
    if (v == Variant::k3DRngdep) return run_back_3dr(argc, argv, v);
    if (v != Variant::k3D) {
        std::cout << "-back_proj is not provided by the GPU front end." << '\n';
        return 0;
    }
    banner(v, "Back Projection");
    const char* fmt = "zTuvdp";
    const char* topo = nullptr;
    const char* val;
    for (int i = 3; i < argc; i++) {
        if (key(argv[i], "prof_format=", &val)) fmt = val;
        else if (key(argv[i], "topo_file=", &val)) topo = val;
    }
    if (topo) {
        std::cout << '\t' << "ERROR: -back_proj over terrain is not provided by the GPU front end" << '\n';
        return 0;
    }
    std::cout << "Interpolating atmosphere data in '" << argv[2] << "' using format '" << fmt << "'..." << '\n';
    std::cout << '\t' << "Inverting wind fields for back projection analysis..." << '\n';
    iga_atmo_t atmo = nullptr;
    int rc = iga_atmo_load(argv[2], fmt, 1, &atmo);   // set_region(..., true): winds reversed
    if (rc == IGA_E_IO) {
        std::cout << '\t' << "ERROR: Invalid atmospheric specification (" << argv[2] << ")" << '\n' << '\t'
                  << iga_strerror(rc) << '\n' << '\n';
        return 0;
    }
    if (rc) return fail("loading the atmosphere", rc);
    iga_fan_params p;
    if ((rc = iga_fan_params_default(atmo, &p))) return fail("parameters", rc);
    print_region(v, p);
    PropOpts o;
    double incl = 15.0, az = 90.0, xr = 0.0, yr = 0.0, freq = 0.1;
    int bounces = 0;
    for (int i = 3; i < argc; i++) {
        const char* a = argv[i];
        if (key(a, "inclination=", &val)) incl = atof(val);
        else if (key(a, "azimuth=", &val)) az = atof(val);
        else if (key(a, "bounces=", &val)) bounces = std::max(0, atoi(val));
        else if (key2(a, "rcvr_x=", "x_rcvr=", &val)) xr = atof(val);
        else if (key2(a, "rcvr_y=", "y_rcvr=", &val)) yr = atof(val);
        else if (common_key(v, a, p, o, false, freq)) {}
        else if (!confirm_unknown(a, false)) return 0;
    }
    if (o.use_blw) {
        std::cout << '\t' << "ERROR: topo_use_BLw (boundary-layer vertical winds) is not provided by the GPU front end" << '\n';
        return 0;
    }
    const double zr = std::max(p.z_grnd, 0.0);   // z_rcvr = max(topo::z, 0)
    if (o.write_atmo && (rc = write_atmo_file(atmo, p, xr, yr, Pi / 2.0 - az * (Pi / 180.0))))
        return fail("write_atmo", rc);
    // the reference echoes geoac::theta / phi converted back to degrees
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << "inclination: " << incl * (Pi / 180.0) * (180.0 / Pi) << '\n';
    std::cout << '\t' << "azimuth: " << 90.0 - (Pi / 2.0 - az * (Pi / 180.0)) * (180.0 / Pi) << '\n';
    std::cout << '\t' << "bounces: " << bounces << '\n';
    std::cout << '\t' << "receiver location: " << xr << ", " << yr << ", " << zr << '\n';
    std::cout << '\t' << "ground elevation: " << p.z_grnd << '\n';
    std::cout << '\t' << "frequency: " << freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << p.tweak_abs << '\n' << '\n';
    if (!o.output_id) {
        strip_extension(argv[2]);
        o.output_id = argv[2];
    }
    const std::string id = o.output_id;
    p.bounces = bounces;
    p.calc_amp = 1;
    p.write_rays = 1;
    p.src[0] = xr; p.src[1] = yr; p.src[2] = zr;
    p.freq = freq;
    p.turn_ht_min = -1.0e30;   // run_back_proj has no turning-height cut
    p.precision = IGA_FP64;
    const int nb = bounces + 1;
    std::vector<double> arr((size_t)nb * IGA_ARRIVAL_COLS);
    long long st = 0;
    int n_out = 0;
    rc = iga_fan_run(atmo, &p, &incl, &az, 1, arr.data(), nb, &n_out, nullptr, &st, nullptr, nullptr, nullptr);
    if (rc) return fail("back projection", rc);
    const long long cap = (long long)nb + st / 5 + 1;
    std::vector<double> rows((size_t)cap * IGA_PROJ_COLS);
    long long np = 0;
    rc = iga_fan_paths(atmo, &p, &incl, &az, 1, IGA_PATH_PROJ, &st, rows.data(), cap, &np, nullptr, nullptr, 0, nullptr,
                       nullptr);
    if (rc) return fail("back projection rows", rc);
    write_projection(id, rows, np);
    print_back_arrival(arr, n_out, nb);
    iga_atmo_destroy(atmo);
    return 0;
}

// {id}.projection.dat of run_back_proj: header and the np rows
void write_projection(const std::string& id, const std::vector<double>& rows, long long np) {
    std::ofstream f((id + ".projection.dat").c_str());
    f << "# x [km]" << '\t' << "y [km]" << '\t' << "z [km]" << '\t' << "time [s]" << '\t' << "X^{(incl)} [km/deg]" << '\t'
      << "Y^{(incl)} [km/deg]" << '\t' << "Z^{(incl)} [km/deg]" << '\t' << "T^{(incl)} [s/deg]" << '\t'
      << "X^{(az)} [km/deg]" << '\t' << "Y^{(az)} [km/deg]" << '\t' << "Z^{(az)} [km/deg]" << '\t' << "T^{(az)} [s/deg]"
      << '\t' << "c_{g,x} [m/s]" << '\t' << "c_{g,y} [m/s]" << '\t' << "c_{g,z} [m/s]" << '\n';
    for (long long j = 0; j < np; j++) {
        const double* q = &rows[(size_t)j * IGA_PROJ_COLS];
        f << q[0];
        for (int c = 1; c < IGA_PROJ_COLS; c++) f << '\t' << q[c];
        f << '\n';
    }
}

// the arrival after the last bounce, as run_back_proj prints it
void print_back_arrival(const std::vector<double>& arr, int n_out, int nb) {
    if (n_out == nb) {
        const double* q = &arr[(size_t)(nb - 1) * IGA_ARRIVAL_COLS];
        std::cout << '\t' << "Back projected arrival:" << '\n';
        std::cout << '\t' << '\t' << "x [km E-W] = " << q[3] << '\n';
        std::cout << '\t' << '\t' << "y [km N-S] = " << q[4] << '\n';
        std::cout << '\t' << '\t' << "time [s] = " << q[5] << '\n';
        std::cout << '\t' << '\t' << "celerity [km/s] = " << q[6] << '\n';
        std::cout << '\t' << '\t' << "turning height [km] = " << q[7] << '\n';
        std::cout << '\t' << '\t' << "arrival inclination [deg] = " << q[8] << '\n';
        std::cout << '\t' << '\t' << "back azimuth = " << q[9] << '\n';
        std::cout << '\t' << '\t' << "trans. coeff. [dB] = " << q[10] << '\n';
        std::cout << '\t' << '\t' << "absorption [dB] = " << q[11] << '\n' << '\n';
    } else {
        std::cout << '\n' << '\t' << '\t' << "Ray path does not return to the ground." << '\n' << '\n';
    }
}

// -back_proj of infraga-3d-rngdep (run_back_proj, main.infraga.3d.rngdep.cpp:548-750):
// one ray from the receiver through the reversed winds of the node grid, flat
// ground (topo::z = 0) or terrain; {id}.projection.dat rows m == 1 and m % 5
// == 0 with the altitude held at the terrain, the console the arrival at the
// last bounce.
int run_back_3dr(int argc, char** argv, Variant v) {
    banner(v, "Back Projection");
    const char* topo = nullptr;
    iga_atmo_t atmo = load_atmosphere(v, argc, argv, &topo, true);   // set_region(..., true): winds reversed
    if (!atmo) return 0;
    const bool has_topo = topo != nullptr;
    iga_fan_params p;
    int rc = iga_fan_params_init(atmo, IGA_GEOM_3D, &p);
    if (rc) return fail("parameters", rc);
    print_region(v, p);
    PropOpts o;
    double incl = 15.0, az = 90.0, xr = 0.0, yr = 0.0, freq = 0.1;
    if (has_topo) {   // the receiver defaults to the centre of the region (main.infraga.3d.rngdep.cpp:585-588)
        xr = (p.x_max + p.x_min) / 2.0;
        yr = (p.y_max + p.y_min) / 2.0;
    }
    int bounces = 0;
    const char* val;
    for (int i = 5; i < argc; i++) {
        const char* a = argv[i];
        if (key(a, "inclination=", &val)) incl = atof(val);
        else if (key(a, "azimuth=", &val)) az = atof(val);
        else if (key(a, "bounces=", &val)) bounces = std::max(0, atoi(val));
        else if (key2(a, "rcvr_x=", "x_rcvr=", &val)) xr = atof(val);
        else if (key2(a, "rcvr_y=", "y_rcvr=", &val)) yr = atof(val);
        else if (common_key(v, a, p, o, has_topo, freq)) {}
        else if (!confirm_unknown(a, false)) return 0;
    }
    if (o.use_blw) {
        std::cout << '\t' << "ERROR: topo_use_BLw (boundary-layer vertical winds) is not provided by the GPU front end" << '\n';
        return 0;
    }
    double zr = 0.0;   // z_rcvr = max(topo::z(x, y), 0); topo::z = 0 without terrain
    if (has_topo) {
        double zz = 0.0;
        iga_atmo_terrain(atmo, xr, yr, &zz, nullptr, nullptr);
        zr = std::max(zz, 0.0);
    }
    if (o.write_atmo && (rc = write_atmo_file(atmo, p, xr, yr, Pi / 2.0 - az * (Pi / 180.0))))
        return fail("write_atmo", rc);
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << "inclination: " << incl * (Pi / 180.0) * (180.0 / Pi) << '\n';
    std::cout << '\t' << "azimuth: " << 90.0 - (Pi / 2.0 - az * (Pi / 180.0)) * (180.0 / Pi) << '\n';
    std::cout << '\t' << "bounces: " << bounces << '\n';
    std::cout << '\t' << "receiver location: " << xr << ", " << yr << ", " << zr << '\n';
    if (!has_topo) std::cout << '\t' << "ground elevation: " << p.z_grnd << '\n';
    std::cout << '\t' << "frequency: " << freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << p.tweak_abs << '\n' << '\n';
    if (!o.output_id) {
        strip_extension(argv[2]);
        o.output_id = argv[2];
    }
    const std::string id = o.output_id;
    p.bounces = bounces;
    p.calc_amp = 1;
    p.write_rays = 1;
    p.src[0] = xr; p.src[1] = yr; p.src[2] = zr;
    p.freq = freq;
    p.turn_ht_min = -1.0e30;   // run_back_proj has no turning-height cut
    p.precision = IGA_FP64;
    const int nb = bounces + 1;
    std::vector<double> arr((size_t)nb * IGA_ARRIVAL_COLS);
    long long st = 0;
    int n_out = 0;
    rc = iga_fan_run(atmo, &p, &incl, &az, 1, arr.data(), nb, &n_out, nullptr, &st, nullptr, nullptr, nullptr);
    if (rc) return fail("back projection", rc);
    const long long cap = (long long)nb + st / 5 + 1;
    std::vector<double> rows((size_t)cap * IGA_PROJ_COLS);
    long long np = 0;
    rc = iga_fan_paths(atmo, &p, &incl, &az, 1, IGA_PATH_PROJ, &st, rows.data(), cap, &np, nullptr, nullptr, 0, nullptr,
                       nullptr);
    if (rc) return fail("back projection rows", rc);
    write_projection(id, rows, np);
    print_back_arrival(arr, n_out, nb);
    iga_atmo_destroy(atmo);
    return 0;
}

// ------------------------------------------------------------------------
// -wnl_wvfrm (infraga-3d, flat ground): run_wnl_wvfrm, main.infraga.3d.cpp:1087-1420
// ------------------------------------------------------------------------

// wvfrm:: settings (util/waveforms.cpp:21-37)
struct WaveOpts {
    double p0 = 10.0, t0 = 0.1, alpha = 4.0;
    long len = 8192;
    int N_rise = 10, N_period = 40;
    const char* file = "none";
    const char* opt = "impulse";
};

// wvfrm::impulse and wvfrm::n_wave (waveforms.cpp:42-62)
double wv_impulse(const WaveOpts& w, double t) {
    if (t < 0.0) return 0.0;
    const double x = t / w.t0, x_pk = (w.alpha + 1.0) - sqrt(w.alpha + 1.0);
    double r = pow(x, w.alpha) * (1.0 - x / (1.0 + w.alpha)) * exp(-x);
    r /= pow(x_pk, w.alpha) * (1.0 - x_pk / (1.0 + w.alpha)) * exp(-x_pk);
    return r;
}
double wv_nwave(const WaveOpts& w, double t) { return fabs(t) <= w.t0 ? t / w.t0 : 0.0; }

// wvfrm::build_wvfrm / load_wvfrm (waveforms.cpp:67-147): t [s], p [Pa]
bool make_waveform(WaveOpts& w, std::vector<double>& t, std::vector<double>& pw) {
    if (strncmp(w.file, "none", 4) != 0) {
        std::cout << '\t' << "Loading waveform from file: " << w.file << "." << '\n';
        std::ifstream f(w.file);
        if (!f.is_open()) return false;
        long len = 0;   // file_length: lines not starting with '#', minus one
        std::string line;
        while (!f.eof()) {
            std::getline(f, line);
            if (line.find('#') != 0) len++;
        }
        len -= 1;
        if (len < 2) return false;
        f.clear();
        f.seekg(0);
        w.len = len;
        t.assign(len, 0.0); pw.assign(len, 0.0);
        long n = 0;
        while (!f.eof() && n < len) {
            std::getline(f, line);
            if (line.find('#') != 0) {
                std::stringstream ss(line);
                ss >> t[n];
                ss >> pw[n];
                n++;
            }
        }
        return true;
    }
    const long len = w.len;
    t.resize(len); pw.resize(len);
    const char* o = w.opt;
    double duration;
    if (strncmp(o, "impulse", 7) == 0) {
        w.alpha = std::max(w.alpha, 0.01);
        duration = w.t0 * len * std::max(((1.0 + w.alpha) - sqrt(1.0 + w.alpha)) / w.N_rise,
                                         2.0 * 3.14159 * sqrt(1 + w.alpha) / w.N_period);
        std::cout << '\t' << "Defining waveform from built in impulse with shaping parameter = " << w.alpha << "." << '\n';
        for (long n = 0; n < len; n++) {
            t[n] = -duration / 2.0 + duration * n / len;
            pw[n] = w.p0 * wv_impulse(w, t[n]);
        }
    } else if (strncmp(o, "Uwave", 5) == 0 || strncmp(o, "u-wave", 6) == 0 || strncmp(o, "U-wave", 6) == 0) {
        w.alpha = std::max(w.alpha, 2.0);
        duration = w.t0 * len * std::max(((1.0 + w.alpha) - sqrt(1.0 + w.alpha)) / w.N_rise,
                                         2.0 * 3.14159 * sqrt(1 + w.alpha) / w.N_period);
        std::cout << '\t' << "Defining waveform from built in U-wave with shaping parameter = " << w.alpha << "." << '\n';
        const double eps = 1.0e-2;
        for (long n = 0; n < len; n++) {
            t[n] = -duration / 2.0 + duration * n / len;
            pw[n] = w.p0 * (wv_impulse(w, t[n] + eps) - wv_impulse(w, t[n] - eps)) / (2.0 * eps);
            pw[n] /= 1.126 * (wv_impulse(w, eps) - wv_impulse(w, -eps)) / (2.0 * eps);
        }
    } else if (strncmp(o, "Nwave", 5) == 0 || strncmp(o, "n-wave", 6) == 0 || strncmp(o, "N-wave", 6) == 0) {
        duration = (w.t0 / w.N_period) * len;
        std::cout << '\t' << "Defining waveform from built in N-wave." << '\n';
        for (long n = 0; n < len; n++) {
            t[n] = -duration / 2.0 + duration * n / len;
            pw[n] = -w.p0 * wv_nwave(w, t[n] - w.t0 / 2.0);
        }
    } else {
        // the fallback takes the shorter of the two time scales (waveforms.cpp:127-130)
        w.alpha = std::max(w.alpha, 0.01);
        duration = w.t0 * len * std::min(((1.0 + w.alpha) - sqrt(1.0 + w.alpha)) / w.N_rise,
                                         2.0 * 3.14159 * sqrt(1 + w.alpha) / w.N_period);
        std::cout << '\t' << "Warning!!  Unrecognized option in waveform.  Options are 'impulse', 'Uwave', and 'Nwave'  Using "
                  << "impulse with shaping parameter " << w.alpha << "." << '\n';
        for (long n = 0; n < len; n++) {
            t[n] = -duration / 2.0 + duration * n / len;
            pw[n] = w.p0 * wv_impulse(w, t[n]);
        }
    }
    return true;
}

int run_wnl(int argc, char** argv, Variant v) {
    if (v != Variant::k3D && v != Variant::kSph) {
        std::cout << "-wnl_wvfrm is not provided by the GPU front end." << '\n';
        return 0;
    }
    const bool sph = v == Variant::kSph;   // run_wnl_wvfrm of main.infraga.sph.cpp:1142-1480
    std::cout << '\n';
    if (sph) {
        std::cout << '\t' << "###########################################" << '\n';
        std::cout << '\t' << "####        Running infraga-sph        ####" << '\n';
        std::cout << '\t' << "####     Weakly Non-Linear Waveform    ####" << '\n';
        std::cout << '\t' << "###########################################" << '\n' << '\n';
    } else {
        std::cout << '\t' << "##########################################" << '\n';
        std::cout << '\t' << "####        Running infraga-3d        ####" << '\n';
        std::cout << '\t' << "####    Weakly Non-Linear Waveform    ####" << '\n';
        std::cout << '\t' << "##########################################" << '\n' << '\n';
    }
    const char* topo = nullptr;
    const char* val;
    for (int i = 3; i < argc; i++)
        if (key(argv[i], "topo_file=", &val)) topo = val;
    if (topo) {
        std::cout << '\t' << "ERROR: -wnl_wvfrm over terrain is not provided by the GPU front end" << '\n';
        return 0;
    }
    iga_atmo_t atmo = load_atmosphere(v, argc, argv, &topo);
    if (!atmo) return 0;
    iga_wnl_params wp;
    int rc = iga_wnl_params_default(atmo, &wp);
    if (!rc && sph) rc = iga_fan_params_init(atmo, IGA_GEOM_SPH, &wp.fan);
    if (rc) return fail("parameters", rc);
    iga_fan_params& p = wp.fan;
    print_region(v, p);
    PropOpts o;
    WaveOpts w;
    double incl = 15.0, az = 90.0, xs = sph ? 30.0 : 0.0, ys = 0.0, zs = 0.0, freq = 0.1;
    int bounces = 0;
    bool write_rays = false;
    for (int i = 3; i < argc; i++) {
        const char* a = argv[i];
        if (key(a, "inclination=", &val)) incl = atof(val);
        else if (key(a, "azimuth=", &val)) az = atof(val);
        else if (key(a, "bounces=", &val)) bounces = std::max(0, atoi(val));
        else if (!sph && key2(a, "src_x=", "x_src=", &val)) xs = atof(val);
        else if (!sph && (key(a, "src_y=", &val) || match(a, "y_src_y=", 6, 6, &val))) ys = atof(val);
        else if (sph && key2(a, "src_lat=", "lat_src=", &val)) xs = atof(val);
        else if (sph && key2(a, "src_lon=", "lon_src=", &val)) ys = atof(val);
        else if (key2(a, "src_alt=", "alt_src=", &val)) zs = atof(val);
        else if (key(a, "write_ray=", &val)) write_rays = str2bool(val);
        else if (key(a, "wvfrm_file=", &val)) w.file = val;
        else if (key(a, "wvfrm_opt=", &val)) w.opt = val;
        else if (key(a, "wvfrm_p0=", &val)) w.p0 = atof(val);
        else if (key(a, "wvfrm_t0=", &val)) w.t0 = atof(val);
        else if (key(a, "wvfrm_alpha=", &val)) w.alpha = atof(val);
        else if (key(a, "wvfrm_ref=", &val)) wp.wvfrm_ref = atof(val);
        else if (key(a, "wvfrm_out_step=", &val)) wp.out_step = atof(val);
        else if (key(a, "wvfrm_ds=", &val)) wp.ds_wvfrm = atof(val);
        // the reference reads N_rise from 15 characters in (its key has 13)
        else if (match(a, "wvfrm_N_rise=", 13, 15, &val)) w.N_rise = (int)atof(a + std::min<size_t>(15, strlen(a)));
        else if (key(a, "wvfrm_N_period=", &val)) w.N_period = (int)atof(val);
        else if (key(a, "wvfrm_len=", &val)) w.len = (long)atof(val);
        else if (key(a, "wvfrm_filt1_g=", &val)) wp.filt1_g = atof(val);
        else if (key(a, "wvfrm_filt1_n1=", &val)) wp.filt1_n1 = atof(val);
        else if (key(a, "wvfrm_filt1_n2=", &val)) wp.filt1_n2 = atof(val);
        else if (key(a, "wvfrm_filt2_g=", &val)) wp.filt2_g = atof(val);
        else if (key(a, "wvfrm_filt2_n1=", &val)) wp.filt2_n1 = atof(val);
        else if (key(a, "wvfrm_filt2_n2=", &val)) wp.filt2_n2 = atof(val);
        else if (common_key(v, a, p, o, false, freq)) {}
        else if (!confirm_unknown(a, false)) { iga_atmo_destroy(atmo); return 0; }
    }
    if (o.use_blw) {
        std::cout << '\t' << "ERROR: topo_use_BLw (boundary-layer vertical winds) is not provided by the GPU front end" << '\n';
        iga_atmo_destroy(atmo);
        return 0;
    }
    if (sph) std::cout << "s_max --> " << p.s_max << '\n';
    zs = std::max(p.z_grnd, zs);   // z_src = max(topo::z(src), z_src) over flat ground
    const double theta = incl * (Pi / 180.0), phi = Pi / 2.0 - az * (Pi / 180.0);
    // the spherical driver keeps the source in radians and echoes it back in degrees
    const double xe = sph ? xs * (Pi / 180.0) * (180.0 / Pi) : xs, ye = sph ? ys * (Pi / 180.0) * (180.0 / Pi) : ys;
    if (o.write_atmo && (rc = write_atmo_file(atmo, p, xs, ys, phi))) return fail("write_atmo", rc);
    const double alpha_in = w.alpha;
    std::cout << '\n' << "Parameter summary:" << '\n';
    std::cout << '\t' << "inclination: " << theta * (180.0 / Pi) << '\n';
    std::cout << '\t' << "azimuth: " << 90.0 - phi * (180.0 / Pi) << '\n';
    std::cout << '\t' << "bounces: " << bounces << '\n';
    std::cout << '\t' << (sph ? "source location (lat, lon, alt): " : "source location: ") << xe << ", " << ye << ", "
              << zs << '\n';
    std::cout << '\t' << "ground elevation: " << p.z_grnd << '\n';
    std::cout << '\t' << "frequency: " << freq << '\n';
    std::cout << '\t' << "S&B atten coeff: " << p.tweak_abs << '\n';
    if (strncmp(w.file, "none", 4) != 0) {
        std::cout << '\t' << "waveform source file: " << w.file << '\n';
    } else {
        std::cout << '\t' << "waveform option: " << w.opt << '\n';
        std::cout << '\t' << "waveform p0: " << w.p0 << '\n';
        std::cout << '\t' << "waveform t0: " << w.t0 << '\n';
        std::cout << '\t' << "waveform alpha: " << alpha_in << '\n';
    }
    std::cout << '\t' << "waveform reference location: " << wp.wvfrm_ref << '\n' << '\n';
    if (!o.output_id) {
        strip_extension(argv[2]);
        o.output_id = argv[2];
    }
    const std::string id = o.output_id;
    p.bounces = bounces;
    p.src[0] = xs; p.src[1] = ys; p.src[2] = zs;
    p.freq = freq;
    p.turn_ht_min = -1.0e30;
    if (sph) p.time_max = 1.0e30;
    std::ofstream raypath;   // opened before the trace, as the reference does
    if (write_rays) {
        raypath.open((id + ".raypaths.dat").c_str());
        if (sph)
            raypath << "# z [km]" << '\t' << "lat [deg]" << '\t' << "lon [deg]";
        else
            raypath << "# x [km]" << '\t' << "y [km]" << '\t' << "z [km]";
        raypath << '\t' << "trans. coeff. [dB]" << '\t' << "absorption [dB]" << '\t' << "time [s]" << '\n';
    }
    std::cout << "Calculating ray path geometry and weakly non-linear waveform evolution..." << '\n';
    std::vector<double> wt, wpr;
    if (!make_waveform(w, wt, wpr)) {
        std::cout << '\t' << "ERROR: cannot read the waveform file " << w.file << '\n';
        iga_atmo_destroy(atmo);
        return 0;
    }
    const int N = (int)w.len;
    if (write_rays) {   // {id}.raypaths.dat rows m == 1 and m % 15 == 0 (main.infraga.3d.cpp:1287-1309)
        iga_fan_params q = p;
        q.calc_amp = 1; q.write_rays = 1; q.precision = IGA_FP64;
        std::vector<double> arr((size_t)(bounces + 1) * IGA_ARRIVAL_COLS);
        long long st = 0;
        int n_out = 0;
        if ((rc = iga_fan_run(atmo, &q, &incl, &az, 1, arr.data(), bounces + 1, &n_out, nullptr, &st, nullptr, nullptr,
                              nullptr)))
            return fail("ray path", rc);
        const long long cap = (long long)(bounces + 1) + st / 15 + 1;
        std::vector<double> rows((size_t)cap * IGA_PATH_COLS);
        long long np = 0;
        if ((rc = iga_fan_paths(atmo, &q, &incl, &az, 1, IGA_PATH_RAYS, &st, rows.data(), cap, &np, nullptr, nullptr, 0,
                                nullptr, nullptr)))
            return fail("ray path rows", rc);
        for (long long j = 0; j < np; j++) {
            const double* r = &rows[(size_t)j * IGA_PATH_COLS];
            if (sph) raypath << std::setprecision(8) << r[0] << '\t' << std::setprecision(8) << r[1];
            else raypath << r[0] << '\t' << r[1];
            raypath << '\t' << r[2] << '\t' << r[3] << '\t' << r[4] << '\t' << r[5] << '\n';
        }
    }
    // the waveform along the ray: events first sized by the ray length bound,
    // grown once if the kernel reports more
    const int nb = bounces + 1;
    const int M1 = N / 2 + 1;
    const size_t snap_w = 1 + (size_t)N + 2 * (size_t)M1;
    std::vector<double> u(N), info(IGA_WNL_INFO), arr((size_t)nb * IGA_ARRIVAL_COLS);
    int n_arr = 0, status = 0;
    int ev_cap = 4096, sn_cap = wp.out_step < 1.0e4 ? 64 : 0;
    std::vector<double> ev, sn;
    for (int attempt = 0; attempt < 2; attempt++) {
        ev.assign((size_t)ev_cap * IGA_WNL_EVENT_COLS, 0.0);
        sn.assign((size_t)sn_cap * snap_w, 0.0);
        rc = iga_wnl_run(atmo, &wp, &incl, &az, 1, wt.data(), wpr.data(), N, u.data(), info.data(), arr.data(), &n_arr,
                         &status, ev.data(), ev_cap, sn_cap ? sn.data() : nullptr, sn_cap);
        if (rc != IGA_E_TRUNCATED) break;
        ev_cap = std::max(ev_cap, (int)info[IGA_WNL_EVENTS]);
        sn_cap = std::max(sn_cap, (int)info[IGA_WNL_SNAPS]);
    }
    if (rc) {
        fail("waveform", rc);
        iga_atmo_destroy(atmo);
        return 0;
    }
    const bool started = info[IGA_WNL_STATUS] == 0.0;
    std::ofstream wout;   // one stream for both files, as the reference (its precision carries over)
    if (started) {
        wout.open((id + ".wvfrm_init.dat").c_str());
        wout << "# t [sec]" << '\t' << "p(t) [Pa]" << '\n';
        for (int n = 0; n < N; n++) wout << std::setprecision(8) << info[IGA_WNL_T_REF] + wt[n] << '\t' << wpr[n] << '\n';
        wout.close();
    }
    const int n_ev = std::min((int)info[IGA_WNL_EVENTS], ev_cap);
    const int n_sn = std::min((int)info[IGA_WNL_SNAPS], sn_cap);
    const double dt = wt[1] - wt[0];
    char buf[512];
    for (int j = 0; j < n_ev; j++) {
        const double* e = &ev[(size_t)j * IGA_WNL_EVENT_COLS];
        if (e[0] == 0.0)
            std::cout << '\t' << (sph ? "Generating" : "Computing") << " waveform at ray length: " << e[1] << '\t'
                      << "altitude: " << e[2] << '\t' << "scaled non-linearity factor: " << e[3] << '\n';
        else
            std::cout << '\t' << "Caustic encountered." << '\n';
    }
    for (int j = 0; j < n_sn; j++) {   // sc_spectrum / sc_waveform files (geoac.eqset.3d.strat.cpp:874-887)
        const double* q = &sn[(size_t)j * snap_w];
        snprintf(buf, sizeof(buf), "sc_spectrum-%04g.dat", q[0]);
        std::ofstream fs(buf);
        for (int k = 0; k < M1; k++)
            fs << 1.0 / dt * k / N << '\t' << q[1 + N + 2 * k] << '\t' << q[2 + N + 2 * k] << '\n';
        fs.close();
        snprintf(buf, sizeof(buf), "sc_waveform-%04g.dat", q[0]);
        std::ofstream fw(buf);
        for (int n = 0; n < N; n++) fw << wt[n] << '\t' << q[1 + n] << '\n';
    }
    const bool landed = (status == 0) && n_arr == nb;
    const double tt = landed ? arr[(size_t)(nb - 1) * IGA_ARRIVAL_COLS + 5] : info[IGA_WNL_TIME];
    if (landed && sph) {   // the latitude's setprecision(8) stays on the stream
        const double* q = &arr[(size_t)(nb - 1) * IGA_ARRIVAL_COLS];
        std::cout << '\n';
        std::cout << '\t' << "Arrival summary:" << '\n';
        std::cout << '\t' << '\t' << "latitude [deg] = " << std::setprecision(8) << q[3] << '\n';
        std::cout << '\t' << '\t' << "longitude [deg] = " << std::setprecision(8) << q[4] << '\n';
        std::cout << '\t' << '\t' << "time [s] = " << q[5] << '\n';
        std::cout << '\t' << '\t' << "celerity [km/s] = " << q[6] << '\n';
        std::cout << '\t' << '\t' << "turning height [km] = " << q[7] << '\n';
        std::cout << '\t' << '\t' << "arrival inclination [deg] = " << q[8] << '\n';
        std::cout << '\t' << '\t' << "back azimuth [deg] = " << q[9] << '\n';
        std::cout << '\t' << '\t' << "trans. coeff. [dB] = " << q[10] << '\n';
        std::cout << '\t' << '\t' << "absorption [dB] = " << q[11] << '\n' << '\n';
    } else if (landed) {
        const double* q = &arr[(size_t)(nb - 1) * IGA_ARRIVAL_COLS];
        std::cout << '\n';
        std::cout << '\t' << "Arrival summary:" << '\n';
        std::cout << '\t' << '\t' << "x [km E-W] = " << q[3] << '\n';
        std::cout << '\t' << '\t' << "y [km N-S] = " << q[4] << '\n';
        std::cout << '\t' << '\t' << "time [s] = " << q[5] << '\n';
        std::cout << '\t' << '\t' << "celerity [km/s] = " << q[6] << '\n';
        std::cout << '\t' << '\t' << "turning height [km] = " << q[7] << '\n';
        std::cout << '\t' << '\t' << "arrival inclination [deg] = " << q[8] << '\n';
        std::cout << '\t' << '\t' << "back azimuth = " << q[9] << '\n';
        std::cout << '\t' << '\t' << "attenuation (geometric) [dB] = " << q[10] << '\n';
        std::cout << '\t' << '\t' << "absorption [dB] = " << q[11] << '\n' << '\n';
    } else {
        std::cout << '\n';
        std::cout << '\t' << '\t' << "Ray path does not return to the ground." << '\n' << '\n';
    }
    if (!started)
        std::cout << '\t' << "Note: the ray is shorter than wvfrm_ref; no waveform was carried along it." << '\n';
    wout.open((id + ".wvfrm_out.dat").c_str());
    wout << (sph ? "# infraga-sph -wnl_wvfrm summary:" : "# infraga-3d -wnl_wvfrm summary:") << '\n';
    wout << "#" << '\t' << "profile: " << argv[2] << '\n';
    wout << "#" << '\t' << "inclination: " << theta * (180.0 / Pi) << '\n';
    wout << "#" << '\t' << "azimuth: " << phi * (180.0 / Pi) << '\n';
    wout << "#" << '\t' << "bounces: " << bounces << '\n';
    wout << "#" << '\t' << (sph ? "source (lat, lon, alt): " : "source location: ") << xe << ", " << ye << ", " << zs
         << '\n';
    wout << "#" << '\t' << "ground elevation: " << p.z_grnd << '\n';
    wout << "#" << '\t' << "S&B atten coeff: " << p.tweak_abs << '\n';
    if (strncmp(w.file, "none", 4) != 0) {
        wout << "#" << '\t' << "waveform source file: " << w.file << '\n';
    } else {
        wout << "#" << '\t' << "waveform option: " << w.opt << '\n';
        wout << "#" << '\t' << "waveform p0: " << w.p0 << '\n';
        wout << "#" << '\t' << "waveform t0: " << w.t0 << '\n';
        wout << "#" << '\t' << "waveform alpha: " << w.alpha << '\n';
    }
    wout << "#" << '\t' << "waveform reference location: " << wp.wvfrm_ref << '\n' << '\n';
    wout << "# t [sec]" << '\t' << "p(t) [Pa]" << '\n';
    const double p0 = info[IGA_WNL_P0], sc = info[IGA_WNL_SCALE];
    for (int n = 0; n < N; n++) {
        wout << std::setprecision(8) << tt + wt[n];
        wout << '\t' << (started ? u[n] * p0 * sc : 0.0);
        wout << '\n';
    }
    wout.close();
    iga_atmo_destroy(atmo);
    return 0;
}

}  // namespace

int run(int argc, char** argv, Variant v, bool accel) {
    g_launch.accel = accel;
    if (accel) {
        if (launch_rank() > 0) return 0;   // one GPU process does the work of the whole launch
        g_launch.threads = launch_size();
    }
    const int min_args = is_rngdep(v) ? 5 : 3;
    if (argc < min_args) {
        usage(v);
        return 0;
    }
    const char* o = argv[1];
    if (strncmp(o, "-version", 8) == 0 || strncmp(o, "-v", 2) == 0) version();
    else if (strncmp(o, "-usage", 6) == 0 || strncmp(o, "-u", 2) == 0) usage(v);
    else if (strncmp(o, "-prop", 5) == 0 || strncmp(o, "-p", 2) == 0) return run_prop(argc, argv, v);
    else if (strncmp(o, "-back_proj", 10) == 0 || strncmp(o, "-b", 2) == 0)
        return run_back(argc, argv, v);
    else if (strncmp(o, "-eig_search", 11) == 0 || strncmp(o, "-s", 2) == 0) {
        return run_eig(argc, argv, v, false);
    } else if (strncmp(o, "-eig_direct", 11) == 0 || strncmp(o, "-d", 2) == 0) {
        return run_eig(argc, argv, v, true);
    } else if (strncmp(o, "-wnl_wvfrm", 10) == 0 || strncmp(o, "-w", 2) == 0)
        return run_wnl(argc, argv, v);
    else
        std::cout << "Unrecognized option." << '\n';
    return 0;
}

}  // namespace cli
