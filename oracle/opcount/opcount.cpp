// Operation counts per RK4 ray-step of the reference's 3D stratified fan
// (test infrastructure only; never linked into the product).
//
// Builds the oracle restatement (src/oracle_3d.cpp, bit-identical to the
// reference solver) with every double replaced by the counting scalar of
// opcount.h, traces a fan, and prints the operation counts per accepted RK4
// step as one JSON object per line:
//
//   opcount <profile.met> <calc_amp 0|1> <bounces> <rng_max> <incl_min> <incl_max> <incl_step> <azimuth>
//
// Region "absorption" holds the operations of SB_alpha (atmo::SB_alpha,
// atmo_state.abs.cart.cpp:12-142, one evaluation per step); "rest" holds
// everything else (set_ds, four update_refs + eval_src_eq stages, the RK4
// combination, travel_time's midpoint evaluation, the stop checks, and the
// per-bounce intercept, reflection and arrival record).
//
// The system headers the restatement uses are included first, so that the
// spelling change below applies to the restatement's code only.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "opcount.h"

#define double ocd
#include "../src/oracle_3d.cpp"
#undef double

static void print_counts(const char* name, const OpCounts& c, long long steps, const char* sep) {
    const double s = (double)steps;
    std::printf("\"%s\": {\"add\": %.4f, \"mul\": %.4f, \"div\": %.4f, \"sqrt\": %.4f, \"exp\": %.4f, "
                "\"log\": %.4f, \"pow\": %.4f, \"trig\": %.4f, \"cbrt\": %.4f}%s",
                name, c.add / s, c.mul / s, c.div / s, c.sqrt / s, c.exp / s, c.log / s, c.pow / s, c.trig / s,
                c.cbrt / s, sep);
}

int main(int argc, char** argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s profile.met calc_amp bounces rng_max incl_min incl_max incl_step azimuth\n",
                     argv[0]);
        return 2;
    }
    const char* met = argv[1];
    orc_fan_cfg cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.src[0] = 0.0; cfg.src[1] = 0.0; cfg.src[2] = 0.0;
    cfg.ds_min = 0.001; cfg.ds_max = 0.05; cfg.s_max = 1000.0;
    cfg.alt_max = 150.0; cfg.rng_max = std::atof(argv[4]);
    cfg.x_min = -2000.0; cfg.x_max = 2000.0; cfg.y_min = -2000.0; cfg.y_max = 2000.0;
    cfg.z_grnd = 0.0; cfg.freq = 0.1; cfg.tweak_abs = 1.0; cfg.turn_ht_min = 0.2;
    cfg.bounces = std::atoi(argv[3]);
    cfg.calc_amp = std::atoi(argv[2]);
    cfg.write_rays = 0; cfg.reverse_winds = 0; cfg.n_threads = 1;
    // launch angles with the reference's FP64-accumulated loop (main.infraga.3d.cpp:407-422)
    std::vector<ocd> th, ph;
    const double i0 = std::atof(argv[5]), i1 = std::atof(argv[6]), di = std::atof(argv[7]), az = std::atof(argv[8]);
    for (double t = i0; t <= i1; t += di) { th.push_back(t); ph.push_back(az); }
    const int n = (int)th.size();
    const int nb = cfg.bounces + 1;
    std::vector<ocd> arr((size_t)n * nb * ORC_ARR_COLS);
    std::vector<int> n_arr(n);
    std::vector<long long> steps(n);

    // the profile load and spline build, counted alone and taken off below
    orc::Profile P;
    if (!orc::load_profile(met, "zTuvdp", false, P)) return 1;
    const OpCounts load0 = op_count_table()[0];
    std::memset(op_count_table(), 0, 2 * sizeof(OpCounts));

    if (orc_fan_3d(met, "zTuvdp", &cfg, th.data(), ph.data(), n, arr.data(), n_arr.data(), steps.data(), nullptr) != 0)
        return 1;
    OpCounts rest = op_count_table()[0];
    rest.add -= load0.add; rest.mul -= load0.mul; rest.div -= load0.div; rest.sqrt -= load0.sqrt;
    rest.exp -= load0.exp; rest.log -= load0.log; rest.pow -= load0.pow; rest.trig -= load0.trig;
    rest.cbrt -= load0.cbrt;
    long long tot = 0, arrivals = 0;
    for (int i = 0; i < n; i++) { tot += steps[i]; arrivals += n_arr[i]; }
    std::printf("{\"calc_amp\": %d, \"rays\": %d, \"arrivals\": %lld, \"ray_steps\": %lld, ", cfg.calc_amp, n,
                arrivals, tot);
    print_counts("rest", rest, tot, ", ");
    print_counts("absorption", op_count_table()[1], tot, "}\n");
    return 0;
}
