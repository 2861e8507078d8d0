// CPU oracle (test infrastructure only; never linked into the product).
//
// Restatement of the reference's 1D natural cubic spline and its segment
// search, following src/util/interpolation.cpp.  Kept in the same operation
// order as the reference so that, compiled with the same flags, results are
// bit-identical to the reference solver wherever libm is.
#pragma once
#include <cmath>
#include <vector>
#include <algorithm>

namespace orc {

// interp::natural_cubic_spline_1D (interpolation.h:36-44)
struct Spline1D {
    int n = 0;
    std::vector<double> x, f, s;   // knots, values, Thomas-solved slopes
};

// interp::find_segment (interpolation.cpp:14-49): cached index, then a
// one-step walk up or down, then a two-ended linear scan.
inline int find_segment(double x, const double* xv, int length, int& prev) {
    if (x > xv[length - 1] || x < xv[0]) return prev;   // reference prints and keeps prev
    bool done = false;
    if (x >= xv[prev] && x <= xv[prev + 1]) done = true;
    if (!done && prev + 2 <= length - 1) {
        if (x >= xv[prev + 1] && x <= xv[prev + 2]) { prev++; done = true; }
    }
    if (!done && prev - 1 >= 0) {
        if (x >= xv[prev - 1] && x <= xv[prev]) { prev--; done = true; }
    }
    if (!done) {
        for (int n = 0; n < length; n++) {
            if (x >= xv[n] && x <= xv[n + 1]) { prev = n; break; }
            else if (x >= xv[(length - 1) - (n + 1)] && x < xv[(length - 1) - n]) { prev = (length - 1) - (n + 1); break; }
        }
    }
    return prev;
}

// interp::in_interval (interpolation.cpp:52-54)
inline double in_interval(double x, double lo, double hi) { return std::min(std::max(x, lo), hi); }

// interp::set(natural_cubic_spline_1D&) (interpolation.cpp:103-136): Thomas
// algorithm for the natural end conditions, back substitution into slopes.
inline void spline_set(Spline1D& sp) {
    const int L = sp.n;
    sp.s.assign(L, 0.0);
    std::vector<double> nc(L - 1), nd(L);
    double ai, bi, ci, di;
    bi = 2.0 / (sp.x[1] - sp.x[0]);
    ci = 1.0 / (sp.x[1] - sp.x[0]);
    di = 3.0 * (sp.f[1] - sp.f[0]) / pow(sp.x[1] - sp.x[0], 2);
    nc[0] = ci / bi;
    nd[0] = di / bi;
    for (int i = 1; i < L - 1; i++) {
        double dx1 = sp.x[i] - sp.x[i - 1], dx2 = sp.x[i + 1] - sp.x[i];
        ai = 1.0 / dx1; bi = 2.0 * (1.0 / dx1 + 1.0 / dx2); ci = 1.0 / dx2;
        di = 3.0 * ((sp.f[i] - sp.f[i - 1]) / pow(dx1, 2) + (sp.f[i + 1] - sp.f[i]) / pow(dx2, 2));
        nc[i] = ci / (bi - nc[i - 1] * ai);
        nd[i] = (di - nd[i - 1] * ai) / (bi - nc[i - 1] * ai);
    }
    ai = 1.0 / (sp.x[L - 1] - sp.x[L - 2]);
    bi = 2.0 / (sp.x[L - 1] - sp.x[L - 2]);
    di = 3.0 * (sp.f[L - 1] - sp.f[L - 2]) / pow(sp.x[L - 1] - sp.x[L - 2], 2);
    nd[L - 1] = (di - nd[L - 2] * ai) / (bi - nc[L - 2] * ai);
    sp.s[L - 1] = nd[L - 1];
    for (int i = L - 2; i > -1; i--) sp.s[i] = nd[i] - nc[i] * sp.s[i + 1];
}

// Hermite-form evaluation shared by eval_f/eval_df/eval_ddf/eval_all
// (interpolation.cpp:144-260).
struct SegEval {
    double f, df, ddf;
};
inline void seg_coeffs(const Spline1D& sp, int k, double x, double& dx, double& X, double& df, double& A, double& B) {
    dx = sp.x[k + 1] - sp.x[k];
    X = (x - sp.x[k]) / dx;
    df = sp.f[k + 1] - sp.f[k];
    A = sp.s[k] * dx - df;
    B = -sp.s[k + 1] * dx + df;
}
inline double eval_f(double x, const Spline1D& sp, int& acc) {
    int k = find_segment(x, sp.x.data(), sp.n, acc);
    double dx, X, df, A, B; seg_coeffs(sp, k, x, dx, X, df, A, B);
    return sp.f[k] + X * (df + (1.0 - X) * (A * (1.0 - X) + B * X));
}
inline double eval_df(double x, const Spline1D& sp, int& acc) {
    int k = find_segment(x, sp.x.data(), sp.n, acc);
    double dx, X, df, A, B; seg_coeffs(sp, k, x, dx, X, df, A, B);
    return df / dx + (1.0 - 2.0 * X) * (A * (1.0 - X) + B * X) / dx + X * (1.0 - X) * (B - A) / dx;
}
inline double eval_ddf(double x, const Spline1D& sp, int& acc) {
    int k = find_segment(x, sp.x.data(), sp.n, acc);
    double dx, X, df, A, B; seg_coeffs(sp, k, x, dx, X, df, A, B);
    return 2.0 * (B - 2.0 * A + (A - B) * 3.0 * X) / pow(dx, 2);
}
inline void eval_all(double x, const Spline1D& sp, int& acc, double& f, double& dfdx) {
    int k = find_segment(x, sp.x.data(), sp.n, acc);
    double dx, X, df, A, B; seg_coeffs(sp, k, x, dx, X, df, A, B);
    f = sp.f[k] + X * (df + (1.0 - X) * (A * (1.0 - X) + B * X));
    dfdx = df / dx + (1.0 - 2.0 * X) * (A * (1.0 - X) + B * X) / dx + X * (1.0 - X) * (B - A) / dx;
}
inline void eval_all(double x, const Spline1D& sp, int& acc, double& f, double& dfdx, double& ddfdxdx) {
    int k = find_segment(x, sp.x.data(), sp.n, acc);
    double dx, X, df, A, B; seg_coeffs(sp, k, x, dx, X, df, A, B);
    f = sp.f[k] + X * (df + (1.0 - X) * (A * (1.0 - X) + B * X));
    dfdx = df / dx + (1.0 - 2.0 * X) * (A * (1.0 - X) + B * X) / dx + X * (1.0 - X) * (B - A) / dx;
    ddfdxdx = 2.0 * (B - 2.0 * A + (A - B) * 3.0 * X) / pow(dx, 2);
}

}  // namespace orc
