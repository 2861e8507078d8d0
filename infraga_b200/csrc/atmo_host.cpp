// Host-side stratified atmosphere: .met parsing and FP64 spline tables.
#include "atmo_host.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/infraga_gpu.h"

namespace iga {

static constexpr double kGamma = 1.4;   // atmo::gam (atmo_state.3d.strat.cpp:25)

void natural_spline_slopes(const std::vector<double>& x, const std::vector<double>& f, std::vector<double>& s) {
    // Tridiagonal system for the knot slopes of a natural cubic spline,
    // forward elimination then back substitution; same normalisation as
    // interp::set (interpolation.cpp:103-136) so the slopes agree to rounding.
    const size_t n = x.size();
    s.assign(n, 0.0);
    std::vector<double> cp(n), dp(n);
    double h = x[1] - x[0];
    double b = 2.0 / h, c = 1.0 / h, d = 3.0 * (f[1] - f[0]) / (h * h);
    cp[0] = c / b;
    dp[0] = d / b;
    for (size_t i = 1; i + 1 < n; i++) {
        const double h1 = x[i] - x[i - 1], h2 = x[i + 1] - x[i];
        const double a = 1.0 / h1;
        b = 2.0 * (1.0 / h1 + 1.0 / h2);
        c = 1.0 / h2;
        d = 3.0 * ((f[i] - f[i - 1]) / (h1 * h1) + (f[i + 1] - f[i]) / (h2 * h2));
        const double den = b - cp[i - 1] * a;
        cp[i] = c / den;
        dp[i] = (d - dp[i - 1] * a) / den;
    }
    h = x[n - 1] - x[n - 2];
    const double a = 1.0 / h;
    b = 2.0 / h;
    d = 3.0 * (f[n - 1] - f[n - 2]) / (h * h);
    dp[n - 1] = (d - dp[n - 2] * a) / (b - cp[n - 2] * a);
    s[n - 1] = dp[n - 1];
    for (size_t i = n - 1; i-- > 0;) s[i] = dp[i] - cp[i] * s[i + 1];
}

void spline_eval(const std::vector<double>& x, const std::vector<double>& f, const std::vector<double>& s,
                 double z, double& val, double& d1, double& d2) {
    const int n = (int)x.size();
    z = std::fmin(std::fmax(z, x[0]), x[n - 1]);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (z < x[mid]) hi = mid; else lo = mid;
    }
    const int k = lo;
    const double dx = x[k + 1] - x[k];
    const double X = (z - x[k]) / dx;
    const double df = f[k + 1] - f[k];
    const double A = s[k] * dx - df;
    const double B = -s[k + 1] * dx + df;
    val = f[k] + X * (df + (1.0 - X) * (A * (1.0 - X) + B * X));
    d1 = df / dx + (1.0 - 2.0 * X) * (A * (1.0 - X) + B * X) / dx + X * (1.0 - X) * (B - A) / dx;
    d2 = 2.0 * (B - 2.0 * A + (A - B) * 3.0 * X) / (dx * dx);
}

int finalize_profile(StratProfile& p, std::string& err) {
    const size_t n = p.z.size();
    if (n < 3 || p.c.size() != n || p.u.size() != n || p.v.size() != n || p.rho.size() != n) {
        err = "profile needs at least 3 knots with matching columns";
        return IGA_E_INVALID;
    }
    for (size_t i = 0; i + 1 < n; i++) {
        if (!(p.z[i + 1] > p.z[i])) { err = "profile altitudes must increase strictly"; return IGA_E_INVALID; }
    }
    for (size_t i = 0; i < n; i++) {
        if (!std::isfinite(p.c[i]) || !std::isfinite(p.u[i]) || !std::isfinite(p.v[i]) || !std::isfinite(p.rho[i]) || !(p.c[i] > 0.0)) {
            err = "profile row " + std::to_string(i) + " has a non-finite value or non-positive sound speed";
            return IGA_E_INVALID;
        }
    }
    natural_spline_slopes(p.z, p.c, p.cs);
    natural_spline_slopes(p.z, p.u, p.us);
    natural_spline_slopes(p.z, p.v, p.vs);
    natural_spline_slopes(p.z, p.rho, p.rhos);
    p.table.assign(n * kKnotStride, 0.0);
    for (size_t i = 0; i < n; i++) {
        double* r = &p.table[i * kKnotStride];
        r[kZ] = p.z[i];
        r[kInvDz] = (i + 1 < n) ? 1.0 / (p.z[i + 1] - p.z[i]) : 0.0;
        r[kC] = p.c[i]; r[kCs] = p.cs[i];
        r[kU] = p.u[i]; r[kUs] = p.us[i];
        r[kV] = p.v[i]; r[kVs] = p.vs[i];
        r[kRho] = p.rho[i]; r[kRhos] = p.rhos[i];
    }
    const double h0 = p.z[1] - p.z[0];
    p.uniform = true;
    for (size_t i = 1; i + 1 < n; i++) {
        if (std::fabs((p.z[i + 1] - p.z[i]) - h0) > 1e-9 * std::fabs(h0)) { p.uniform = false; break; }
    }
    p.inv_dz = 1.0 / h0;
    return IGA_OK;
}

int load_met(const char* path, const char* format, bool reverse_winds, StratProfile& out, std::string& err) {
    int fmt;
    if (strncmp(format, "zTuvdp", 6) == 0) fmt = 0;
    else if (strncmp(format, "zuvwTdp", 7) == 0) fmt = 1;
    else if (strncmp(format, "zcuvd", 5) == 0) fmt = 2;
    else { err = std::string("unrecognized profile format '") + format + "' (valid: zTuvdp, zuvwTdp, zcuvd)"; return IGA_E_INVALID; }

    FILE* fp = fopen(path, "rb");
    if (!fp) { err = std::string("cannot open profile '") + path + "'"; return IGA_E_IO; }
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, got);
    fclose(fp);

    // Line accounting of file_length (fileIO.cpp:18-35): every getline()
    // result not starting with '#' counts, including the empty one after a
    // final newline, and the row count is that number minus one.
    std::vector<std::string> lines;
    size_t pos = 0;
    while (true) {
        size_t e = text.find('\n', pos);
        if (e == std::string::npos) { lines.push_back(text.substr(pos)); break; }
        lines.push_back(text.substr(pos, e - pos));
        pos = e + 1;
    }
    int count = 0;
    for (auto& l : lines) if (l.rfind("#", 0) != 0) count++;
    const int n_rows = count - 1;
    if (n_rows < 3) { err = std::string("profile '") + path + "' has fewer than 3 data rows"; return IGA_E_IO; }

    out = StratProfile();
    const int ncol = (fmt == 0) ? 6 : (fmt == 1) ? 7 : 5;
    int row = 0;
    for (size_t li = 0; li < lines.size() && row < n_rows; li++) {
        const std::string& l = lines[li];
        if (l.rfind("#", 0) == 0) continue;
        double v[7];
        const char* s = l.c_str();
        for (int cidx = 0; cidx < ncol; cidx++) {
            char* end;
            errno = 0;
            v[cidx] = strtod(s, &end);
            if (end == s) {
                err = std::string("profile '") + path + "' line " + std::to_string(li + 1) + ": expected " +
                      std::to_string(ncol) + " numeric columns";
                return IGA_E_IO;
            }
            s = end;
        }
        double z, c, u, vv, rho;
        if (fmt == 0) { z = v[0]; u = v[2]; vv = v[3]; rho = v[4]; c = std::sqrt(0.1 * kGamma * v[5] / rho) / 1000.0; }
        else if (fmt == 1) { z = v[0]; u = v[1]; vv = v[2]; rho = v[5]; c = std::sqrt(0.1 * kGamma * v[6] / rho) / 1000.0; }
        else { z = v[0]; c = v[1] / 1000.0; u = v[2]; vv = v[3]; rho = v[4]; }
        if (reverse_winds) { u /= -1000.0; vv /= -1000.0; }
        else { u /= 1000.0; vv /= 1000.0; }
        out.z.push_back(z); out.c.push_back(c); out.u.push_back(u); out.v.push_back(vv); out.rho.push_back(rho);
        row++;
    }
    // a file whose values fail the checks is a malformed file
    const int rc = finalize_profile(out, err);
    return rc == IGA_E_INVALID ? IGA_E_IO : rc;
}

}  // namespace iga
