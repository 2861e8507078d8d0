// Evaluation of the range-dependent atmosphere and terrain tables
// (layouts in atmo_rngdep.h), shared by the host (per-launch constants) and
// the device kernels.
//
// Hybrid atmosphere at (lat, lon, z): the reference's bicubic patches
// (interp::eval_all, interpolation.cpp:1544-1788) over the cell's four corner
// nodes, with corner data from node splines in z.  Bicubic patch in Hermite
// form: with H0 = 1-3t^2+2t^3, H1 = 3t^2-2t^3, G0 = t-2t^2+t^3, G1 = t^3-t^2,
//   F = sum_corners V Hx Hy + (Vx dx) Gx Hy + (Vy dy) Hx Gy + (Vxy dx dy) Gx Gy,
// which is the reference's 16x16 bicubic_conversion_matrix product written
// out (interpolation.cpp:686-703).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace iga {

#ifndef IGA_HD
#define IGA_HD __host__ __device__ __forceinline__
#endif

// record layout (atmo_rngdep.h)
constexpr int kRecP = 8, kRecX = 9, kRecLen = 64, kRecXOff = 32;

struct Basis1 {   // cubic Hermite basis in one horizontal direction at t
    double h0, h1, g0, g1;
};

IGA_HD Basis1 basis_val(double t) {
    const double t2 = t * t, t3 = t2 * t;
    return {1.0 - 3.0 * t2 + 2.0 * t3, 3.0 * t2 - 2.0 * t3, t - 2.0 * t2 + t3, t3 - t2};
}
// d/dt of the basis divided by the cell width (a d/dx basis)
IGA_HD Basis1 basis_der(double t, double inv_w) {
    const double t2 = t * t;
    return {(6.0 * t2 - 6.0 * t) * inv_w, (6.0 * t - 6.0 * t2) * inv_w, (1.0 - 4.0 * t + 3.0 * t2) * inv_w,
            (3.0 * t2 - 2.0 * t) * inv_w};
}
IGA_HD Basis1 basis_der2(double t, double inv_w2) {
    return {(12.0 * t - 6.0) * inv_w2, (6.0 - 12.0 * t) * inv_w2, (6.0 * t - 4.0) * inv_w2, (6.0 * t - 2.0) * inv_w2};
}

// Bicubic patch value from corner data c[4][4] = {V, Vx*dx, Vy*dy, Vxy*dx*dy}
// per corner (0: (kx,ky), 1: (kx+1,ky), 2: (kx,ky+1), 3: (kx+1,ky+1)).
IGA_HD double patch(const double (&c)[4][4], const Basis1& bx, const Basis1& by) {
    const double hx[2] = {bx.h0, bx.h1}, gx[2] = {bx.g0, bx.g1};
    const double hy[2] = {by.h0, by.h1}, gy[2] = {by.g0, by.g1};
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int a = q & 1, b = q >> 1;
        s += c[q][0] * hx[a] * hy[b] + c[q][1] * gx[a] * hy[b] + c[q][2] * hx[a] * gy[b] + c[q][3] * gx[a] * gy[b];
    }
    return s;
}

// Cubic Hermite in z through (v0, s0) and (v1, s1) over a segment of width h
// (interp::eval_node_*, interpolation.cpp:1070-1182).
struct Herm {
    double X, h, ih;
};
IGA_HD double herm_val(double v0, double s0, double v1, double s1, const Herm& q) {
    const double df = v1 - v0, A = s0 * q.h - df, B = -s1 * q.h + df;
    return v0 + q.X * (df + (1.0 - q.X) * (A * (1.0 - q.X) + B * q.X));
}
IGA_HD double herm_der(double v0, double s0, double v1, double s1, const Herm& q) {
    const double df = v1 - v0, A = s0 * q.h - df, B = -s1 * q.h + df;
    return (df + (1.0 - 2.0 * q.X) * (A * (1.0 - q.X) + B * q.X) + q.X * (1.0 - q.X) * (B - A)) * q.ih;
}
IGA_HD double herm_der2(double v0, double s0, double v1, double s1, const Herm& q) {
    const double df = v1 - v0, A = s0 * q.h - df, B = -s1 * q.h + df;
    return 2.0 * (B - 2.0 * A + (A - B) * 3.0 * q.X) * (q.ih * q.ih);
}

// Segment index of x in the increasing array a[0..n) (x already clamped):
// a[k] <= x <= a[k+1], starting from the cached k.
IGA_HD int seg_find(const double* a, int n, double x, int k) {
    if (k < 0) k = 0;
    if (k > n - 2) k = n - 2;
    while (k > 0 && x < a[k]) --k;
    while (k < n - 2 && x > a[k + 1]) ++k;
    return k;
}

// Located point in the hybrid grid.
struct HybLoc {
    int kx, ky, kz;
    double tx, ty, dx, dy;
    Herm zq;      // vertical coordinate at the clamped z
    Herm zq_raw;  // at the unclamped z (the reference's d2f/dz2 block, interpolation.cpp:1762-1780)
};

struct HybView {
    const double* tab;   // nx*ny*nz*kRecLen
    const double* x;     // lat [rad]
    const double* y;     // lon [rad]
    const double* z;     // km
    int nx, ny, nz;
};

IGA_HD void hyb_locate(const HybView& g, double lat, double lon, double zr, HybLoc& L, int& cx, int& cy, int& cz) {
    const double xe = fmin(fmax(lat, g.x[0]), g.x[g.nx - 1]);
    const double ye = fmin(fmax(lon, g.y[0]), g.y[g.ny - 1]);
    const double ze = fmin(fmax(zr, g.z[0]), g.z[g.nz - 1]);
    cx = seg_find(g.x, g.nx, xe, cx);
    cy = seg_find(g.y, g.ny, ye, cy);
    cz = seg_find(g.z, g.nz, ze, cz);
    L.kx = cx; L.ky = cy; L.kz = cz;
    L.dx = g.x[cx + 1] - g.x[cx];
    L.dy = g.y[cy + 1] - g.y[cy];
    L.tx = (xe - g.x[cx]) / L.dx;
    L.ty = (ye - g.y[cy]) / L.dy;
    const double h = g.z[cz + 1] - g.z[cz];
    L.zq.h = h; L.zq.ih = 1.0 / h; L.zq.X = (ze - g.z[cz]) / h;
    L.zq_raw = L.zq; L.zq_raw.X = (zr - g.z[cz]) / h;
}

// Pointer to the record of corner q at knot kz.
IGA_HD const double* hyb_rec(const HybView& g, const HybLoc& L, int q) {
    const int ix = L.kx + (q & 1), iy = L.ky + (q >> 1);
    return g.tab + ((size_t)(ix * g.ny + iy) * g.nz + L.kz) * kRecLen;
}

// Field values and derivatives (index 0 = z, 1 = lat, 2 = lon, the
// reference's (r, theta, phi) order after its index rotation,
// atmo_state.sph.rngdep.cpp:136-141).
struct HybF1 {
    double f, d[3];
};
struct HybF2 {
    double f, d[3], dd[3][3];
};

// f only (for c/u/v/rho at segment midpoints and arrival rows)
IGA_HD double hyb_f(const HybView& g, const HybLoc& L, int fld) {
    double c4[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double* r0 = hyb_rec(g, L, q) + fld * kRecP;
        const double* r1 = r0 + kRecLen;
#pragma unroll
        for (int m = 0; m < 4; m++) c4[q][m] = herm_val(r0[2 * m], r0[2 * m + 1], r1[2 * m], r1[2 * m + 1], L.zq);
        c4[q][1] *= L.dx; c4[q][2] *= L.dy; c4[q][3] *= L.dx * L.dy;
    }
    return patch(c4, basis_val(L.tx), basis_val(L.ty));
}

// f and the gradient (interp::eval_all first form, interpolation.cpp:1544-1616)
IGA_HD void hyb_f1(const HybView& g, const HybLoc& L, int fld, HybF1& o) {
    double cv[4][4], cz[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double* r0 = hyb_rec(g, L, q) + fld * kRecP;
        const double* r1 = r0 + kRecLen;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            cv[q][m] = herm_val(r0[2 * m], r0[2 * m + 1], r1[2 * m], r1[2 * m + 1], L.zq);
            cz[q][m] = herm_der(r0[2 * m], r0[2 * m + 1], r1[2 * m], r1[2 * m + 1], L.zq);
        }
        cv[q][1] *= L.dx; cv[q][2] *= L.dy; cv[q][3] *= L.dx * L.dy;
        cz[q][1] *= L.dx; cz[q][2] *= L.dy; cz[q][3] *= L.dx * L.dy;
    }
    const Basis1 bx = basis_val(L.tx), by = basis_val(L.ty);
    o.f = patch(cv, bx, by);
    o.d[1] = patch(cv, basis_der(L.tx, 1.0 / L.dx), by);
    o.d[2] = patch(cv, bx, basis_der(L.ty, 1.0 / L.dy));
    o.d[0] = patch(cz, bx, by);
}

// f, gradient and Hessian (interp::eval_all second form,
// interpolation.cpp:1618-1788) for c/u/v (fld 0..2).
IGA_HD void hyb_f2(const HybView& g, const HybLoc& L, int fld, HybF2& o) {
    double cv[4][4], cz[4][4], czz[4][4], cq[4][4], cr[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double* r0 = hyb_rec(g, L, q);
        const double* r1 = r0 + kRecLen;
        const double* p0 = r0 + fld * kRecP;
        const double* p1 = r1 + fld * kRecP;
        const double* x0 = r0 + kRecXOff + fld * kRecX;
        const double* x1 = r1 + kRecXOff + fld * kRecX;
#pragma unroll
        for (int m = 0; m < 4; m++) {
            cv[q][m] = herm_val(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq);
            cz[q][m] = herm_der(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq);
            czz[q][m] = herm_der2(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq_raw);
        }
        // d2f/dx2 block: Q (FDx f values, D slopes), FDx Q, FDxy f, FDxy Q
        cq[q][0] = herm_val(p0[2], x0[0], p1[2], x1[0], L.zq);
        cq[q][1] = herm_val(x0[1], x0[2], x1[1], x1[2], L.zq);
        cq[q][2] = cv[q][3];
        cq[q][3] = herm_val(x0[3], x0[4], x1[3], x1[4], L.zq);
        // d2f/dy2 block: R (FDy f values, D slopes), FDxy f, FDy R, FDxy R
        cr[q][0] = herm_val(p0[4], x0[0], p1[4], x1[0], L.zq);
        cr[q][1] = cv[q][3];
        cr[q][2] = herm_val(x0[5], x0[6], x1[5], x1[6], L.zq);
        cr[q][3] = herm_val(x0[7], x0[8], x1[7], x1[8], L.zq);
        const double dxdy = L.dx * L.dy;
        cv[q][1] *= L.dx; cv[q][2] *= L.dy; cv[q][3] *= dxdy;
        cz[q][1] *= L.dx; cz[q][2] *= L.dy; cz[q][3] *= dxdy;
        czz[q][1] *= L.dx; czz[q][2] *= L.dy; czz[q][3] *= dxdy;
        cq[q][1] *= L.dx; cq[q][2] *= L.dy; cq[q][3] *= dxdy;
        cr[q][1] *= L.dx; cr[q][2] *= L.dy; cr[q][3] *= dxdy;
    }
    const Basis1 bx = basis_val(L.tx), by = basis_val(L.ty);
    const Basis1 dbx = basis_der(L.tx, 1.0 / L.dx), dby = basis_der(L.ty, 1.0 / L.dy);
    o.f = patch(cv, bx, by);
    o.d[1] = patch(cv, dbx, by);
    o.d[2] = patch(cv, bx, dby);
    o.d[0] = patch(cz, bx, by);
    o.dd[1][2] = o.dd[2][1] = patch(cv, dbx, dby);
    o.dd[0][1] = o.dd[1][0] = patch(cz, dbx, by);
    o.dd[0][2] = o.dd[2][0] = patch(cz, bx, dby);
    o.dd[0][0] = patch(czz, bx, by);
    o.dd[1][1] = patch(cq, dbx, by);
    o.dd[2][2] = patch(cr, bx, dby);
}

// ---- terrain: tensor-product natural bicubic ----
struct TopoView {
    const double* tab;   // nx*ny*4: f, f_x, f_y, f_xy
    const double* x;
    const double* y;
    int nx, ny;
};

struct TopoVal {
    double z, d[2], dd[3];   // height [km above r_earth], d/dlat, d/dlon, (xx, xy, yy)
};

// order: 0 height only, 1 + gradient, 2 + Hessian, at (lat, lon) clamped to
// the terrain grid like topo::z (atmo_state.sph.rngdep.cpp:47-56); rays stay
// inside it (break_check limits), where clamping changes nothing.
IGA_HD void topo_eval(const TopoView& t, double lat, double lon, int order, TopoVal& o, int& cx, int& cy) {
    const double xe = fmin(fmax(lat, t.x[0]), t.x[t.nx - 1]);
    const double ye = fmin(fmax(lon, t.y[0]), t.y[t.ny - 1]);
    cx = seg_find(t.x, t.nx, xe, cx);
    cy = seg_find(t.y, t.ny, ye, cy);
    const double dx = t.x[cx + 1] - t.x[cx], dy = t.y[cy + 1] - t.y[cy];
    const double tx = (xe - t.x[cx]) / dx, ty = (ye - t.y[cy]) / dy;
    double c4[4][4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double* r = t.tab + ((size_t)(cx + (q & 1)) * t.ny + (cy + (q >> 1))) * 4;
        c4[q][0] = r[0]; c4[q][1] = r[1] * dx; c4[q][2] = r[2] * dy; c4[q][3] = r[3] * dx * dy;
    }
    const Basis1 bx = basis_val(tx), by = basis_val(ty);
    o.z = patch(c4, bx, by);
    if (order >= 1) {
        const Basis1 dbx = basis_der(tx, 1.0 / dx), dby = basis_der(ty, 1.0 / dy);
        o.d[0] = patch(c4, dbx, by);
        o.d[1] = patch(c4, bx, dby);
        if (order >= 2) {
            o.dd[0] = patch(c4, basis_der2(tx, 1.0 / (dx * dx)), by);
            o.dd[1] = patch(c4, dbx, dby);
            o.dd[2] = patch(c4, bx, basis_der2(ty, 1.0 / (dy * dy)));
        }
    }
}

}  // namespace iga
