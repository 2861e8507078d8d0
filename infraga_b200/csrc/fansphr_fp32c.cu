// FP32-compensated ray-fan kernel: spherical (global) geometry,
// range-dependent atmosphere (hybrid 3D splines), flat ground or terrain.
//
// Same equations, RK4 driver, stop checks, terrain reflection and bounce
// logic as fansphr_fp64_kernel (geoac.eqset.sph.rngdep.cpp, rk4solver.cpp,
// run_prop of main.infraga.sph.rngdep.cpp), with the arithmetic split as in
// the 3D stratified FP32C kernel (fan3d_fp32c.cu):
//
//   * the six ray equations (r, lat, lon, nu_r, nu_lat, nu_lon) in FP64, from
//     the FP64 value/slope blocks of the node records (c, u, v and their
//     gradients: the hyb_f1 part of the hybrid evaluation), the boundary-layer
//     scaling over the terrain in FP64;
//   * the twelve Jacobian auxiliaries (R_th, mu_th, R_ph, mu_ph) in FP32, their
//     state summed with TwoSum; the Hessians of c, u, v they read are formed
//     partly in FP32 from an FP32 copy of the records' second-derivative
//     blocks (hyb_x32: half the bytes of the largest part of a record read),
//     the entries formed from the value blocks in FP64;
//   * travel time, Sutherland-Bass absorption, reflection and amplitude in
//     FP64, at the same points as the FP64 kernel;
//   * focusing escalation as in the 3D kernel: a ray reaching an arrival with
//     |D| < kFocusRatioS * max|D| before its first caustic is marked and traced
//     again from launch with FP64 auxiliaries by fansphr_fp32c_retrace_kernel.
//
// FP64-only forms (sampled paths, the stratified-over-terrain ST variant,
// eigenray traces) stay on fansphr_fp64.cu.
#include "fansphr_common.cuh"

namespace iga {

namespace {

#ifndef IGA_SPHRC_THREADS
#define IGA_SPHRC_THREADS 128
#endif
constexpr int kThreadsS = IGA_SPHRC_THREADS;
constexpr int kThreadsSR = 64;       // re-trace kernel
constexpr double kFocusRatioS = 0.2;

template <bool AMP> struct AuxS { static constexpr int n = AMP ? 12 : 1; };

template <class T>
__device__ __forceinline__ void acc_pair_s(T& hi, T& lo, T inc) {   // Knuth's TwoSum
    const T s = hi + inc;
    const T bb = s - hi;
    const T e = (hi - (s - bb)) + (inc - bb);
    const T l = lo + e;
    hi = s + l;
    lo = l - (hi - s);
}

// Atmosphere at a stage: values and gradients in FP64, Hessians in T.
template <class T>
struct AtmC {
    double c, dc[3], u, du[3], v, dv[3];
    T ddc[3][3], ddu[3][3], ddv[3][3];
};

__device__ __forceinline__ float herm_val_f(float v0, float s0, float v1, float s1, float X, float h) {
    const float df = v1 - v0, A = s0 * h - df, B = -s1 * h + df;
    return v0 + X * (df + (1.0f - X) * (A * (1.0f - X) + B * X));
}

// Horizontal Hermite bases of a cell (value and d/dx, d/dy forms), in FP64
// and FP32, formed once per evaluation point for the three fields.
struct CellBasis {
    double hx[2], gx[2], hy[2], gy[2], dhx[2], dgx[2], dhy[2], dgy[2];
    float fhx[2], fgx[2], fhy[2], fgy[2], fdhx[2], fdhy[2];
};

__device__ __forceinline__ CellBasis cell_basis(const HybLoc& L) {
    const Basis1 bx = basis_val(L.tx), by = basis_val(L.ty);
    const Basis1 dbx = basis_der(L.tx, 1.0 / L.dx), dby = basis_der(L.ty, 1.0 / L.dy);
    CellBasis c;
    c.hx[0] = bx.h0; c.hx[1] = bx.h1; c.gx[0] = bx.g0; c.gx[1] = bx.g1;
    c.hy[0] = by.h0; c.hy[1] = by.h1; c.gy[0] = by.g0; c.gy[1] = by.g1;
    c.dhx[0] = dbx.h0; c.dhx[1] = dbx.h1; c.dgx[0] = dbx.g0; c.dgx[1] = dbx.g1;
    c.dhy[0] = dby.h0; c.dhy[1] = dby.h1; c.dgy[0] = dby.g0; c.dgy[1] = dby.g1;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        c.fhx[k] = (float)c.hx[k]; c.fgx[k] = (float)c.gx[k]; c.fhy[k] = (float)c.hy[k]; c.fgy[k] = (float)c.gy[k];
        c.fdhx[k] = (float)c.dhx[k]; c.fdhy[k] = (float)c.dhy[k];
    }
    return c;
}

// Field fld (0 c, 1 u, 2 v) at L (interp::eval_all, interpolation.cpp:
// 1544-1788, as hyb_f2): f, the gradient and the Hessian entries formed from
// the FP64 value blocks (d2/dz2, d2/dz dlat, d2/dz dlon, d2/dlat dlon) in
// FP64, the two formed from the second-derivative blocks (d2/dlat2,
// d2/dlon2) in FP32 from their FP32 copies (hyb_x32).  The patches are summed
// corner by corner as the corner data are formed, so no corner array is held.
__device__ __forceinline__ void hyb_f2_c(const HybView& g, const float* __restrict__ x32, const HybLoc& L,
                                         const CellBasis& B, int fld, HybF1& o, float (&dd)[3][3]) {
    const float Xf = (float)L.zq.X, hf = (float)L.zq.h;
    const double dxdy = L.dx * L.dy;
    const float dxf = (float)L.dx, dyf = (float)L.dy, dxdyf = (float)dxdy;
    double f = 0.0, d0 = 0.0, d1 = 0.0, d2 = 0.0, h00 = 0.0, h01 = 0.0, h02 = 0.0, h12 = 0.0;
    float h11 = 0.0f, h22 = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int a = q & 1, b = q >> 1;
        const int ix = L.kx + a, iy = L.ky + b;
        const size_t rec = (size_t)(ix * g.ny + iy) * g.nz + L.kz;
        const double* p0 = g.tab + rec * kRecLen + fld * kRecP;
        const double* p1 = p0 + kRecLen;
        const float* x0 = x32 + rec * kHybX32 + fld * kRecX;
        const float* x1 = x0 + kHybX32;
        double cv[4], cz[4], czz[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            cv[m] = herm_val(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq);
            cz[m] = herm_der(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq);
            czz[m] = herm_der2(p0[2 * m], p0[2 * m + 1], p1[2 * m], p1[2 * m + 1], L.zq_raw);
        }
        const float cv3f = (float)cv[3];
        const float q0 = herm_val_f((float)p0[2], x0[0], (float)p1[2], x1[0], Xf, hf);
        const float q1 = herm_val_f(x0[1], x0[2], x1[1], x1[2], Xf, hf) * dxf;
        const float q2 = cv3f * dyf;
        const float q3 = herm_val_f(x0[3], x0[4], x1[3], x1[4], Xf, hf) * dxdyf;
        const float r0 = herm_val_f((float)p0[4], x0[0], (float)p1[4], x1[0], Xf, hf);
        const float r1 = cv3f * dxf;
        const float r2 = herm_val_f(x0[5], x0[6], x1[5], x1[6], Xf, hf) * dyf;
        const float r3 = herm_val_f(x0[7], x0[8], x1[7], x1[8], Xf, hf) * dxdyf;
        cv[1] *= L.dx; cv[2] *= L.dy; cv[3] *= dxdy;
        cz[1] *= L.dx; cz[2] *= L.dy; cz[3] *= dxdy;
        czz[1] *= L.dx; czz[2] *= L.dy; czz[3] *= dxdy;
        const double hx = B.hx[a], gx = B.gx[a], hy = B.hy[b], gy = B.gy[b];
        const double dhx = B.dhx[a], dgx = B.dgx[a], dhy = B.dhy[b], dgy = B.dgy[b];
        f += cv[0] * hx * hy + cv[1] * gx * hy + cv[2] * hx * gy + cv[3] * gx * gy;
        d1 += cv[0] * dhx * hy + cv[1] * dgx * hy + cv[2] * dhx * gy + cv[3] * dgx * gy;
        d2 += cv[0] * hx * dhy + cv[1] * gx * dhy + cv[2] * hx * dgy + cv[3] * gx * dgy;
        d0 += cz[0] * hx * hy + cz[1] * gx * hy + cz[2] * hx * gy + cz[3] * gx * gy;
        h12 += cv[0] * dhx * dhy + cv[1] * dgx * dhy + cv[2] * dhx * dgy + cv[3] * dgx * dgy;
        h01 += cz[0] * dhx * hy + cz[1] * dgx * hy + cz[2] * dhx * gy + cz[3] * dgx * gy;
        h02 += cz[0] * hx * dhy + cz[1] * gx * dhy + cz[2] * hx * dgy + cz[3] * gx * dgy;
        h00 += czz[0] * hx * hy + czz[1] * gx * hy + czz[2] * hx * gy + czz[3] * gx * gy;
        const float fhx = B.fhx[a], fgx = B.fgx[a], fhy = B.fhy[b], fgy = B.fgy[b];
        const float fdhx = B.fdhx[a], fdhy = B.fdhy[b];
        const float fdgx = (float)dgx, fdgy = (float)dgy;
        h11 += q0 * fdhx * fhy + q1 * fdgx * fhy + q2 * fdhx * fgy + q3 * fdgx * fgy;
        h22 += r0 * fhx * fdhy + r1 * fgx * fdhy + r2 * fhx * fdgy + r3 * fgx * fdgy;
    }
    o.f = f; o.d[0] = d0; o.d[1] = d1; o.d[2] = d2;
    dd[0][0] = (float)h00;
    dd[0][1] = dd[1][0] = (float)h01;
    dd[0][2] = dd[2][0] = (float)h02;
    dd[1][1] = h11;
    dd[1][2] = dd[2][1] = (float)h12;
    dd[2][2] = h22;
}

// atm_full (fansphr_common.cuh) with the Hessians in T: for T = double the
// FP64 evaluation itself.
template <bool AMP, class T>
__device__ __forceinline__ void atm_full_c(const Fan3DArgs& a, const Views& vw, Cells& cl, double r, double lat,
                                           double lon, AtmC<T>& m) {
    if constexpr (sizeof(T) == sizeof(double) || !AMP) {
        AtmFull f;
        atm_full<AMP, false>(a, vw, cl, r, lat, lon, f);
        m.c = f.c; m.u = f.u; m.v = f.v;
#pragma unroll
        for (int n = 0; n < 3; n++) {
            m.dc[n] = f.dc[n]; m.du[n] = f.du[n]; m.dv[n] = f.dv[n];
            if (AMP) {
#pragma unroll
                for (int k = 0; k < 3; k++) { m.ddc[n][k] = (T)f.ddc[n][k]; m.ddu[n][k] = (T)f.ddu[n][k]; m.ddv[n][k] = (T)f.ddv[n][k]; }
            }
        }
    } else {
        HybLoc L;
        hyb_locate(vw.hyb, lat, lon, r - a.r_earth, L, cl.hx, cl.hy, cl.hz);
        HybF1 c1, u1, v1;
        float cdd[3][3], udd[3][3], vdd[3][3];
        const CellBasis B = cell_basis(L);
        hyb_f2_c(vw.hyb, a.hyb_x32, L, B, 0, c1, cdd);
        hyb_f2_c(vw.hyb, a.hyb_x32, L, B, 1, u1, udd);
        hyb_f2_c(vw.hyb, a.hyb_x32, L, B, 2, v1, vdd);
        // boundary-layer scaling over the terrain (or flat ground), as atm_full
        const double zr = r - a.r_earth;
        double zg = a.r_grnd, dzg[2] = {0.0, 0.0}, ddzg[3] = {0.0, 0.0, 0.0};
        double X = 0.0;
        if (zr < a.x_cut) {
            if (vw.has_topo) {
                TopoVal t;
                const bool in_bl = zr < a.z_bl;
                topo_eval(vw.topo, lat, lon, in_bl ? 2 : 0, t, cl.tx, cl.ty);
                zg = a.r_earth + t.z;
                if (in_bl) { dzg[0] = t.d[0]; dzg[1] = t.d[1]; ddzg[0] = t.dd[0]; ddzg[1] = t.dd[1]; ddzg[2] = t.dd[2]; }
            }
            X = exp(-(r - zg) * a.inv_bl);
        }
        const double ib = a.inv_bl, ib2 = ib * ib;
        const double dX[3] = {-X * ib, X * ib * dzg[0], X * ib * dzg[1]};
        const double iop = 1.0 / (1.0 + X), iop2 = iop * iop, iop3 = iop2 * iop;
        const double sc0 = (1.0 - X) * iop;
        double dsc[3];
#pragma unroll
        for (int n = 0; n < 3; n++) dsc[n] = -2.0 * dX[n] * iop2;
        m.c = c1.f; m.u = u1.f * sc0; m.v = v1.f * sc0;
#pragma unroll
        for (int n = 0; n < 3; n++) {
            m.dc[n] = c1.d[n];
            m.du[n] = u1.d[n] * sc0 + u1.f * dsc[n];
            m.dv[n] = v1.d[n] * sc0 + v1.f * dsc[n];
        }
        const float sc0f = (float)sc0;
        if (X == 0.0) {   // above the boundary layer: S = 1, S' = S'' = 0
#pragma unroll
            for (int n = 0; n < 3; n++) {
#pragma unroll
                for (int k = 0; k < 3; k++) { m.ddc[n][k] = cdd[n][k]; m.ddu[n][k] = udd[n][k]; m.ddv[n][k] = vdd[n][k]; }
            }
        } else {
            double ddX[3][3];
            ddX[0][0] = X * ib2;
            ddX[0][1] = ddX[1][0] = -X * ib2 * dzg[0];
            ddX[0][2] = ddX[2][0] = -X * ib2 * dzg[1];
            ddX[1][1] = (ddzg[0] + dzg[0] * dzg[0] * ib) * (X * ib);
            ddX[1][2] = ddX[2][1] = (ddzg[1] + dzg[0] * dzg[1] * ib) * (X * ib);
            ddX[2][2] = (ddzg[2] + dzg[1] * dzg[1] * ib) * (X * ib);
#pragma unroll
            for (int n = 0; n < 3; n++) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double dds = -2.0 * (ddX[n][k] * iop2 - 2.0 * dX[n] * dX[k] * iop3);
                    m.ddc[n][k] = cdd[n][k];
                    m.ddu[n][k] = (T)(udd[n][k] * sc0f) + (T)(u1.d[n] * dsc[k] + u1.d[k] * dsc[n] + u1.f * dds);
                    m.ddv[n][k] = (T)(vdd[n][k] * sc0f) + (T)(v1.d[n] * dsc[k] + v1.d[k] * dsc[n] + v1.f * dds);
                }
            }
        }
    }
}

// rhs_sphr (fansphr_common.cuh: update_refs + eval_src_eq,
// geoac.eqset.sph.rngdep.cpp:238-437, w = 0) on the split state: ray part fd
// in FP64, auxiliaries fa (R_th, mu_th, R_ph, mu_ph) in T.
template <bool AMP, class T>
__device__ __forceinline__ void rhs_sphr_c(const Fan3DArgs& a, const Views& vw, Cells& cl, const double* yd, const T* ya,
                                           double* fd, T* fa) {
    AtmC<T> m;
    atm_full_c<AMP, T>(a, vw, cl, yd[0], yd[1], yd[2], m);
    const double r = yd[0];
    double st, ct;
    sincos(yd[1], &st, &ct);
    const double ir = 1.0 / r, ict = 1.0 / ct, tnt = st * ict;
    const double n0 = yd[3], n1 = yd[4], n2 = yd[5];
    const double num = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const double inum = 1.0 / num;
    const double cg0 = m.c * n0 * inum, cg1 = m.c * n1 * inum + m.v, cg2 = m.c * n2 * inum + m.u;
    const double cgm = sqrt(cg0 * cg0 + cg1 * cg1 + cg2 * cg2);
    const double icg = 1.0 / cgm;
    const double G[3] = {1.0, ir, ir * ict};
    const double Tg[3] = {-ir * (n1 * cg1 + n2 * cg2), n0 * m.v + n0 * cg1 + n2 * cg2 * tnt,
                          n0 * m.u * ct + (n1 * m.u - n2 * m.v) * st + cg2 * (n0 * ct - n1 * st)};
    const double cg[3] = {cg0, cg1, cg2};
    double K[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        K[i] = num * m.dc[i] + n1 * m.dv[i] + n2 * m.du[i];
        fd[i] = G[i] * cg[i] * icg;
        fd[3 + i] = -G[i] * icg * (K[i] + Tg[i]);
    }
    if (AMP) {
        const T icgT = (T)icg, icg2 = icgT * icgT, irT = (T)ir, ir2 = irT * irT, ictT = (T)ict;
        const T stT = (T)st, ctT = (T)ct, tntT = (T)tnt;
        const T n0T = (T)n0, n1T = (T)n1, n2T = (T)n2, numT = (T)num, inumT = (T)inum;
        const T cin = (T)(m.c * inum), cin2 = cin * inumT;
        const T mu_ = (T)m.u, mv_ = (T)m.v;
        const T cgT[3] = {(T)cg0, (T)cg1, (T)cg2};
        const T GT[3] = {T(1), irT, irT * ictT};
        T dcT[3], duT[3], dvT[3], KT[3], TgT[3];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            dcT[i] = (T)m.dc[i]; duT[i] = (T)m.du[i]; dvT[i] = (T)m.dv[i];
            KT[i] = (T)K[i]; TgT[i] = (T)Tg[i];
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const T* R = ya + 6 * j;
            const T* mu = ya + 3 + 6 * j;
            const T dc = R[0] * dcT[0] + R[1] * dcT[1] + R[2] * dcT[2];
            const T du = R[0] * duT[0] + R[1] * duT[1] + R[2] * duT[2];
            const T dv = R[0] * dvT[0] + R[1] * dvT[1] + R[2] * dvT[2];
            const T dnu = (n0T * mu[0] + n1T * mu[1] + n2T * mu[2]) * inumT;
            const T g0 = n0T * inumT * dc + cin * mu[0] - cin2 * n0T * dnu;
            const T g1 = n1T * inumT * dc + cin * mu[1] - cin2 * n1T * dnu + dv;
            const T g2 = n2T * inumT * dc + cin * mu[2] - cin2 * n2T * dnu + du;
            const T gg[3] = {g0, g1, g2};
            const T dm = (cgT[0] * g0 + cgT[1] * g1 + cgT[2] * g2) * icgT;
            const T dG[3] = {T(0), -R[0] * ir2, -R[0] * ir2 * ictT + stT * irT * ictT * ictT * R[1]};
            const T dT[3] = {
                R[0] * ir2 * (n1T * cgT[1] + n2T * cgT[2]) - irT * (mu[1] * cgT[1] + n1T * g1 + mu[2] * cgT[2] + n2T * g2),
                (mu[0] * mv_ + n0T * dv) + mu[0] * cgT[1] + n0T * g1 + (mu[2] * cgT[2] + n2T * g2) * tntT +
                    n2T * cgT[2] * R[1] * ictT * ictT,
                (mu[0] * mu_ + n0T * du) * ctT - (n0T * mu_) * R[1] * stT +
                    (mu[1] * mu_ + n1T * du - mu[2] * mv_ - n2T * dv) * stT + (n1T * mu_ - n2T * mv_) * R[1] * ctT +
                    g2 * (n0T * ctT - n1T * stT) + cgT[2] * ((mu[0] - n1T * R[1]) * ctT - (mu[1] + n0T * R[1]) * stT)};
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const T ddc = R[0] * m.ddc[i][0] + R[1] * m.ddc[i][1] + R[2] * m.ddc[i][2];
                const T ddu = R[0] * m.ddu[i][0] + R[1] * m.ddu[i][1] + R[2] * m.ddu[i][2];
                const T ddv = R[0] * m.ddv[i][0] + R[1] * m.ddv[i][1] + R[2] * m.ddv[i][2];
                fa[6 * j + i] = dG[i] * cgT[i] * icgT + GT[i] * gg[i] * icgT - GT[i] * cgT[i] * icg2 * dm;
                fa[3 + 6 * j + i] = -dG[i] * icgT * (KT[i] + TgT[i]) + GT[i] * icg2 * dm * KT[i] -
                                    GT[i] * icgT * (dnu * dcT[i] + numT * ddc + mu[1] * dvT[i] + mu[2] * duT[i] +
                                                    n1T * ddv + n2T * ddu + dT[i]);
            }
        }
    }
}

// One RK4 step (rk4solver.cpp:30-55): increments incd (FP64), inca (T), and
// the stage-1 direction f1 for the caustic test.
template <bool AMP, class T>
__device__ __forceinline__ void rk4_sphr_c(const Fan3DArgs& a, const Views& vw, Cells& cl, double ds, const double* yd,
                                           const T* ya, double* incd, T* inca, double* f1) {
    constexpr int NA = AuxS<AMP>::n;
    const T dsf = (T)ds, sixth = T(1) / T(6), third = T(1) / T(3), half = T(0.5);
    double stgd[6], fd[6];
    T stga[NA], fa[NA];
    rhs_sphr_c<AMP>(a, vw, cl, yd, ya, fd, fa);
#pragma unroll
    for (int i = 0; i < 3; i++) f1[i] = fd[i];
#pragma unroll
    for (int i = 0; i < 6; i++) { const double t = ds * fd[i]; incd[i] = t * (1.0 / 6.0); stgd[i] = yd[i] + t * 0.5; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] = t * sixth; stga[i] = ya[i] + t * half; }
    }
    rhs_sphr_c<AMP>(a, vw, cl, stgd, stga, fd, fa);
#pragma unroll
    for (int i = 0; i < 6; i++) { const double t = ds * fd[i]; incd[i] += t * (1.0 / 3.0); stgd[i] = yd[i] + t * 0.5; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] += t * third; stga[i] = ya[i] + t * half; }
    }
    rhs_sphr_c<AMP>(a, vw, cl, stgd, stga, fd, fa);
#pragma unroll
    for (int i = 0; i < 6; i++) { const double t = ds * fd[i]; incd[i] += t * (1.0 / 3.0); stgd[i] = yd[i] + t; }
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) { const T t = dsf * fa[i]; inca[i] += t * third; stga[i] = ya[i] + t; }
    }
    rhs_sphr_c<AMP>(a, vw, cl, stgd, stga, fd, fa);
#pragma unroll
    for (int i = 0; i < 6; i++) incd[i] += (ds * fd[i]) * (1.0 / 6.0);
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) inca[i] += (dsf * fa[i]) * sixth;
    }
}

// One ray of the fan with the auxiliaries in T (the loop of
// fansphr_fp64_kernel without sampled paths).  Shared memory per lane: the
// ray part of row k-2 (prow, FP64) and the auxiliaries' last step (dprevf,
// FP32: it enters only the intercept extrapolation).  Returns true, with
// nothing of the ray's record final, when T is FP32 and the ray reaches a
// focusing arrival before its first caustic.
template <bool AMP, class T>
__device__ __forceinline__ bool fan_ray_sc(const Fan3DArgs& a, const Views& vw, double* prow, float* dprevf, int ray) {
    constexpr int NA = AuxS<AMP>::n;
    constexpr int N = DimSph<AMP>::n;
    constexpr bool ESCALATE = AMP && sizeof(T) == sizeof(float);
    const int nb = a.bounces + 1;
    const double theta0 = a.theta_deg[ray] * (kPi / 180.0);
    const double phi0 = kPi / 2.0 - a.phi_deg[ray] * (kPi / 180.0);
    double yd[6];
    T ya[NA], yl[NA];
    {
        double y[N];
        ray_init_sph<AMP>(a, theta0, phi0, y);
#pragma unroll
        for (int i = 0; i < 6; i++) yd[i] = y[i];
        if (AMP) {
#pragma unroll
            for (int i = 0; i < NA; i++) { ya[i] = (T)y[6 + i]; yl[i] = (T)(y[6 + i] - (double)ya[i]); }
        }
    }
    Cells cl{0, 0, 0, 0, 0};
    int bnc = 0, kb = 0, na = 0, caustics = 0;
    bool focused = false;
    T D_prev = T(0), D_max = T(0);
    long long steps = 0;
    double s = 0.0, tt = 0.0, att = 0.0, pt = 0.0, pa = 0.0, rmax = 0.0;
#pragma unroll
    for (int i = 0; i < 6; i++) prow[i * blockDim.x] = yd[i];
    if (AMP) {
#pragma unroll
        for (int i = 0; i < NA; i++) dprevf[i * blockDim.x] = 0.0f;
    }

    while (true) {
        rmax = fmax(rmax, yd[0] - a.r_earth);
        double ds = a.ds_max;   // set_ds (geoac.eqset.sph.rngdep.cpp:227-233)
        if (yd[0] - a.r_earth < a.z_bl)
            ds -= (a.ds_max - a.ds_min) * exp(-(yd[0] - topo_r(a, vw, cl, yd[1], yd[2])) / 0.2);
        s += ds;
        double incd[6], f1[3];
        T inca[NA];
        rk4_sphr_c<AMP>(a, vw, cl, ds, yd, ya, incd, inca, f1);
        if (AMP && (a.aux || ESCALATE) && kb >= 1) {   // caustics between rows 1..k-1 of the bounce
            const T f0 = (T)f1[0], g1 = (T)f1[1], g2 = (T)f1[2];
            const T* Rt = ya;
            const T* Rp = ya + 6;
            const T D = f0 * (Rt[1] * Rp[2] - Rp[1] * Rt[2]) - Rt[0] * (g1 * Rp[2] - g2 * Rp[1]) +
                        Rp[0] * (g1 * Rt[2] - g2 * Rt[1]);
            if (kb >= 2 && D * D_prev < T(0)) caustics++;
            D_prev = D;
            if (ESCALATE) D_max = fmax(D_max, fabs(D));
        }
        kb++;
        double nd[6];
#pragma unroll
        for (int i = 0; i < 6; i++) nd[i] = yd[i] + incd[i];

        bool esc = s > a.s_max;
        if (!esc) {
            if (nd[2] > kPi) nd[2] -= 2.0 * kPi;
            else if (nd[2] < -kPi) nd[2] += 2.0 * kPi;
            esc = (nd[1] < -kPi / 2.0 || nd[1] > kPi / 2.0) || (nd[0] - a.r_earth > a.alt_max) ||
                  beyond_range(a, nd[1], nd[2]) || (nd[1] < a.lat_min || nd[1] > a.lat_max) ||
                  (nd[2] < a.lon_min || nd[2] > a.lon_max);
        }
        // ground_check (geoac.eqset.sph.rngdep.cpp:496-503)
        const bool gnd = !esc && (nd[0] - a.r_earth <= a.topo_zmax) && (nd[0] < topo_r(a, vw, cl, nd[1], nd[2]));

        double dt, da;
        seg_increment_sphr<false>(a, vw, cl, yd, nd, dt, da);
        if (a.write_rays) { tt += pt; att += pa; pt = dt; pa = da; }
        else { pt += dt; pa += da; }

        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(nd[0]) || !isfinite(nd[1]) || !isfinite(nd[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < 6; i++) { prow[i * blockDim.x] = yd[i]; yd[i] = nd[i]; }
            if (AMP) {
#pragma unroll
                for (int i = 0; i < NA; i++) { dprevf[i * blockDim.x] = (float)inca[i]; acc_pair_s(ya[i], yl[i], inca[i]); }
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.sph.rngdep.cpp:499-541) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        int status = -1;
        if (a.topo_tab == nullptr && rmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        else if (tt / 3600.0 > a.time_max_h) status = 6;
        if (status < 0) {
            // the full 18-state rows k (below ground) and k-1
            double rk[N], r1[N];
#pragma unroll
            for (int i = 0; i < 6; i++) { rk[i] = nd[i]; r1[i] = yd[i]; }
            if (AMP) {
#pragma unroll
                for (int i = 0; i < NA; i++) {
                    r1[6 + i] = (double)ya[i] + (double)yl[i];
                    rk[6 + i] = r1[6 + i] + (double)inca[i];
                }
            }
            double jac = 0.0, amp = 0.0;
            if (AMP) {
                amp = amp_db_sphr<false>(a, vw, cl, rk, a.theta_deg[ray] * (kPi / 180.0),
                                         kPi / 2.0 - a.phi_deg[ray] * (kPi / 180.0), &jac);
                // jac = r^2 cos(lat) x the determinant D of the caustic test
                if (ESCALATE && !focused && caustics == 0 &&
                    fabs(jac) < kFocusRatioS * (double)D_max * rk[0] * rk[0] * cos(rk[1])) {
                    if (a.retrace) return true;
                    focused = true;
                }
            }
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            AtmPt mk;
            atm_point<false>(a, vw, cl, nd[0], nd[1], nd[2], mk);
            // the range-dependent run_prop records +asin(...) (main.infraga.sph.rngdep.cpp:514)
            const double incl = asin(mk.c / a.c0 * nd[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-nd[4], -nd[5]) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            out[0] = a.theta_deg[ray];
            out[1] = a.phi_deg[ray];
            out[2] = (double)bnc;
            out[3] = nd[1] * (180.0 / kPi);
            out[4] = nd[2] * (180.0 / kPi);
            out[5] = tt;
            out[6] = gc_dist(a.r_earth, nd[1], nd[2], a.src_x, a.src_y, a.cos_lat_src) / tt;
            out[7] = rmax;
            out[8] = incl;
            out[9] = baz;
            out[10] = amp;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux_sph(ax, a, rk, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            // row k-2: the ray part from shared memory, the auxiliaries one step back
            double p2[N];
#pragma unroll
            for (int i = 0; i < 6; i++) p2[i] = prow[i * blockDim.x];
            if (AMP) {
#pragma unroll
                for (int i = 0; i < NA; i++) p2[6 + i] = r1[6 + i] - (double)dprevf[i * blockDim.x];
            }
            reflect_sphr<N, AMP, false>(a, vw, cl, r1, p2, 1);
#pragma unroll
            for (int i = 0; i < 6; i++) yd[i] = r1[i];
            if (AMP) {
#pragma unroll
                for (int i = 0; i < NA; i++) { ya[i] = (T)r1[6 + i]; yl[i] = (T)(r1[6 + i] - (double)ya[i]); }
            }
            bnc++;
            if (bnc > a.bounces) status = 0;
        }
        if (status < 0) {
            s = 0.0; kb = 0;
#pragma unroll
            for (int i = 0; i < 6; i++) prow[i * blockDim.x] = yd[i];
            continue;
        }
        a.n_arr[ray] = na;
        a.ray_steps[ray] = steps;
        if (a.ray_status)
            a.ray_status[ray] = status | (sizeof(T) == sizeof(double) && AMP ? kRayAuxFp64 : 0) | (focused ? kRayFocus : 0);
        return false;
    }
}

struct LaneSmem {
    Views vw;
    double* prow;
    float* dprevf;
};

// Node coordinates in shared memory, then per lane [6] FP64 and [12] FP32.
__device__ __forceinline__ LaneSmem stage_sphr_c(const Fan3DArgs& a, double* s_mem) {
    double* s_hz = s_mem;
    double* s_hx = s_hz + a.hyb_nz;
    double* s_hy = s_hx + a.hyb_nx;
    double* s_tx = s_hy + a.hyb_ny;
    double* s_ty = s_tx + a.topo_nx;
    double* s_lane = s_ty + a.topo_ny;
    for (int i = threadIdx.x; i < a.hyb_nz; i += blockDim.x) s_hz[i] = a.hyb_z[i];
    for (int i = threadIdx.x; i < a.hyb_nx; i += blockDim.x) s_hx[i] = a.hyb_x[i];
    for (int i = threadIdx.x; i < a.hyb_ny; i += blockDim.x) s_hy[i] = a.hyb_y[i];
    for (int i = threadIdx.x; i < a.topo_nx; i += blockDim.x) s_tx[i] = a.topo_x[i];
    for (int i = threadIdx.x; i < a.topo_ny; i += blockDim.x) s_ty[i] = a.topo_y[i];
    __syncthreads();
    LaneSmem l;
    l.vw.hyb = HybView{a.hyb_tab, s_hx, s_hy, s_hz, a.hyb_nx, a.hyb_ny, a.hyb_nz};
    l.vw.topo = TopoView{a.topo_tab, s_tx, s_ty, a.topo_nx, a.topo_ny};
    l.vw.has_topo = a.topo_tab != nullptr;
    l.prow = s_lane + threadIdx.x;
    l.dprevf = reinterpret_cast<float*>(s_lane + 6 * blockDim.x) + threadIdx.x;
    return l;
}

inline size_t smem_sphr_c(const Fan3DArgs& a, int threads) {
    // the per-lane block starts on an 8-byte boundary after the coordinates
    return (size_t)(a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) * sizeof(double) +
           (size_t)threads * (6 * sizeof(double) + 12 * sizeof(float));
}

template <bool AMP>
__global__ void __launch_bounds__(kThreadsS, 1) fansphr_fp32c_kernel(const __grid_constant__ Fan3DArgs a) {
    extern __shared__ double s_mem[];
    const LaneSmem l = stage_sphr_c(a, s_mem);
    for (int ray = (int)atomicAdd(a.queue, 1u); ray < a.n_rays; ray = (int)atomicAdd(a.queue, 1u))
        if (fan_ray_sc<AMP, float>(a, l.vw, l.prow, l.dprevf, ray)) a.n_arr[ray] = -1;
}

// The marked rays, traced from launch with FP64 auxiliaries: few, so one
// small CTA per SM scans the fan through the workspace's second counter.
__global__ void __launch_bounds__(kThreadsSR, 1)
    fansphr_fp32c_retrace_kernel(const __grid_constant__ Fan3DArgs a, unsigned int* __restrict__ queue) {
    extern __shared__ double s_mem[];
    const LaneSmem l = stage_sphr_c(a, s_mem);
    for (int ray = (int)atomicAdd(queue, 1u); ray < a.n_rays; ray = (int)atomicAdd(queue, 1u))
        if (a.n_arr[ray] < 0) fan_ray_sc<true, double>(a, l.vw, l.prow, l.dprevf, ray);
}

template <bool AMP>
cudaError_t launch_sc(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    const int threads = a.block > 0 ? a.block : kThreadsS;
    auto kern = fansphr_fp32c_kernel<AMP>;
    const size_t smem = smem_sphr_c(a, threads);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, n_sm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long want = ((long long)a.n_rays + threads - 1) / threads;
    long long grid = (long long)n_sm * per_sm;
    if (want < grid) grid = want;
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    if (grid < 1) grid = 1;
    if (grid_used) *grid_used = (int)grid;
    kern<<<(unsigned)grid, threads, smem, stream>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess || !AMP || !a.retrace) return e;
    auto rk = fansphr_fp32c_retrace_kernel;
    const size_t smem_r = smem_sphr_c(a, kThreadsSR);
    if ((e = cudaFuncSetAttribute(rk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r)) != cudaSuccess)
        return e;
    const long long grid_r = std::min<long long>(n_sm, ((long long)a.n_rays + kThreadsSR - 1) / kThreadsSR);
    rk<<<(unsigned)grid_r, kThreadsSR, smem_r, stream>>>(a, a.queue + 1);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fansphr_fp32c(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    if (a.hyb_tab == nullptr || (calc_amp && a.hyb_x32 == nullptr)) return cudaErrorInvalidValue;
    return calc_amp ? launch_sc<true>(a, stream, grid_used) : launch_sc<false>(a, stream, grid_used);
}

}  // namespace iga
