// geom.cuh -- FP64 geometry of the backprojection, on the device.
//
// Every function here rounds each operation exactly as an x86-64 build of
// the reference C/Fortran does: explicit __d*_rn intrinsics stop the compiler
// from contracting a*b+c into an FMA, and the operand order is the source
// order of the reference expression cited beside each function.  The only
// inexact-by-design steps are the CUDA sin/cos of the lat/lon angles (the
// reference CPU path uses glibc's; both are within an ulp or two).
#pragma once
#include "common.cuh"

namespace srg {

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Pixel ECEF on WGS-84 (sentinel/azimuth_compress.cu:117-131), split into
// the factors that depend on the line only and on the column only, so that a
// tile can evaluate each sine and cosine once; pixel_ecef composes them with
// the same operations in the same order.
struct LineTrig {
    double slat, clat, re, rez;  // sin, cos of the latitude; prime-vertical radius; re - re*e2
};
__device__ __forceinline__ LineTrig line_trig(const BurstDev &B, int line) {
    const double a = 6378137.0;
    const double e2 = 0.0066943799901499996;
    const double lat = dadd(B.firstlat, dmul((double)(line + B.firstline), B.deltalat));
    const double rlat = dmul(lat, B.deg2rad);
    LineTrig L;
    sincos(rlat, &L.slat, &L.clat);
    L.re = ddiv(a, __dsqrt_rn(dsub(1.0, dmul(dmul(e2, L.slat), L.slat))));
    L.rez = dsub(L.re, dmul(L.re, e2));
    return L;
}
__device__ __forceinline__ void col_trig(const BurstDev &B, int pix, double &slon, double &clon) {
    const double rlon = dmul(dadd(B.firstlon, dmul((double)pix, B.deltalon)), B.deg2rad);
    sincos(rlon, &slon, &clon);
}
__device__ __forceinline__ void pixel_ecef_from(double slat, double clat, double re, double rez,
                                                double slon, double clon, double hgt, double &x,
                                                double &y, double &z) {
    const double rh = dadd(re, hgt);
    x = dmul(dmul(rh, clat), clon);
    y = dmul(dmul(rh, clat), slon);
    z = dmul(dadd(rez, hgt), slat);
}
__device__ __forceinline__ void pixel_ecef(const BurstDev &B, int line, int pix, double hgt,
                                           double &x, double &y, double &z) {
    const LineTrig L = line_trig(B, line);
    double slon, clon;
    col_trig(B, pix, slon, clon);
    pixel_ecef_from(L.slat, L.clat, L.re, L.rez, slon, clon, hgt, x, y, z);
}

// azoff of one pixel from its line's parabola (azimuth_compress.cu:169-175),
// -1 when outside (ap/2, P - ap/2).
__device__ __forceinline__ double pixel_azoff(const BurstDev &B, const double *coef, int pix) {
    const float q = __fdiv_rn((float)(pix - B.firstpix), (float)(B.lastpix - B.firstpix));
    const double arg = dsub(dmul((double)q, 2.0), 1.0);
    const double fit = dadd(dadd(dmul(dmul(coef[0], arg), arg), dmul(coef[1], arg)), coef[2]);
    if (fit > (double)B.ap2 && fit < (double)(B.P - B.ap2)) return fit;
    return -1.0;
}

// Aperture window [azs, aze) of a pixel (azimuth_compress.cu:54-58); an
// unformed pixel gets the empty window [0, 0).
__device__ __forceinline__ void pixel_window(const BurstDev &B, double azoff, int &azs, int &aze) {
    if (azoff > 0.) {
        int a0 = (int)round(dsub(azoff, (double)B.ap2));
        int a1 = (int)round(dadd(azoff, (double)B.ap2));
        azs = max(a0, 0);
        aze = min(a1, B.P - 1);
    } else {
        azs = 0;
        aze = 0;
    }
}

// 4-point Hermite of position and velocity (sentinel/orbithermite.f:21-70).
__device__ inline void hermite4(const double *x, const double *v, const double *t, double tq,
                                double *xq, double *vq) {
    double h[4], hd[4], f0[4], f1[4], g0[4], g1[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f1[i] = dsub(tq, t[i]);
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j != i) s = dadd(s, ddiv(1.0, dsub(t[i], t[j])));
        f0[i] = dsub(1.0, dmul(dmul(2.0, dsub(tq, t[i])), s));
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double p = 1.0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k != i) p = ddiv(dmul(p, dsub(tq, t[k])), dsub(t[i], t[k]));
        h[i] = p;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double q = 1.0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k != i && k != j) q = ddiv(dmul(q, dsub(tq, t[k])), dsub(t[i], t[k]));
            if (j != i) s = dadd(s, dmul(ddiv(1.0, dsub(t[i], t[j])), q));
        }
        hd[i] = s;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        g1[i] = dadd(h[i], dmul(dmul(2.0, dsub(tq, t[i])), hd[i]));
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (i != j) s = dadd(s, ddiv(1.0, dsub(t[i], t[j])));
        g0[i] = dmul(2.0, dsub(dmul(f0[i], hd[i]), dmul(h[i], s)));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double sp = 0.0, sv = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            sp = dadd(sp, dmul(dmul(dadd(dmul(x[3 * i + c], f0[i]), dmul(v[3 * i + c], f1[i])), h[i]), h[i]));
#pragma unroll
        for (int i = 0; i < 4; ++i)
            sv = dadd(sv, dmul(dadd(dmul(x[3 * i + c], g0[i]), dmul(v[3 * i + c], g1[i])), h[i]));
        xq[c] = sp;
        vq[c] = sv;
    }
}

// Orbit state vectors for device-side interpolation.
struct Orbit {
    const double *t;   // [n]
    const double *x;   // [n][3]
    const double *v;   // [n][3]
    int n;
};

// Clamped-window interpolation (sentinel/intp_orbit.f90:1-25).
__device__ inline void intp_orbit(const Orbit &o, double tq, double *xq, double *vq) {
    int loc = (int)ddiv(dsub(tq, o.t[0]), dsub(o.t[1], o.t[0]));
    if (loc < 2) loc = 2;
    if (loc > o.n - 2) loc = o.n - 2;
    const int s = loc - 2;
    hermite4(o.x + 3 * s, o.v + 3 * s, o.t + s, tq, xq, vq);
}

__device__ __forceinline__ double dot3x(const double *a, const double *b) {
    return dadd(dadd(dmul(a[0], b[0]), dmul(a[1], b[1])), dmul(a[2], b[2]));
}

// Newton zero-Doppler solve (sentinel/orbitrangetime.f90:22-69).  Returns
// the range at the converged time.
__device__ inline double zero_doppler_range(const Orbit &o, const double *xyz, double t0,
                                            const double *sx0, const double *sv0) {
    double sx[3] = {sx0[0], sx0[1], sx0[2]};
    double sv[3] = {sv0[0], sv0[1], sv0[2]};
    double dr[3];
    double t = t0;
    for (int it = 1; it <= 51; ++it) {
        const double tprev = t;
        dr[0] = dsub(xyz[0], sx[0]);
        dr[1] = dsub(xyz[1], sx[1]);
        dr[2] = dsub(xyz[2], sx[2]);
        const double fn = dot3x(dr, sv);
        const double c1 = -dot3x(sv, sv);
        const double fnprime = dadd(c1, dmul(0.0, fn));
        t = dsub(t, ddiv(fn, fnprime));
        intp_orbit(o, t, sx, sv);
        if (fabs(dsub(t, tprev)) < 5.0e-9) break;
    }
    dr[0] = dsub(xyz[0], sx[0]);
    dr[1] = dsub(xyz[1], sx[1]);
    dr[2] = dsub(xyz[2], sx[2]);
    return __dsqrt_rn(dot3x(dr, dr));
}

}  // namespace srg
