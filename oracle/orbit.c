/*
 * oracle/orbit.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of SRG's orbit helpers, used as the checker for the CUDA
 * path and as the `orbitrangetime_` symbol that the compiled reference CPU
 * backprojection (sentinel/azimuth_compress_cpu.c) needs at link time.
 * Nothing in the shipped library links or calls this file.
 *
 * Restated routines (Fortran originals; gfortran is not available, so these
 * cannot be compiled and compared directly -- parity for them is pinned
 * indirectly, through the compiled reference backprojection that calls
 * orbitrangetime_, and against the analytic orbit the scenes are made from):
 *
 *   orbithermite_   sentinel/orbithermite.f:3-85   4-point Hermite (value +
 *                   derivative) interpolation of position and velocity.
 *   intp_orbit_     sentinel/intp_orbit.f90:1-25   window selection: index
 *                   truncated toward zero, clamped to [2, n-2] (1-based), then
 *                   Hermite over the four vectors that start one before it.
 *   orbitrangetime_ sentinel/orbitrangetime.f90:1-73  Newton zero-Doppler
 *                   solve, at most 51 iterations, stop when |dt| < 5e-9 s.
 *
 * Every expression keeps the left-to-right evaluation order of the Fortran
 * source, and the file is compiled without FMA contraction
 * (-ffp-contract=off), so the results are those of an x86-64 gfortran -O0
 * build of the originals.
 *
 * Array conventions follow the Fortran callers: positions and velocities are
 * stored [n][3] (Fortran xx(3,n), column-major), times [n].
 */
#include <math.h>
#include "srg_oracle.h"

/* orbithermite.f:3-85.  x, v: [4][3]; t: [4]; tq: query time. */
void orbithermite_(const double *x, const double *v, const double *t,
                   const double *tq, double *xq, double *vq)
{
    enum { N = 4 };
    const double tt = *tq;
    double h[N], hd[N], f0[N], f1[N], g0[N], g1[N];

    /* orbithermite.f:23-30 */
    for (int i = 0; i < N; ++i) {
        f1[i] = tt - t[i];
        double s = 0.0;
        for (int j = 0; j < N; ++j)
            if (j != i) s = s + 1.0 / (t[i] - t[j]);
        f0[i] = 1.0 - 2.0 * (tt - t[i]) * s;
    }
    /* orbithermite.f:32-47: Lagrange basis h and its derivative hd */
    for (int i = 0; i < N; ++i) {
        double p = 1.0;
        for (int k = 0; k < N; ++k)
            if (k != i) p = p * (tt - t[k]) / (t[i] - t[k]);
        h[i] = p;
        double s = 0.0;
        for (int j = 0; j < N; ++j) {
            double q = 1.0;
            for (int k = 0; k < N; ++k)
                if (k != i && k != j) q = q * (tt - t[k]) / (t[i] - t[k]);
            if (j != i) s = s + 1.0 / (t[i] - t[j]) * q;
        }
        hd[i] = s;
    }
    /* orbithermite.f:49-56 */
    for (int i = 0; i < N; ++i) {
        g1[i] = h[i] + 2.0 * (tt - t[i]) * hd[i];
        double s = 0.0;
        for (int j = 0; j < N; ++j)
            if (i != j) s = s + 1.0 / (t[i] - t[j]);
        g0[i] = 2.0 * (f0[i] * hd[i] - h[i] * s);
    }
    /* orbithermite.f:58-70 */
    for (int c = 0; c < 3; ++c) {
        double sp = 0.0, sv = 0.0;
        for (int i = 0; i < N; ++i)
            sp = sp + (x[3 * i + c] * f0[i] + v[3 * i + c] * f1[i]) * h[i] * h[i];
        for (int i = 0; i < N; ++i)
            sv = sv + (x[3 * i + c] * g0[i] + v[3 * i + c] * g1[i]) * h[i];
        xq[c] = sp;
        vq[c] = sv;
    }
}

/* intp_orbit.f90:1-25.  Returns 0 always (as the original does). */
int intp_orbit_(const double *timeorbit, const double *xx, const double *vv,
                const int *numstatevec, const double *time, double *xyz,
                double *vel)
{
    /* Fortran integer assignment from real*8 truncates toward zero. */
    int loc = (int)((*time - timeorbit[0]) / (timeorbit[1] - timeorbit[0]));
    if (loc < 2) loc = 2;
    if (loc > *numstatevec - 2) loc = *numstatevec - 2;
    /* xx(1, loc-1) in 1-based Fortran is element (loc-2) 0-based. */
    const int s = loc - 2;
    orbithermite_(xx + 3 * s, vv + 3 * s, timeorbit + s, time, xyz, vel);
    return 0;
}

static double dot3(const double *a, const double *b)
{
    /* gfortran dot_product: accumulate from zero, in index order. */
    double s = 0.0;
    s = s + a[0] * b[0];
    s = s + a[1] * b[1];
    s = s + a[2] * b[2];
    return s;
}

/* orbitrangetime.f90:1-73.  satx0/satv0 are inputs only (copied), exactly as
 * in the original: the caller's arrays are not updated. */
void orbitrangetime_(const double *xyz, const double *timeorbit, const double *xx,
                     const double *vv, const int *numstatevec, const double *tline0,
                     const double *satx0, const double *satv0, double *tline,
                     double *range)
{
    double sx[3] = {satx0[0], satx0[1], satx0[2]};
    double sv[3] = {satv0[0], satv0[1], satv0[2]};
    double dr[3];
    double t = *tline0;

    for (int it = 1; it <= 51; ++it) {
        const double tprev = t;
        dr[0] = xyz[0] - sx[0];
        dr[1] = xyz[1] - sx[1];
        dr[2] = xyz[2] - sx[2];
        const double fn = dot3(dr, sv);          /* dopfact */
        const double c1 = -dot3(sv, sv);
        const double c2 = 0.0;
        const double fnprime = c1 + c2 * fn;
        t = t - fn / fnprime;
        (void)intp_orbit_(timeorbit, xx, vv, numstatevec, &t, sx, sv);
        if (fabs(t - tprev) < 5.0e-9) break;
    }
    dr[0] = xyz[0] - sx[0];
    dr[1] = xyz[1] - sx[1];
    dr[2] = xyz[2] - sx[2];
    *tline = t;
    *range = sqrt(dot3(dr, dr));
}

/* Per-pulse satellite position and velocity, sentinel/sentineltimingsub.f90:
 * timedelta = timeorbit(2) - timeorbit(1) (:41); for each line time,
 * ilocation = (time - timeorbit(1)) / timedelta assigned to an integer
 * (truncation toward zero, :61), then orbithermite over the four vectors that
 * start at 1-based ilocation - 1 (:62), with no clamp.  pos, vel: [P][3].
 * Where the window would leave the vector array (the reference reads outside
 * it there) the pulse is left unset; returns how many such pulses there were. */
int srg_oracle_pulse_orbit(const double *times, int P, const double *timeorbit,
                           const double *xx, const double *vv, int numstatevec,
                           double *pos, double *vel)
{
    const double timedelta = timeorbit[1] - timeorbit[0];
    int outside = 0;
    for (int k = 0; k < P; ++k) {
        const double time = times[k];
        const int ilocation = (int)((time - timeorbit[0]) / timedelta);
        const int s = ilocation - 2; /* 0-based index of 1-based ilocation - 1 */
        if (s < 0 || s + 3 > numstatevec - 1) {
            ++outside;
            continue;
        }
        orbithermite_(xx + 3 * s, vv + 3 * s, timeorbit + s, &time, pos + 3 * k, vel + 3 * k);
    }
    return outside;
}
