/*
 * oracle/backproject.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the per-burst backprojection of SRG:
 *   CPU twin  sentinel/azimuth_compress_cpu.c:40-403
 *   GPU entry sentinel/azimuth_compress.cu:33-562 (its arithmetic variants:
 *             FP32 range interpolation, 1/(azend-azstart) scaling, the
 *             |Re| > 1e-18 merge)
 *
 * It is the checker for the CUDA library; the shipped library never links it.
 * Its parity with the reference is pinned by the tests against the reference
 * CPU file compiled from source (oracle/_ref, see oracle/Makefile) and against
 * the golden fixtures that compiled reference produced (tests/golden/).
 *
 * Compiled with -ffp-contract=off so each operation rounds as in an x86-64
 * gcc build of the reference; expressions keep the reference's order.
 *
 * Deliberate, documented differences from the reference, all in places where
 * the reference reads memory it never wrote (so its result there is
 * undefined):
 *   - the per-line parabola of the last line of a burst is zero (the
 *     reference never computes it), so that line is never formed;
 *   - pixels outside [firstpix, lastpix] get azoff = -1 (never formed);
 *   - a formed pixel with azend == azstart (aperture < 2) yields 0 in the GPU
 *     form (the reference computes 0 * inf = NaN, which its merge skips).
 */
#define _GNU_SOURCE
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "srg_oracle.h"

static double pi_value(void) { return 4.0 * atan2(1.0, 1.0); }

void srg_oracle_limits(const double *latlons, double firstlat, double deltalat,
                       double firstlon, double deltalon, int demwidth,
                       int demlength, int *firstline, int *lastline,
                       int *firstpix, int *lastpix)
{
    /* azimuth_compress.cu:295-300 (int() truncates toward zero) */
    int ll = (int)((latlons[0] - firstlat) / deltalat);
    int fl = (int)((latlons[1] - firstlat) / deltalat);
    if (fl < 0) fl = 0;
    if (ll < 0) ll = 0;
    if (fl > demlength - 1) fl = demlength - 1;
    if (ll > demlength - 1) ll = demlength - 1;
    /* azimuth_compress.cu:378-379: lastpix is clamped to W, not W-1 */
    int fp = (int)((latlons[2] - firstlon) / deltalon);
    if (fp < 0) fp = 0;
    int lp = (int)((latlons[3] - firstlon) / deltalon);
    if (lp > demwidth) lp = demwidth;
    *firstline = fl;
    *lastline = ll;
    *firstpix = fp;
    *lastpix = lp;
}

void srg_oracle_setxyz(const int16_t *dem, double *xyz, double *xyzfit,
                       int demwidth, double firstlat, double deltalat,
                       double firstlon, double deltalon, int firstline,
                       int nlines, int firstpix, int lastpix)
{
    const double pi = pi_value();
    const double deg2rad = pi / 180.;
    const double a = 6378137.0;
    const double e2 = 0.0066943799901499996;
    const int half = (lastpix - firstpix) / 2 - 1;
    const int fitpix[3] = {firstpix, firstpix + half, firstpix + 2 * half};
    const long total = (long)nlines * demwidth;

    memset(xyzfit, 0, sizeof(double) * 9 * (size_t)nlines);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < total; ++idx) {
        const int line = (int)(idx / demwidth);
        const int pix = (int)(idx - (long)line * demwidth);
        double *p = xyz + 3 * idx;
        p[0] = 0.;
        p[1] = 0.;
        p[2] = 0.;
        if (pix < firstpix || pix > lastpix) continue;
        const double lat = firstlat + (line + firstline) * deltalat;
        const double rlat = lat * deg2rad;
        const double rlon = (firstlon + pix * deltalon) * deg2rad;
        const double hgt = dem[idx];
        const double slat = sin(rlat);
        const double re = a / sqrt(1.0 - e2 * slat * slat);
        p[0] = (re + hgt) * cos(rlat) * cos(rlon);
        p[1] = (re + hgt) * cos(rlat) * sin(rlon);
        p[2] = (re - (re * e2) + hgt) * slat;
        for (int s = 0; s < 3; ++s) {
            if (pix == fitpix[s]) {
                xyzfit[9 * line + 3 * s + 0] = p[0];
                xyzfit[9 * line + 3 * s + 1] = p[1];
                xyzfit[9 * line + 3 * s + 2] = p[2];
            }
        }
    }
}

void srg_oracle_line_coefs(const double *xyzfit, int nlines,
                           const double *timeorbit, const double *xx,
                           const double *vv, int numstatevec, double tmid,
                           const double *xyz_mid, const double *vel_mid,
                           double wvl, double angc0, double angc1, double prf,
                           int rawdatalines, double *coef)
{
    const double pi = pi_value();
    memset(coef, 0, sizeof(double) * 3 * (size_t)nlines);
    /* the reference loops line = firstline .. lastline-1: nlines-1 rows */
    for (int line = 0; line < nlines - 1; ++line) {
        int y[3];
        for (int s = 0; s < 3; ++s) {
            const double *g = xyzfit + 9 * line + 3 * s;
            double tline, rngpix;
            orbitrangetime_(g, timeorbit, xx, vv, &numstatevec, &tmid, xyz_mid,
                            vel_mid, &tline, &rngpix);
            /* azimuth_compress_cpu.c:339-346: look vector from the burst-centre
             * position (orbitrangetime_ does not update satx/satv). */
            double u0 = g[0] - xyz_mid[0];
            double u1 = g[1] - xyz_mid[1];
            double u2 = g[2] - xyz_mid[2];
            const double umag = sqrt(u0 * u0 + u1 * u1 + u2 * u2);
            u0 = u0 / umag;
            u1 = u1 / umag;
            u2 = u2 / umag;
            const double udotv = vel_mid[0] * u0 + vel_mid[1] * u1 + vel_mid[2] * u2;
            const double fd = (2.0 / wvl) * udotv;
            const double veff = sqrt(vel_mid[0] * vel_mid[0] + vel_mid[1] * vel_mid[1] +
                                     vel_mid[2] * vel_mid[2]);
            const double td =
                (rngpix * (wvl) / 2. / veff / veff * fd - rngpix * (angc0) * pi / 180. / veff) /
                (1. + rngpix * (angc1) * pi / 180. / veff);
            y[s] = (int)(td * (prf) + rawdatalines / 2);
        }
        coef[3 * line + 0] = 0.5 * (y[0] + y[2] - 2. * y[1]);
        coef[3 * line + 1] = 0.5 * (y[2] - y[0]);
        coef[3 * line + 2] = y[1];
    }
}

void srg_oracle_setazoff(const double *coef, double *azoff, int demwidth,
                         int nlines, int firstpix, int lastpix, int aperture,
                         int rawdatalines)
{
    const long total = (long)nlines * demwidth;
    for (long idx = 0; idx < total; ++idx) {
        const int line = (int)(idx / demwidth);
        const int pix = (int)(idx - (long)line * demwidth);
        azoff[idx] = -1;
        if (pix < firstpix || pix > lastpix) continue;
        const double arg = ((float)(pix - firstpix) / (float)(lastpix - firstpix) * 2. - 1.);
        const double fit = coef[line * 3 + 0] * arg * arg + coef[line * 3 + 1] * arg +
                           coef[line * 3 + 2];
        if (fit > aperture / 2 && fit < rawdatalines - aperture / 2) azoff[idx] = fit;
    }
}

int64_t srg_oracle_pixelint(const float *burst, const double *satloc,
                            const double *xyz, const double *azoff,
                            int demwidth, int aperture, int rawdatalines,
                            int samples, double rngstart, double rngend,
                            double dmrg, double wvl, int nlines, float *out,
                            double *acc, const srg_oracle_opts *opts)
{
    const double pi = pi_value();
    const double k4pi = 4. * pi / wvl; /* 4.*pi/wvl*range groups left to right */
    const double rmax = rngend - dmrg;
    const long total = (long)nlines * demwidth;
    const int gpu_lerp = opts ? opts->gpu_lerp : 0;
    const int gpu_scale = opts ? opts->gpu_scale : 0;
    int64_t terms = 0;
#ifdef _OPENMP
    if (opts && opts->nthreads > 0) omp_set_num_threads(opts->nthreads);
#endif

#pragma omp parallel for schedule(dynamic, 64) reduction(+ : terms)
    for (long idx = 0; idx < total; ++idx) {
        double sre = 0., sim = 0.;
        int n = 0;
        if (azoff[idx] > 0.) {
            int a0 = (int)round(azoff[idx] - aperture / 2);
            int a1 = (int)round(azoff[idx] + aperture / 2);
            if (a0 < 0) a0 = 0;
            if (a1 > rawdatalines - 1) a1 = rawdatalines - 1;
            n = a1 - a0;
            const double *p = xyz + 3 * idx;
            for (int az = a0; az < a1; ++az) {
                const double vx = p[0] - satloc[3 * az + 0];
                const double vy = p[1] - satloc[3 * az + 1];
                const double vz = p[2] - satloc[3 * az + 2];
                const double range = sqrt(vx * vx + vy * vy + vz * vz);
                if (!(range >= rngstart && range <= rmax)) continue;
                const double r = (range - rngstart) / dmrg;
                const int ir = (int)floor(r);
                const double fr = r - ir;
                const float *b0 = burst + 2 * ((size_t)az * samples + ir);
                const float *b1 = b0 + 2;
                float cre, cim;
                if (gpu_lerp) {
                    const float w0 = (float)(1 - fr);
                    const float w1 = (float)fr;
                    cre = b0[0] * w0 + b1[0] * w1;
                    cim = b0[1] * w0 + b1[1] * w1;
                } else {
                    cre = (float)((double)b0[0] * (1 - fr) + (double)b1[0] * fr);
                    cim = (float)((double)b0[1] * (1 - fr) + (double)b1[1] * fr);
                }
                const double phase = k4pi * range;
                const double c = cos(phase), s = sin(phase);
                /* complex multiply (a+bi)(c+di) = (ac-bd) + (ad+bc)i */
                const double pre = (double)cre * c - (double)cim * s;
                const double pim = (double)cre * s + (double)cim * c;
                sre = sre + pre;
                sim = sim + pim;
                ++terms;
            }
        }
        if (acc) {
            acc[2 * idx + 0] = sre;
            acc[2 * idx + 1] = sim;
        }
        float ore = (float)sre, oim = (float)sim;
        if (gpu_scale) {
            if (n > 0) {
                const float sc = (float)(1. / (double)n);
                ore = ore * sc;
                oim = oim * sc;
            } else {
                ore = 0.f;
                oim = 0.f;
            }
        }
        out[2 * idx + 0] = ore;
        out[2 * idx + 1] = oim;
    }
    return terms;
}

/* Executed-term count of pixelint without the sum: the same aperture window
 * (azimuth_compress_cpu.c:50-57) and range test (:63-64) per pixel and pulse. */
int64_t srg_oracle_count_terms(const double *satloc, const double *xyz, const double *azoff,
                               int demwidth, int aperture, int rawdatalines, double rngstart,
                               double rngend, double dmrg, int nlines, int nthreads)
{
    const double rmax = rngend - dmrg;
    const long total = (long)nlines * demwidth;
    int64_t terms = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : terms)
    for (long idx = 0; idx < total; ++idx) {
        if (!(azoff[idx] > 0.)) continue;
        int a0 = (int)round(azoff[idx] - aperture / 2);
        int a1 = (int)round(azoff[idx] + aperture / 2);
        if (a0 < 0) a0 = 0;
        if (a1 > rawdatalines - 1) a1 = rawdatalines - 1;
        const double *p = xyz + 3 * idx;
        for (int az = a0; az < a1; ++az) {
            const double vx = p[0] - satloc[3 * az + 0];
            const double vy = p[1] - satloc[3 * az + 1];
            const double vz = p[2] - satloc[3 * az + 2];
            const double range = sqrt(vx * vx + vy * vy + vz * vz);
            if (range >= rngstart && range <= rmax) ++terms;
        }
    }
    return terms;
}

/* Merge rules. */
static int merge_gpu(float re) { return fabs((double)re) > 1.e-18; }
static int merge_cpu(float re)
{
    /* C abs() of the double converted to int (azimuth_compress_cpu.c:387):
     * truncation toward zero; out-of-range and NaN convert to INT_MIN on
     * x86-64, whose abs() stays negative. */
    const double d = (double)re;
    int iv;
    if (d > -2147483649.0 && d < 2147483648.0) iv = (int)d;
    else iv = INT_MIN;
    return iv != 0 && iv != INT_MIN;
}

int64_t srg_oracle_burst(const float *burst, const double *satloc,
                         int rawdatalines, int samples, int demwidth,
                         int demlength, const int16_t *dem, float *geo,
                         double deltalat, double deltalon, double firstlat,
                         double firstlon, const double *latlons,
                         const double *timeorbit, const double *xx,
                         const double *vv, int numstatevec, double rngstart,
                         double rngend, double tmid, const double *xyz_mid,
                         const double *vel_mid, double dmrg, double wvl,
                         int aperture, double angc0, double angc1, double prf,
                         float *raw, int *firstline_out, int *nlines_out,
                         const srg_oracle_opts *opts)
{
    int firstline, lastline, firstpix, lastpix;
    srg_oracle_limits(latlons, firstlat, deltalat, firstlon, deltalon, demwidth,
                      demlength, &firstline, &lastline, &firstpix, &lastpix);
    const int nlines = lastline - firstline + 1;
    if (firstline_out) *firstline_out = firstline;
    if (nlines_out) *nlines_out = nlines;
    const int gpu_form = opts && opts->gpu_scale;
    if (!gpu_form && nlines == 1) return -1; /* azimuth_compress_cpu.c:254-257 */

    const size_t npix = (size_t)nlines * demwidth;
    double *xyz = malloc(sizeof(double) * 3 * npix);
    double *xyzfit = malloc(sizeof(double) * 9 * (size_t)nlines);
    double *coef = malloc(sizeof(double) * 3 * (size_t)nlines);
    double *azoff = malloc(sizeof(double) * npix);
    float *out = malloc(sizeof(float) * 2 * npix);
    const int16_t *slab = dem + (size_t)firstline * demwidth;

    srg_oracle_setxyz(slab, xyz, xyzfit, demwidth, firstlat, deltalat, firstlon,
                      deltalon, firstline, nlines, firstpix, lastpix);
    srg_oracle_line_coefs(xyzfit, nlines, timeorbit, xx, vv, numstatevec, tmid,
                          xyz_mid, vel_mid, wvl, angc0, angc1, prf, rawdatalines,
                          coef);
    srg_oracle_setazoff(coef, azoff, demwidth, nlines, firstpix, lastpix,
                        aperture, rawdatalines);
    const int64_t terms =
        srg_oracle_pixelint(burst, satloc, xyz, azoff, demwidth, aperture,
                            rawdatalines, samples, rngstart, rngend, dmrg, wvl,
                            nlines, out, NULL, opts);
    float *dst = geo + 2 * (size_t)firstline * demwidth;
    for (size_t i = 0; i < npix; ++i) {
        const int m = gpu_form ? merge_gpu(out[2 * i]) : merge_cpu(out[2 * i]);
        if (m) {
            dst[2 * i] = out[2 * i];
            dst[2 * i + 1] = out[2 * i + 1];
        }
    }
    if (raw) memcpy(raw, out, sizeof(float) * 2 * npix);
    free(xyz);
    free(xyzfit);
    free(coef);
    free(azoff);
    free(out);
    return terms;
}

void srg_oracle_azimuth_compress_(
    const float *burstdata, const double *satloc, const int *rawdatalines,
    const int *samplesPerBurst, const int *demwidth, const int *demlength,
    const int *fdout, const int *fddem, const double *deltalat,
    const double *deltalon, const double *firstlat, const double *firstlon,
    const double *latlons, const double *timeorbit, const double *xx,
    const double *vv, const int *numstatevec, const double *rngstart,
    const double *rngend, const double *tstart, const double *tend,
    const double *tmid, const double *xyz_mid, const double *vel_mid,
    const double *t, const double *dtaz, const double *dmrg,
    const double *wvl, const int *aperture, const int *iaperture,
    const double *angc0, const double *angc1, const double *prf)
{
    (void)tstart; (void)tend; (void)t; (void)dtaz; (void)iaperture;
    int firstline, lastline, firstpix, lastpix;
    srg_oracle_limits(latlons, *firstlat, *deltalat, *firstlon, *deltalon,
                      *demwidth, *demlength, &firstline, &lastline, &firstpix,
                      &lastpix);
    const int nlines = lastline - firstline + 1;
    const int W = *demwidth;
    const size_t npix = (size_t)nlines * W;
    int16_t *slab = calloc(npix, sizeof(int16_t));
    if (pread(*fddem, slab, npix * 2, (off_t)firstline * W * 2) < 0) { /* keep going, as the reference */ }
    double *xyz = malloc(sizeof(double) * 3 * npix);
    double *xyzfit = malloc(sizeof(double) * 9 * (size_t)nlines);
    double *coef = malloc(sizeof(double) * 3 * (size_t)nlines);
    double *azoff = malloc(sizeof(double) * npix);
    float *out = malloc(sizeof(float) * 2 * npix);
    float *cur = calloc(2 * npix, sizeof(float));
    srg_oracle_setxyz(slab, xyz, xyzfit, W, *firstlat, *deltalat, *firstlon,
                      *deltalon, firstline, nlines, firstpix, lastpix);
    srg_oracle_line_coefs(xyzfit, nlines, timeorbit, xx, vv, *numstatevec, *tmid,
                          xyz_mid, vel_mid, *wvl, *angc0, *angc1, *prf,
                          *rawdatalines, coef);
    srg_oracle_setazoff(coef, azoff, W, nlines, firstpix, lastpix, *aperture,
                        *rawdatalines);
    srg_oracle_opts o = {1, 1, 0};
    srg_oracle_pixelint(burstdata, satloc, xyz, azoff, W, *aperture, *rawdatalines,
                        *samplesPerBurst, *rngstart, *rngend, *dmrg, *wvl, nlines,
                        out, NULL, &o);
    const off_t off = (off_t)firstline * W * 8;
    if (pread(*fdout, cur, npix * 8, off) < 0) { /* as the reference: ignore */ }
    for (size_t i = 0; i < npix; ++i) {
        if (merge_gpu(out[2 * i])) {
            cur[2 * i] = out[2 * i];
            cur[2 * i + 1] = out[2 * i + 1];
        }
    }
    if (pwrite(*fdout, cur, npix * 8, off) < 0) { /* as the reference: ignore */ }
    free(slab); free(xyz); free(xyzfit); free(coef); free(azoff); free(out); free(cur);
}
