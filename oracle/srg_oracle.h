/*
 * oracle/srg_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of SRG's per-burst time-domain backprojection
 * (sentinel/azimuth_compress_cpu.c, sentinel/azimuth_compress.cu) and of the
 * orbit helpers it calls.  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark use it, always as the checker.
 */
#ifndef SRG_ORACLE_H
#define SRG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- orbit helpers (oracle/orbit.c), Fortran calling convention ---- */
void orbithermite_(const double *x, const double *v, const double *t,
                   const double *tq, double *xq, double *vq);
int intp_orbit_(const double *timeorbit, const double *xx, const double *vv,
                const int *numstatevec, const double *time, double *xyz,
                double *vel);
void orbitrangetime_(const double *xyz, const double *timeorbit, const double *xx,
                     const double *vv, const int *numstatevec, const double *tline0,
                     const double *satx0, const double *satv0, double *tline,
                     double *range);

/* Per-pulse orbit of sentinel/sentineltimingsub.f90:41,55-63 (unclamped
 * Hermite window).  Returns the number of pulses left unset because their
 * window would leave the state-vector array. */
int srg_oracle_pulse_orbit(const double *times, int P, const double *timeorbit,
                           const double *xx, const double *vv, int numstatevec,
                           double *pos, double *vel);

/* ---- backprojection (oracle/backproject.c) ---- */

/* Arithmetic variant of the per-pixel sum.
 *   gpu_lerp = 0: range interpolation in double, rounded to complex64
 *                 (azimuth_compress_cpu.c:73);
 *   gpu_lerp = 1: interpolation in FP32 (azimuth_compress.cu:69).
 *   gpu_scale = 1: multiply the complex64 sum by (float)(1/(azend-azstart))
 *                 (azimuth_compress.cu:78-79); 0: unscaled (CPU form).
 *   nthreads:  OpenMP threads (<= 0: runtime default). */
typedef struct srg_oracle_opts {
    int gpu_lerp;
    int gpu_scale;
    int nthreads;
} srg_oracle_opts;

/* Line / pixel limits of a burst from its lat/lon box
 * (azimuth_compress.cu:295-301 and 378-379). */
void srg_oracle_limits(const double *latlons, double firstlat, double deltalat,
                       double firstlon, double deltalon, int demwidth,
                       int demlength, int *firstline, int *lastline,
                       int *firstpix, int *lastpix);

/* DEM slab -> ECEF (azimuth_compress_cpu.c:89-152).  dem: [nlines][W] int16
 * (rows firstline..); xyz: [nlines][W][3]; xyzfit: [nlines][9]. */
void srg_oracle_setxyz(const int16_t *dem, double *xyz, double *xyzfit,
                       int demwidth, double firstlat, double deltalat,
                       double firstlon, double deltalon, int firstline,
                       int nlines, int firstpix, int lastpix);

/* Per-line azimuth-centre parabola (azimuth_compress_cpu.c:321-359).
 * coef: [nlines][3].  The reference leaves the last row unset; here it is
 * zero, which makes the last line of every burst unformed. */
void srg_oracle_line_coefs(const double *xyzfit, int nlines,
                           const double *timeorbit, const double *xx,
                           const double *vv, int numstatevec, double tmid,
                           const double *xyz_mid, const double *vel_mid,
                           double wvl, double angc0, double angc1, double prf,
                           int rawdatalines, double *coef);

/* azoff from the parabolas (azimuth_compress_cpu.c:155-175).  Pixels outside
 * [firstpix, lastpix] (left unset by the reference) get -1. */
void srg_oracle_setazoff(const double *coef, double *azoff, int demwidth,
                         int nlines, int firstpix, int lastpix, int aperture,
                         int rawdatalines);

/* Per-pixel aperture sum (azimuth_compress_cpu.c:40-86 / .cu:33-82).
 * burst: [P][S] complex64 as interleaved float; out: [nlines][W] complex64.
 * acc (optional): [nlines][W] complex128, the double sum before rounding.
 * Returns the number of executed terms. */
int64_t srg_oracle_pixelint(const float *burst, const double *satloc,
                            const double *xyz, const double *azoff,
                            int demwidth, int aperture, int rawdatalines,
                            int samples, double rngstart, double rngend,
                            double dmrg, double wvl, int nlines, float *out,
                            double *acc, const srg_oracle_opts *opts);

/* Executed-term count of srg_oracle_pixelint on the same inputs (its window
 * and range test, no sum). */
int64_t srg_oracle_count_terms(const double *satloc, const double *xyz, const double *azoff,
                               int demwidth, int aperture, int rawdatalines, double rngstart,
                               double rngend, double dmrg, int nlines, int nthreads);

/* One whole burst in memory.  dem: the full [demlength][W] int16 DEM;
 * geo: the full [demlength][W] complex64 raster, merged in place with the
 * GPU rule (|Re| > 1e-18, azimuth_compress.cu:527-531) when
 * opts->gpu_scale, else with the CPU rule (integer abs,
 * azimuth_compress_cpu.c:385-389).  raw (optional): [nlines][W] complex64
 * output before the merge.  Returns the executed term count, or -1 when the
 * burst is skipped (CPU form, nlines == 1). */
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
                         const srg_oracle_opts *opts);

/* The 33-argument by-reference entry with the GPU entry's semantics
 * (azimuth_compress.cu:181-562): reads the DEM slab from *fddem, merges into
 * *fdout.  Uses pread/pwrite; prints nothing. */
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
    const double *angc0, const double *angc1, const double *prf);

#ifdef __cplusplus
}
#endif
#endif
