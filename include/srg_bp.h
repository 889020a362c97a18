/*
 * srg_bp.h -- C ABI of the B200 (sm_100a) time-domain backprojection library
 * (libsrg_bp.so), a drop-in for the azimuth-compression entry of ASFHyP3/SRG.
 *
 * Plain C: pointers, sizes and scalars only.  Complex samples are complex64,
 * stored as interleaved float pairs (re, im), exactly the layout of Fortran
 * `complex` and C `float _Complex`.
 *
 * Error convention of the status-returning entries: 0 on success, a negative
 * SRG_E* code otherwise; srg_last_error() returns a one-line message for the
 * calling thread.
 */
#ifndef SRG_BP_H
#define SRG_BP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SRG_OK            0
#define SRG_E_ARG        -1   /* invalid argument or size */
#define SRG_E_CUDA       -2   /* a CUDA runtime call failed */
#define SRG_E_IO         -3   /* DEM read or .geo read/write failed */
#define SRG_E_TIMEOUT    -4   /* a bounded device-side wait gave up */
#define SRG_E_NOMEM      -5   /* device or host allocation failed */
#define SRG_E_UNSUPPORTED -6  /* configuration not supported by this build */

/* Arithmetic of the per-term sum. */
#define SRG_FORM_FP64   0  /* geometry, phase, sincos and accumulation in FP64,
                              FP32 range interpolation: the arithmetic of
                              sentinel/azimuth_compress.cu:59-79 */
#define SRG_FORM_SPLIT  1  /* FP64 only for orbit, pixel ECEF and one reference
                              range per tile and pulse; compensated FP32 for the
                              per-term differential range and phase */

typedef struct srg_bp_options {
    int form;          /* SRG_FORM_FP64 or SRG_FORM_SPLIT */
    int tile_cfg;      /* kernel shape index (srg_tile_config_count()); -1: tuned default */
    int device;        /* CUDA device ordinal; -1: current device */
    int centres_on_host; /* must be 0: the per-line azimuth centres are solved
                            on the GPU (1 is SRG_E_UNSUPPORTED wherever the
                            entry would solve them) */
    int verbose;       /* 1: print the reference's "Burst line limits" line */
    int spin_limit;    /* polls of a bounded device-side wait (for range lines
                          still uploading, or for a staged tile) before the
                          kernel gives up and the call returns SRG_E_TIMEOUT;
                          0: the default, 4,194,304 (about 1-2 s) */
    int full_lines;    /* drop-in: 1 uploads every line in full; 0 (default)
                          only its range band (srg_dropin_last_bytes) */
    long long scratch_limit; /* bytes of device scratch one drop-in call may
                          hold (range lines, orbit, DEM box, output box, work
                          list); a call needing more returns SRG_E_NOMEM before
                          any GPU work; 0: no limit */
    int overlap;       /* drop-in: 1 returns once the call's range lines are
                          on the device; the end of its sum, the copy back and
                          the merge into *fdout finish behind the caller (in
                          call order, on a descriptor duplicated from fdout),
                          while the next call reads its DEM box and uploads.
                          A failure of that part is returned by the next call
                          on the device or by srg_dropin_flush().  The merge
                          into *fdout of a call is complete when the next
                          call without overlap, srg_dropin_flush() or the
                          process's normal exit returns.  The device then
                          keeps two calls' scratch (two contexts, used in
                          turn).  0 (default): every call returns with its
                          merge done, as the reference.
                          The environment variable SRG_DROPIN_OVERLAP=1 sets
                          it in the process-wide defaults. */
    int tile_shear;    /* lines per 32 grid columns by which the tiles are
                          sheared (a tile's column x sits floor(tile_shear x /
                          32) lines lower), in [-SRG_MAX_TILE_SHEAR,
                          SRG_MAX_TILE_SHEAR] and offsetting a tile's columns
                          by fewer lines than it is tall; 0 (the default):
                          rectangular tiles; SRG_TILE_SHEAR_AUTO: chosen per
                          burst from its geometry so that a tile's rows of
                          pixels follow the lines of constant azimuth centre.
                          That pays on gentle terrain (fewer pulses per tile)
                          and costs over strong relief (a tile's range window
                          outgrows the staged one), so the scene plan's tuner
                          times both (srg_scene_autotune).  The
                          warp-specialised shapes take it; the
                          first-generation shapes keep rectangular tiles.
                          Results depend on it only through the split form's
                          per-tile closed forms (within its error budget). */
} srg_bp_options;

#define SRG_TILE_SHEAR_AUTO 1000
#define SRG_MAX_TILE_SHEAR 8

/* Fill *o with the defaults (split form, tuned tile, current device,
 * centres on the GPU, quiet, default wait limit, range band, no scratch
 * limit, calls not overlapped unless SRG_DROPIN_OVERLAP=1, rectangular
 * tiles). */
void srg_bp_default_options(srg_bp_options *o);

/* Message of the last failing call on this thread ("" if none). */
const char *srg_last_error(void);

/* ------------------------------------------------------------------------
 * Drop-in entry.  Replaces
 *     extern "C" void azimuth_compress_(...)   sentinel/azimuth_compress.cu:181-214
 * called by reference from sentinel/backprojectgpusub.f90:244-247
 * (gfortran implicit interface: lower-case name + '_', every argument by
 * reference, no hidden lengths).  Same 33 arguments, same meaning, same file
 * side effects: reads DEM rows [firstline, firstline+nlines) from *fddem and
 * read-modify-writes the same rows of the complex64 raster on *fdout,
 * replacing a pixel where |Re(new)| > 1e-18 (azimuth_compress.cu:510-537).
 * Like the reference it returns nothing; failures are reported on stderr and
 * in srg_last_error().  Uses the options of srg_set_default_options()
 * (split form unless changed).  tstart, tend, t, dtaz and iaperture are
 * accepted and unused, as in the reference.
 * ------------------------------------------------------------------------ */
void azimuth_compress_(
    float *burstdata,      /* [rawdatalines][samplesPerBurst] complex64 */
    double *satloc,        /* [rawdatalines][3] ECEF m */
    int *rawdatalines, int *samplesPerBurst, int *demwidth, int *demlength,
    int *fdout, int *fddem,
    double *deltalat, double *deltalon, double *firstlat, double *firstlon,
    double *latlons,       /* [4] min lat, max lat, min lon, max lon (deg) */
    double *timeorbit,     /* [numstatevec] s */
    double *xx, double *vv,/* [numstatevec][3] ECEF m, m/s */
    int *numstatevec,
    double *rngstart, double *rngend, double *tstart, double *tend,
    double *tmid, double *xyz_mid, double *vel_mid, double *t, double *dtaz,
    double *dmrg, double *wvl, int *aperture, int *iaperture,
    double *angc0, double *angc1, double *prf);

/* Same call with a status and explicit options (opts may be NULL).  On
 * SRG_E_TIMEOUT only rows whose every formed pixel was computed have been
 * merged into *fdout; the other rows are left as they were. */
int srg_azimuth_compress(
    const float *burstdata, const double *satloc, int rawdatalines,
    int samplesPerBurst, int demwidth, int demlength, int fdout, int fddem,
    double deltalat, double deltalon, double firstlat, double firstlon,
    const double *latlons, const double *timeorbit, const double *xx,
    const double *vv, int numstatevec, double rngstart, double rngend,
    double tmid, const double *xyz_mid, const double *vel_mid, double dmrg,
    double wvl, int aperture, double angc0, double angc1, double prf,
    const srg_bp_options *opts);

/* Options used by azimuth_compress_ (process-wide). */
void srg_set_default_options(const srg_bp_options *o);

/* Bytes the last drop-in call on `device` (-1: current) copied to the device
 * (range lines of its range band, orbit, DEM box) and back (row blocks of the
 * output box).  The drop-in uploads only the range bins a term of a formed
 * pixel can read (with a margin of 8 bins), found on the device from the DEM
 * box and the azimuth centres before the lines go up; the reference uploads
 * every line in full (azimuth_compress.cu:367-368). */
int srg_dropin_last_bytes(int device, long long *h2d, long long *d2h);

/* Waits until every overlapped drop-in call on `device` (-1: every device)
 * has finished its merge; returns the first failure among them not yet
 * returned by a later call (message in srg_last_error()), else SRG_OK.
 * Runs by itself at the process's normal exit. */
int srg_dropin_flush(int device);

/* ------------------------------------------------------------------------
 * Per-burst scalars of the azimuth_compress_ call, derived as
 * sentinel/backprojectgpusub.f90 derives them before each call: burstparams
 * (:406-429) from the first line's header, the steering-angle fit fdopcoefs
 * (:262-309, linfit :381-403; all but 20 lines at each end), the aperture
 * (:190-209, from the velocity of pulse P/2 in 1-based numbering) and the
 * azimuth and range limits (:213-227).  Replaces that Fortran, which the
 * caller runs on the host; the arithmetic keeps its single- and
 * double-precision steps, so the values are the reference's bit for bit.
 * ------------------------------------------------------------------------ */
typedef struct srg_burst_params_t {
    double starttime;  /* s of day, line 0's header bytes 68-75 */
    double prf;        /* Hz */
    double samplefreq; /* Hz */
    double pri;        /* s */
    double range0;     /* m, near range incl. the reference's 60 m calibration */
    double wvl;        /* m (the reference's single-precision literal) */
    double angc0, angc1; /* steering fit: angle (deg) = angc0 + angc1 t */
    double tstart, tend, tmid, dtaz; /* s */
    double rngstart, rngend, dmrg;   /* m */
    int aperture;      /* pulses */
    int pad;
} srg_burst_params_t;

/* lines: [P][ld] complex64 decoded range lines of one burst whose first 10
 * samples (80 bytes) still hold each line's header (the reference zeroes
 * them only after this step, backprojectgpusub.f90:191); S: samples per line
 * including those 10; satvel: [P][3] per-pulse velocity (m/s).  Host
 * pointers.  SRG_E_ARG for fewer than 41 lines, a zero PRI code or an
 * unknown range decimation code. */
int srg_burst_params(const float *lines, long long ld, int P, int S, const double *satvel,
                     srg_burst_params_t *out);

/* ------------------------------------------------------------------------
 * Device-resident bursts (no file I/O; all pointers are device pointers
 * unless noted).  The unit of the batched scene launch.
 * ------------------------------------------------------------------------ */
typedef struct srg_burst_desc {
    const float *burst;      /* [P][ldb] complex64 range lines (device) */
    const double *satloc;    /* [P][3] (device) */
    const int16_t *dem;      /* DEM row `firstline` of the grid, row stride dem_ld elements (device) */
    float *out;              /* output row 0 (= grid line firstline), row stride out_ld complex64,
                                column c = grid pixel c + out_pix0 (device) */
    const double *coef;      /* optional [nlines][3] azimuth-centre parabolas (device);
                                NULL: solved on the device from the orbit below */
    int64_t ldb, dem_ld, out_ld;
    int P, S;
    int demwidth;            /* W */
    int firstline, nlines, firstpix, lastpix; /* as derived by the reference from latlons */
    int out_pix0;
    int aperture;
    double firstlat, deltalat, firstlon, deltalon;
    double rngstart, rngend, dmrg, wvl;
    /* azimuth-centre inputs (host pointers; used when coef == NULL) */
    const double *timeorbit, *xx, *vv;
    int numstatevec;
    double tmid, xyz_mid[3], vel_mid[3], angc0, angc1, prf;
    /* the range bins held in `burst`: bins [bin0, bin0 + nbins) of every
     * line, column c of a row being bin bin0 + c (bin0 even); terms whose taps
     * fall outside read zeros.  0 and 0: the whole line (nbins = S). */
    int bin0, nbins;
} srg_burst_desc;

/* Backproject `n` bursts in one persistent launch on `stream` (a
 * cudaStream_t; NULL = default stream).  Each burst writes its pixels
 * [firstpix, min(lastpix, W-1)] x [0, nlines) of `out` (formed pixels get the
 * scaled complex64 sum, the others 0); bursts must not share output pixels
 * (see srg_merge_device for the ordered merge).  Asynchronous: returns after
 * enqueueing; srg_sync_check() reports device-side errors. */
int srg_bp_bursts_device(const srg_burst_desc *bursts, int n,
                         const srg_bp_options *opts, void *stream);

/* Tile shear (lines per 32 columns) and tiles across and down that shape
 * `tile_cfg` (-1: the split form's default) takes for burst *b under
 * `tile_shear` (SRG_TILE_SHEAR_AUTO: the geometric choice).  Host only: no
 * device memory is read, only the descriptor's scalars. */
int srg_tile_shear(const srg_burst_desc *b, int tile_cfg, int tile_shear, int *shear,
                   int *tiles_x, int *tiles_y);

/* One burst whose range lines are still being copied to the device, in
 * blocks of pulse rows, by the caller (a pipelined upload; the drop-in entry
 * does the same with its own copies).  The caller raises the device word
 * *ready_word to ready_base + n once the first n * ready_rows pulse rows are
 * in device memory (e.g. a 4-byte copy on its copy stream after each block;
 * the word must only grow, and start below ready_base + 1).  The kernel starts
 * at once and takes each chunk of pulses when its rows are in, waiting at
 * most opts->spin_limit polls; if a wait gives up, the tiles not yet stored
 * keep their old output and srg_sync_check() returns SRG_E_TIMEOUT.  Only the
 * default split shape has such a twin (SRG_E_UNSUPPORTED otherwise).
 * Asynchronous, as srg_bp_bursts_device.  No reference counterpart (the
 * reference copies the whole burst before it launches, azimuth_compress.cu:
 * 367-368). */
int srg_bp_burst_device_gated(const srg_burst_desc *b, const int *ready_word, int ready_base,
                              int ready_rows, const srg_bp_options *opts, void *stream);

/* ------------------------------------------------------------------------
 * Scene plans: a reusable, graph-captured pass over a fixed set of
 * device-resident bursts (e.g. the 27 bursts of an IW scene, or a stack of
 * repeat-pass acquisitions), with an ordered merge into a scene raster.
 * No reference counterpart: the reference processes one burst per call
 * (sentinel/backprojectgpusub.f90:140-248 loops azimuth_compress_ serially)
 * and merges each into the .geo file in that order.
 * ------------------------------------------------------------------------ */
typedef struct srg_scene srg_scene;

/* Build a plan.  Every descriptor's coef must be NULL (the plan solves the
 * azimuth centres on the device each pass).  scene (device, complex64,
 * scene_lines x scene_cols, row stride scene_ld) may be NULL; otherwise each
 * pass merges burst outputs into it in burst order with the reference's rule
 * (|Re| > 1e-18), burst rows placed at grid line firstline + row and column
 * out_pix0 + c.  Allocates the plan's own device memory. */
int srg_scene_create(const srg_burst_desc *bursts, int n, float *scene, int64_t scene_ld,
                     int scene_lines, int scene_cols, const srg_bp_options *opts,
                     srg_scene **out);
/* Enqueue one pass on `stream`: azimuth centres of every line of every burst
 * (one launch), the persistent backprojection of all bursts (one launch),
 * the ordered merge (one launch).  On a non-default stream the first pass
 * is captured in a CUDA graph that later passes replay. */
int srg_scene_run(srg_scene *s, void *stream);
/* Enqueue chosen stages of a pass without a graph: 1 = azimuth centres,
 * 2 = backprojection, 4 = merge (OR them). */
int srg_scene_run_stages(srg_scene *s, int stages, void *stream);
/* Wait for `stream` and report device-side errors of the plan's kernels. */
int srg_scene_sync(srg_scene *s, void *stream);
/* Exact executed-term count of one pass (computed once, blocking). */
int srg_scene_terms(srg_scene *s, int64_t *terms);
/* Autotuner: time every compiled kernel shape of the plan's form on this
 * scene (`iters` timed launches each) and keep the fastest, or take the
 * cached best shape of a scene of the same shape (srg_scene_autotune); with
 * rectangular and with geometrically sheared tiles (srg_bp_options.
 * tile_shear), whichever is faster on this scene (timed on every call). */
int srg_scene_tune(srg_scene *s, int iters, int *best_cfg, double *best_ms);
/* Autotuner with the range interpolation in its search.  With
 * interp_budget > 0 it first estimates, from a sample of every burst's lines,
 * the RMS phase error (rad) each interpolation adds (srg_interp_error): the
 * reference's linear interpolation of the original lines when that is within
 * the budget, else linear interpolation between the bins of 2x-oversampled
 * lines, which the plan then makes in every pass (srg_oversample_range_device
 * into buffers of its own; the lines must be whole, bin0 = 0).  It then times
 * the kernel shapes of the plan's form, unless use_cache finds the best shape
 * of an earlier tuning of a scene of the same shape (same form,
 * interpolation, and bursts' pulses, samples, grid lines and columns to
 * within 64, 1024, 64, 64); results are kept for the process and, when the
 * environment variable SRG_TUNE_CACHE names a file, appended to it and read
 * back by later processes.  srg_scene_tune is this with no interpolation
 * budget and the cache on.  No reference counterpart. */
#define SRG_INTERP_LINEAR       0  /* the original lines (azimuth_compress.cu:65-69) */
#define SRG_INTERP_OVERSAMPLED2 1  /* 2x-oversampled lines, 8-tap half samples */
typedef struct srg_tune_request {
    int iters;             /* timed launches per shape (< 1: 3) */
    int use_cache;         /* 1: take a cached shape without timing */
    double interp_budget;  /* RMS phase error (rad) the interpolation may add;
                              <= 0: keep the plan's interpolation */
} srg_tune_request;
typedef struct srg_tune_result {
    int tile_cfg;          /* shape in use */
    int interp;            /* SRG_INTERP_* in use */
    int from_cache;        /* 1: the shape came from the cache (no shape timed) */
    int tile_shear;        /* tile shear in use: 0 (rectangular tiles) or
                              SRG_TILE_SHEAR_AUTO (the geometric shear), timed
                              against each other on every call: which pays
                              depends on the terrain, which the cache does not
                              key on */
    double ms;             /* mean backprojection time of the choice (-1:
                              nothing timed: a cached shape and no burst that
                              the geometric shear would shear) */
    double err_linear, err_oversampled; /* estimated RMS phase error (rad) of
                              each interpolation (-1: not estimated) */
} srg_tune_result;
int srg_scene_autotune(srg_scene *s, const srg_tune_request *req, srg_tune_result *res);
/* Use an interpolation (SRG_INTERP_*) without tuning, and read it back. */
int srg_scene_set_interp(srg_scene *s, int interp);
int srg_scene_interp(const srg_scene *s);

/* Expected RMS phase error (rad) that linear interpolation adds to a term,
 * on the lines as they are (*err_linear) and after 2x oversampling
 * (*err_oversampled), from the mean power spectrum of `sample_lines` lines
 * spread over the nlines lines ([nlines][ld] complex64, nsamps samples,
 * device).  For a fractional offset u the linear interpolant differs from
 * the band-limited line by (1-u) + u e^{i 2 pi nu} - e^{i 2 pi nu u} per unit
 * of spectrum at nu cycles/sample (on the oversampled line, the same between
 * an original and a filtered half sample); half that error power lies across
 * the signal.  Blocking; allocates scratch (cuFFT). */
int srg_interp_error(const float *lines, long long ld, int nlines, int nsamps, int sample_lines,
                     double *err_linear, double *err_oversampled, void *stream);

/* Select a kernel shape, or a form and shape (-1: that form's default).
 * Blocking: waits for the device to finish the work in flight (the plan's
 * burst descriptors are rewritten), on any stream. */
int srg_scene_set_shape(srg_scene *s, int tile_cfg);
int srg_scene_set_form(srg_scene *s, int form, int tile_cfg);
/* Kernel shape index in use. */
int srg_scene_shape(const srg_scene *s);
/* Tile shear (lines per 32 columns) in use for burst `burst` of the plan. */
int srg_scene_tile_shear(const srg_scene *s, int burst, int *shear);
void srg_scene_destroy(srg_scene *s);

/* Exact count of executed terms (pixel, pulse pairs inside the aperture
 * window that pass the reference's range test) of the given bursts, computed
 * on the device with the reference's FP64 arithmetic.  Blocking. */
int srg_count_terms_device(const srg_burst_desc *bursts, int n, int64_t *terms,
                           void *stream);

/* Ordered merge of a burst output into a raster: dst[l][c] = src[l][c] where
 * |Re(src)| > 1e-18 (azimuth_compress.cu:527-531).  Device pointers. */
int srg_merge_device(float *dst, int64_t dst_ld, const float *src, int64_t src_ld,
                     int rows, int cols, void *stream);

/* Per-line azimuth-centre parabolas (azimuth_compress.cu:438-481) computed
 * on the device into coef_out ([nlines][3], device).  Blocking. */
int srg_line_centres_device(const srg_burst_desc *b, double *coef_out, void *stream);

/* Per-pulse ECEF position and velocity by 4-point Hermite interpolation of
 * the state vectors (sentinel/sentineltimingsub.f90:55-66, orbithermite.f),
 * one thread per pulse.  times/pos/vel: device; timeorbit/xx/vv: host. */
int srg_pulse_orbit_device(const double *times, int P, const double *timeorbit,
                           const double *xx, const double *vv, int numstatevec,
                           double *pos, double *vel, void *stream);

/* Synchronise `stream` and report any device-side error flag raised by the
 * library's kernels since the last check (SRG_E_TIMEOUT) or CUDA error. */
int srg_sync_check(void *stream);

/* ------------------------------------------------------------------------
 * No-allocation variant of srg_bp_bursts_device for one burst.  It has no
 * counterpart in the reference (whose entry allocates and frees device memory
 * on every burst).
 *
 * For callers that cannot call cudaMalloc: a process whose device memory is
 * already reserved by a pool it does not own (a serving runtime or a
 * framework allocator holding the HBM), or a latency-critical stream that
 * cannot take the device-wide synchronisation of cudaMalloc/cudaFree.  The
 * caller passes the inputs and the output (as for srg_bp_bursts_device);
 * the work counter, error word, burst and TMA descriptors, orbit state
 * vectors and per-line azimuth-centre parabolas live in one static device
 * array of SRG_NOALLOC_SCRATCH_BYTES that every GPU loading this library
 * holds until the process exits.  Limits: at most SRG_NOALLOC_MAX_LINES grid
 * lines, and at most SRG_NOALLOC_MAX_STATEVEC state vectors when b->coef is
 * NULL; larger bursts are rejected with SRG_E_ARG before any GPU work.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress): make that first call before any stream capture.
 * Every call shares the array and clears only the counter and the error word;
 * calls whose GPU work overlaps (other streams, other host threads) race.
 * opts->centres_on_host with b->coef NULL is SRG_E_UNSUPPORTED, as in
 * srg_bp_bursts_device.  Blocking: the call copies its descriptors from host
 * memory, waits for `stream` (cudaStreamSynchronize) and reads the error word
 * back before it returns, with SRG_E_TIMEOUT if a device-side wait gave up.
 * ------------------------------------------------------------------------ */
#define SRG_NOALLOC_MAX_LINES    8192
#define SRG_NOALLOC_MAX_STATEVEC 64
#define SRG_NOALLOC_SCRATCH_BYTES (2048 + 7 * 8 * SRG_NOALLOC_MAX_STATEVEC + 3 * 8 * SRG_NOALLOC_MAX_LINES)
int srg_bp_burst_device_noalloc(const srg_burst_desc *b, const srg_bp_options *opts,
                                void *stream);

/* Testing hook: set the drop-in entry's call number on `device` (-1:
 * current), 0 .. 2^24.  The number restarts at 1 after 2^24 calls; a test
 * sets it near there to run calls across the restart. */
int srg_test_set_dropin_sequence(int device, int seq);

/* Calibration: measured FMA issue-rate peak of the current device in
 * TFLOP/s (2 flops per FMA), FP32 (fp64 = 0) or FP64 (fp64 = 1), from a
 * full-occupancy chain-of-FMA kernel timed with CUDA events.  Blocking. */
int srg_measure_fma_peak(int fp64, double *tflops);

/* Number of compiled kernel shapes, and the shape of one of them. */
int srg_tile_config_count(void);
int srg_tile_config(int idx, int *tile_x, int *tile_y, int *threads, int *chunk,
                    int *window);
/* Human-readable kernel template and shape of shape `idx` ("" if none). */
const char *srg_tile_config_name(int idx);

/* Synthetic-scene support: forward-project a per-pixel reflectivity field
 * (complex64, [nlines][refl_ld] of the burst's grid rows, device) into
 * the burst's range lines (accumulates into burst, device), with a
 * sinc^2 azimuth antenna pattern of length `antenna_m`, a linear range
 * response and FP64 geometry.  `range_offset` (nullable, float metres,
 * [nlines][refl_ld], device) lengthens each scatterer's range, e.g. by its
 * line-of-sight surface motion.  Atomic accumulation: not bit-reproducible.
 * No reference counterpart (the reference processes recorded data). */
int srg_forward_project_device(const srg_burst_desc *b, const float *refl,
                               int64_t refl_ld, const double *satvel,
                               double antenna_m, const float *range_offset, void *stream);

/* ---- Interferogram formation (replaces the crossmul program,
 * int/crossmul.f90:95-185, which SRG runs on pairs of .geo files) ----
 * Each line of both images (scaled by `scale`) is upsampled 2x across by
 * FFT (zero-padded to nnn = the first power of two >= na, spectrum halves
 * moved to the ends of a 2*nnn array, inverse FFT, / nnn / 2); the images are
 * cross-multiplied (slc1 * conj(slc2)) and their powers kept; pairs of
 * upsampled samples are summed, then `looksdn` lines down and `looksac`
 * samples across; the amplitude pair is square-rooted (|slc1|, |slc2|).  With
 * `mask` != 0 an output sample is zeroed when |sum of the unscaled input over
 * its look window| <= 1e-6 in either image (the reference's default 'y').
 * Inputs: [nlines][ld] complex64 (device); nlines plays the reference's
 * <valid_lines>.  Outputs: [nlines/looksdn][na/looksac] complex64 (device).
 * Enqueued on `stream`.  FFTs in FP32 (the reference uses FFTW in single
 * precision, so results agree to FP32 rounding, not bit for bit): for lines
 * of 2,049-4,096 samples (nnn = 4,096) kernels of the library's own that
 * transform each line in shared memory (and, with looksdn = 1, form the
 * pairs there too, with no scratch but read-only tables), otherwise cuFFT.
 * The device's scratch (upsampled images) is shared by every call on it:
 * calls on the same device whose GPU work overlaps (other streams) race,
 * except those that form the pairs in shared memory. */
int srg_crossmul_device(const float *slc1, const float *slc2, long long ld, int na, int nlines,
                        int looksac, int looksdn, float scale, int mask, float *igram,
                        float *amp, void *stream);
/* Sequential pairs (k, k+1), k = 0..n-2, of a stack of n images (device
 * pointer arrays on the host), each image transformed once; igrams[k] and
 * amps[k] receive pair k.  No reference counterpart (the reference runs the
 * crossmul program once per pair). */
int srg_crossmul_stack_device(const float *const *slcs, int n, long long ld, int na, int nlines,
                              int looksac, int looksdn, float scale, int mask,
                              float *const *igrams, float *const *amps, void *stream);

/* ---- Range compression (replaces the range loop of sentinel/processsub.f90:86-123) ----
 * The chirp replica of the decoded pulse parameters (processsub.f90:101-107:
 * t = (j-1)/samplefreq in FP32, phase = 2 pi startfreq t + pi ramprate t^2 in
 * FP64, each sample rounded to complex64 and divided by npts, npts =
 * int(pulselength * samplefreq) in FP32), written zero-padded to n complex
 * samples into `replica` (host); *npts_out receives npts. */
int srg_range_replica(float samplefreq, float startfreq, float ramprate, float pulselength,
                      float *replica, int n, int *npts_out);
/* Range-compress `nlines` decoded echo lines ([nlines][ld_in] complex64 on
 * the device, the 10-word line header already stripped, nsamps <= 32768
 * samples each): zero-pad to 32,768, forward FFT, times the conjugate of the
 * replica's 32,768-point spectrum, inverse FFT (unnormalised, as FFTW's), and
 * write the first nvalid = nsamps - npts samples of each line to `out`
 * ([nlines][ld_out] complex64, device; *nvalid_out receives nvalid).
 * Enqueued on `stream`.  Pulses of up to 4,096 samples: one fused kernel
 * forms those samples by overlap-save (8,192-point transforms in shared
 * memory; the same samples, the 32,768-point correlation never wrapping into
 * them); longer pulses: cuFFT.  FP32 throughout (the reference uses FFTW in
 * single precision: results agree to FP32 rounding, not bit for bit).  The
 * device's scratch (the filter spectrum of the last pulse parameters, the
 * padded line blocks of the cuFFT path) is shared by every call on it: calls
 * on the same device whose GPU work overlaps (other streams) race. */
int srg_range_compress_device(const float *lines, long long ld_in, int nlines, int nsamps,
                              float samplefreq, float startfreq, float ramprate,
                              float pulselength, float *out, long long ld_out, int *nvalid_out,
                              void *stream);

/* ---- Finer range lines (no reference counterpart: the reference
 * interpolates the original line linearly) ----
 * 2x oversampling of range lines for the backprojection's linear
 * interpolation: out[2i] = in[i]; out[2i+1] = 8-tap Hann-windowed sinc at the
 * half-sample point (taps from srg_oversample_taps, unit DC gain, FP32);
 * samples beyond the line read as 0.  in: [nlines][ld_in] complex64 with
 * nsamps samples, out: [nlines][ld_out] complex64 with 2*nsamps - 1 samples
 * (device).  A burst so oversampled is backprojected with S' = 2*nsamps - 1,
 * dmrg' = dmrg / 2 and the same rngstart and rngend. */
void srg_oversample_taps(float taps[4]);
int srg_oversample_range_device(const float *in, long long ld_in, int nlines, int nsamps,
                                float *out, long long ld_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SRG_BP_H */
