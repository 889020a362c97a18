// common.cuh -- device-side descriptors shared by the backprojection kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace srg {

// Default poll limit of the kernels' bounded waits (try_wait polls, each
// suspending up to ~1 us; a launch may set another through BurstDev::spin).
constexpr unsigned kSpinLimit = 1u << 22;

// Error bits raised by kernels into the device error word.
enum : int {
    ERR_TMA_TIMEOUT = 1,   // a bounded mbarrier wait for a TMA tile gave up
    ERR_BAD_BURST = 2,     // a work item referenced an inconsistent burst
    ERR_UPLOAD_TIMEOUT = 4,  // a bounded wait for range lines still in transfer gave up
};

// Everything a kernel needs about one burst, prepared on the host.  Field
// names follow the reference's (sentinel/azimuth_compress.cu).
struct BurstDev {
    const float2 *burst;      // [P][ldb] complex64: bins [bin0, bin0 + nbins) of each line
    const double *satloc;     // [P][3]
    const short *dem;         // row 0 = grid line firstline; stride dem_ld
    float2 *out;              // row 0 = grid line firstline; stride out_ld
    const double *coef;       // [nlines][3]
    long long ldb, dem_ld, out_ld;
    int P, S, W;
    int firstline, nlines, firstpix, lastpix;  // lastpix as the reference (may be W)
    int lastpix_eff;          // min(lastpix, W-1)
    int out_pix0;
    int aperture, ap2;        // ap2 = aperture / 2 (integer division, as the reference)
    int tiles_x, tiles_y, tile_base;
    // Lines per 32 columns by which the tiles are sheared (0: rectangular
    // tiles); see tile_dline.
    int shear;
    // Azimuth-centre slopes (pulses) and range slopes (bins) per grid line
    // and per column: host estimates from the geometry that choose the shear
    double slope_line, slope_col, rbin_line, rbin_col;
    int tmap;                 // index of this burst's TMA descriptor, -1 = none
    unsigned spin;            // polls of a bounded device-side wait (the launch's first burst's)
    // The lines held in device memory: logical range bins [bin0, bin0 + nbins)
    // of [0, S) (bin0 even; the whole line: 0 and S).  Bin b of pulse k is at
    // burst[k * ldb + b - bin0]; bins outside read as zero.
    int bin0, nbins;
    double firstlat, deltalat, firstlon, deltalon, deg2rad;
    double rngstart, rmax;    // rmax = rngend - dmrg (the reference's upper range test)
    double dmrg, k4pi;        // k4pi = 4*pi/wvl, grouped as the reference
    double K;                 // 2 / wvl: cycles of two-way phase per metre
    double inv_dmrg;
    float K_hi, K_lo;         // K as an unevaluated float sum
    float K_f, inv_dmrg_f;
    // Range lines still uploading (the drop-in entry): null, or a device word
    // that the copy stream raises to ready_base + n once the first
    // n * ready_rows pulse rows are in device memory.
    const int *ready;
    int ready_base, ready_rows;
    // Rows finished while the sum still runs (the drop-in entry): null, or per
    // row block of rb_tile_rows tile rows a count of stored tiles, the count of
    // kept tiles (the work list adds it up), and a word set to rb_seq once
    // the two agree; the work list also sets *rb_order to
    // lines_against_pulses (the order the blocks finish in).
    int *rb_count, *rb_expect, *rb_done, *rb_order;
    int rb_tile_rows, rb_seq;
};

// Largest tile shear, in lines per 32 columns.
constexpr int kMaxShear = 8;

// Tile geometry.  Tile ti of a burst (tiles_x per tile row) covers columns
// px0 + [0, tx), px0 = firstpix + (ti % tiles_x) * tx, and on its column
// px0 + x the lines ly0 + y + tile_dline(shear, x) - tile_dmax(shear, tx),
// y in [0, ty), with ly0 = (ti / tiles_x) * ty.  On every column the tile
// rows partition the lines; with the shear a tile's rows of pixels follow
// the lines of constant azimuth centre across the columns, so its pixels
// share more of their apertures.  Tile row r touches the lines
// [r ty - span, r ty + ty), span = tile_span(shear, tx) < ty.
__host__ __device__ __forceinline__ int tile_dline(int shear, int x) {
    const int v = shear * x;
    return v >= 0 ? v / 32 : -((31 - v) / 32);  // floor(shear * x / 32)
}
__host__ __device__ __forceinline__ int tile_dmax(int shear, int tx) {
    return shear > 0 ? tile_dline(shear, tx - 1) : 0;
}
__host__ __device__ __forceinline__ int tile_span(int shear, int tx) {
    return shear > 0 ? tile_dline(shear, tx - 1) : -tile_dline(shear, tx - 1);
}

// Grid lines run against the pulses (the azimuth centre of the last formed
// line precedes the first's): a burst's tiles are then taken from the last
// line back when its range lines arrive in pulse order.
__device__ __forceinline__ bool lines_against_pulses(const BurstDev &B) {
    return B.nlines >= 3 && B.coef[3 * (B.nlines - 2) + 2] < B.coef[2];
}

// Kernel shape of the tiled backprojection.
struct TileShape {
    int tx, ty, threads, chunk, window;
};

}  // namespace srg
