// kernels.h -- host-visible launchers of the device kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "common.cuh"
#include "geom.cuh"

namespace srg {

// Scalars of the per-line azimuth-centre solve (azimuth_compress.cu:438-481).
struct CentreParams {
    double tmid, xm[3], vm[3], wvl, angc0, angc1, prf, pi;
};

// One burst's share of a batched azimuth-centre launch.
struct CentreJob {
    Orbit orbit;          // device state vectors
    CentreParams cp;
    double *coef;         // [nlines][3] output (device)
    int line_base;        // first global index of this burst's lines
    int pad;
};

struct KernelEntry {
    int form;
    TileShape shape;   // threads = block size
    int smem;          // dynamic shared memory bytes
    const void *fn;
    const char *name;  // template and shape, for reports
    int shears;        // 1: the kernel takes sheared tiles (BurstDev::shear)
};

extern const KernelEntry kKernels[];
extern const int kNumKernels;
extern const KernelEntry kGatedKernels[];
extern const int kNumGatedKernels;
// The twin of `e` that waits for range lines still uploading, or nullptr.
const KernelEntry *gated_twin(const KernelEntry &e);

// tile_list: the kept tiles from launch_tile_list (list[0] = count, list[1..]
// = tile indices); nullptr = every tile in [0, total).
cudaError_t launch_tiles(const KernelEntry &e, int grid, size_t smem, cudaStream_t st,
                         const BurstDev *bursts, int nb, int total, const CUtensorMap *tmaps,
                         int *counter, int *err, const int *tile_list = nullptr);

// Work list of the backprojection (kernels.cu: tile_mask_kernel): the tiles
// of tx x ty pixels that can hold a formed pixel, ascending, with the pixels
// of the dropped tiles zeroed.  Scratch layout: list [total + 1] ints,
// segment counts, mask [total] bytes.  band (optional, preset to
// {INT_MAX, -1}): lowered / raised to the first and last line of the kept
// tiles (lines relative to each burst's first line).
constexpr int kTileSegShift = 12;
constexpr int kTileSeg = 1 << kTileSegShift;
inline int *tile_list_segments(void *scratch, int total) {
    return static_cast<int *>(scratch) + total + 1;
}
inline unsigned char *tile_list_mask(void *scratch, int total) {
    return reinterpret_cast<unsigned char *>(tile_list_segments(scratch, total) +
                                             (total + kTileSeg - 1) / kTileSeg);
}
inline size_t tile_list_bytes(int total) {
    return sizeof(int) * ((size_t)total + 1 + (total + kTileSeg - 1) / kTileSeg) + (size_t)total;
}
cudaError_t launch_tile_list(const BurstDev *bursts, int nbursts, int max_burst_tiles, int total,
                             int tx, int ty, void *scratch, cudaStream_t st, int *band = nullptr);
cudaError_t launch_line_centres(const BurstDev &B, const Orbit &o, const CentreParams &cp,
                                double *coef, cudaStream_t st);
cudaError_t launch_line_centres_batch(const BurstDev *bursts, const CentreJob *jobs, int n,
                                      int total, cudaStream_t st);
// tile_mask (optional): the work-list mask of the backprojection that wrote the
// outputs, for tiles of tx x ty pixels (see merge_scene_kernel).
cudaError_t launch_merge_scene(const BurstDev *bursts, int n, float2 *dst, long long dst_ld,
                               int lines, int cols, cudaStream_t st,
                               const unsigned char *tile_mask = nullptr, int tx = 0, int ty = 0);
cudaError_t launch_count_terms(const BurstDev &B, unsigned long long *terms, int sms,
                               cudaStream_t st);
// Lowest and highest range bin (band[0], band[1], preset to INT_MAX / INT_MIN)
// that the terms of the burst's formed pixels can read, given R^2 convex in
// the pulse index (kernels.cu: range_band_kernel).
cudaError_t launch_range_band(const BurstDev &B, int *band, int sms, cudaStream_t st);
cudaError_t launch_merge(float2 *dst, long long dst_ld, const float2 *src, long long src_ld,
                         int rows, int cols, int sms, cudaStream_t st);
cudaError_t launch_pulse_orbit(const double *times, int P, const Orbit &o, double *pos,
                               double *vel, cudaStream_t st);
cudaError_t launch_forward_project(const BurstDev &B, const float2 *refl, long long refl_ld,
                                   const double *satvel, double antenna, const float *range_offset,
                                   cudaStream_t st);

cudaError_t launch_fma_peak(int fp64, int blocks, int iters, void *sink, cudaStream_t st);

inline int shared_bytes(const KernelEntry &e) { return e.smem; }

}  // namespace srg
