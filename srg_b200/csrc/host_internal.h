// host_internal.h -- host-side helpers shared by the C-ABI translation units
// of libsrg_bp.so (capi.cu, noalloc.cu).  Not part of the public ABI.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/srg_bp.h"
#include "kernels.h"

namespace srg {
namespace detail {

// Range bins of margin on each side of the drop-in's range band.
constexpr int kBandMargin = 8;

// Record a one-line error message for srg_last_error() and return `code`.
int fail(int code, const char *fmt, ...);

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return SRG_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max(bytes, (size_t)256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(SRG_E_NOMEM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        }
        cap = want;
        // New scratch starts at zero (flag words are read before any kernel
        // writes them).  The zeroing runs on the legacy stream, which the
        // library's non-blocking streams do not wait for: it must be finished
        // before the buffer is handed out, or a kernel on another stream could
        // write the buffer first and have it zeroed after (as when another
        // context's persistent kernel holds every SM and delays the zeroing).
        e = cudaMemset(p, 0, want);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(SRG_E_CUDA, "zeroing of new scratch failed: %s", cudaGetErrorString(e));
        }
        return SRG_OK;
    }
};

// Per-device scratch, reused by every call on that device.
struct DevCtx {
    int dev = -1;
    int sms = 0;
    std::mutex mu;
    DevBuf flags;     // [0] work counter, [1] error word, [2..3] term counter (u64)
    DevBuf bursts;    // BurstDev[]
    DevBuf tmaps;     // CUtensorMap[]
    DevBuf coef;      // doubles
    DevBuf tiles;     // work list of the backprojection (tile_list_bytes)
    DevBuf orbit;     // state vectors
    DevBuf in_burst, in_sat, in_dem, out;  // drop-in staging
    void *host_stage = nullptr;            // pinned host staging (drop-in entry)
    size_t host_cap = 0;
    // drop-in entry: its own streams (the burst upload overlaps the azimuth
    // centres), events of the row blocks copied back, a pinned error word
    static constexpr int kOutBlocks = 16;
    // flags words of the drop-in: [kBandWord, +1] first / last line of the kept
    // tiles, [kReadyWord] rows-uploaded word; host_flags[kReadyHost + k] holds
    // the value the copy stream writes after upload block k
    static constexpr int kBandWord = 4, kReadyWord = 6, kReadyHost = 8, kUploadBlocks = 8;
    // the range band of the drop-in's lines: device words [kRangeWord, +1],
    // their host copy host_flags[kRangeHost, +1]; bins of margin on each side
    static constexpr int kRangeWord = 8, kRangeHost = 2;
    // bytes the last drop-in call copied to and from the device
    long long last_h2d = 0, last_d2h = 0;
    // row blocks copied back while the sum still runs (gated kernel): device
    // words rb[k] stored-tile counts, rb[kRowBlocks + k] kept-tile counts,
    // rb[2 kRowBlocks] the order word, rb[3 kRowBlocks + k] done words;
    // host_rb[0 .. kRowBlocks] the kept counts and the order word, copied back
    // with the band, host_rb[2 kRowBlocks + k] the stored count read with
    // block k
    static constexpr int kRowBlocks = kOutBlocks;
    DevBuf rb;
    int *host_rb = nullptr;
    // drop-in call number on this device, 1 .. kSeqLimit (then it restarts)
    static constexpr int kSeqLimit = 1 << 24;
    int upload_seq = 0;
    bool dropin_ready = false;
    cudaStream_t s_main = nullptr, s_copy = nullptr, s_back = nullptr;
    cudaEvent_t ev_burst = nullptr, ev_flags = nullptr, ev_band = nullptr, ev_blk[kOutBlocks] = {};
    int *host_flags = nullptr;
    // kernel attributes set once per device (any entry, any host thread)
    std::mutex attrs_mu;
    bool attrs_done[64] = {};
    bool gated_attrs_done[8] = {};
};

// Per-device context (sets the device current).
int get_ctx(int device, DevCtx **out);
using StreamValueFn = CUresult (*)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
struct StreamValueOps {
    StreamValueFn wait = nullptr, write = nullptr;
};
StreamValueOps stream_value_ops();
// Streams, events and pinned error word of the drop-in entry (made once).
int ensure_dropin(DevCtx &c);
// Kernel entry for a form and shape index (-1: the default of that form).
const KernelEntry *pick_kernel(int form, int cfg);
int kernel_index(const KernelEntry *e);
void ensure_attrs(DevCtx &c, int idx);
int validate_desc(const srg_burst_desc &d);
BurstDev make_burst_dev(const srg_burst_desc &d, const double *coef);
// B.shear, B.tiles_x and B.tiles_y for the tiles of kernel `ke`.  shear:
// srg_bp_options::tile_shear; SRG_TILE_SHEAR_AUTO takes the shear that, by
// B's azimuth-centre slopes, leaves the fewest pixel-pulse slots per tile
// row.  Kernels with rectangular tiles get 0.  SRG_E_ARG for a shear out of
// range.
int set_tiles(BurstDev &B, const KernelEntry &ke, int shear);
// 0 and *out filled when a TMA descriptor can describe the burst, else -1.
int make_tmap(const BurstDev &B, int box_x, int box_y, CUtensorMap *out);
double ref_pi();
// |x - s_k|^2 is convex in the pulse index k for every pixel x that can have
// a term in range (the range band's bisection relies on it).
bool pulses_convex(const double *satloc, int P, double rngend);
// Every one of the n values is finite.
bool all_finite(const double *v, size_t n);

}  // namespace detail
}  // namespace srg
