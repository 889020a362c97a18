// noalloc.cu -- srg_bp_burst_device_noalloc: one burst, no device allocation.
//
// Who needs it: callers that cannot call cudaMalloc -- a host process whose
// device memory is already reserved by a pool it does not own (a serving
// runtime or a framework allocator that holds the HBM and forbids raw
// allocations), or a latency-critical stream where the implicit
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.
// They pass the burst inputs and the output buffer; everything else the
// backprojection needs lives in `g_noalloc_scratch` below.
//
// The scratch is one file-scope device array of kScratchBytes, held by every
// GPU that loads this library until the process exits.  Its host-side name
// is only a stand-in: the device address is looked up once per device, with
// that device current, by cudaGetSymbolAddress and handed to the kernels.
// Every call shares the array and leaves its contents behind; the work
// counter and error word are cleared at the start of each call.  Calls whose
// GPU work overlaps (other streams, other host threads) race on it.
#include <cstring>
#include <mutex>
#include <vector>

#include "host_internal.h"

using namespace srg;
using namespace srg::detail;

namespace {

// Layout of the scratch (bytes).
constexpr int kMaxLines = SRG_NOALLOC_MAX_LINES;
constexpr int kMaxStateVec = SRG_NOALLOC_MAX_STATEVEC;
constexpr size_t kOffFlags = 0;        // int work counter, int error word
constexpr size_t kOffBurst = 256;      // BurstDev
constexpr size_t kOffTmap = 1024;      // CUtensorMap (64-byte aligned)
constexpr size_t kOffOrbit = 2048;     // [n] times, [n][3] positions, [n][3] velocities
constexpr size_t kOffCoef = kOffOrbit + 7 * sizeof(double) * kMaxStateVec;
constexpr size_t kScratchBytes = kOffCoef + 3 * sizeof(double) * kMaxLines;
static_assert(kScratchBytes == SRG_NOALLOC_SCRATCH_BYTES, "header and layout disagree");
static_assert(sizeof(BurstDev) <= kOffTmap - kOffBurst, "BurstDev outgrew its slot");
static_assert(kOffTmap % 64 == 0 && kOffCoef % 8 == 0, "alignment");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_addr_mu;
void *g_addr[64] = {};

// Device address of the scratch on the current device (looked up once).
int scratch_address(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> g(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(SRG_E_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        }
        g_addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_addr[dev]);
    return SRG_OK;
}

}  // namespace

extern "C" int srg_bp_burst_device_noalloc(const srg_burst_desc *b, const srg_bp_options *opts,
                                           void *stream) {
    if (!b) return fail(SRG_E_ARG, "null burst descriptor");
    int rc = validate_desc(*b);
    if (rc) return rc;
    if (b->nlines > kMaxLines)
        return fail(SRG_E_ARG, "no-alloc entry: burst has %d grid lines, the maximum is %d",
                    b->nlines, kMaxLines);
    if (!b->coef && b->numstatevec > kMaxStateVec)
        return fail(SRG_E_ARG, "no-alloc entry: %d state vectors, the maximum is %d",
                    b->numstatevec, kMaxStateVec);
    srg_bp_options o;
    srg_bp_default_options(&o);
    if (opts) o = *opts;
    if (o.centres_on_host && !b->coef)  // as srg_bp_bursts_device
        return fail(SRG_E_UNSUPPORTED, "host centres need host DEM (use the file entry)");
    const KernelEntry *ke = pick_kernel(o.form, o.tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", o.form, o.tile_cfg);
    DevCtx *c = nullptr;
    rc = get_ctx(o.device, &c);
    if (rc) return rc;
    unsigned char *scr = nullptr;
    rc = scratch_address(c->dev, &scr);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *flags = reinterpret_cast<int *>(scr + kOffFlags);
    BurstDev *d_burst = reinterpret_cast<BurstDev *>(scr + kOffBurst);
    CUtensorMap *d_tmap = reinterpret_cast<CUtensorMap *>(scr + kOffTmap);
    double *d_orbit = reinterpret_cast<double *>(scr + kOffOrbit);
    double *d_coef = reinterpret_cast<double *>(scr + kOffCoef);

#define NA_CK(call)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) return fail(SRG_E_CUDA, "%s failed: %s", #call,              \
                                           cudaGetErrorString(e_));                         \
    } while (0)

    // counter and error word must start at zero; the rest is overwritten
    NA_CK(cudaMemsetAsync(flags, 0, 2 * sizeof(int), st));
    const double *coef = b->coef;
    if (!coef) {
        const int n = b->numstatevec;
        double host[7 * kMaxStateVec];
        std::memcpy(host, b->timeorbit, sizeof(double) * n);
        std::memcpy(host + n, b->xx, sizeof(double) * 3 * n);
        std::memcpy(host + 4 * n, b->vv, sizeof(double) * 3 * n);
        // pageable source: staged before cudaMemcpyAsync returns
        NA_CK(cudaMemcpyAsync(d_orbit, host, sizeof(double) * 7 * n, cudaMemcpyHostToDevice, st));
        Orbit orb{d_orbit, d_orbit + n, d_orbit + 4 * n, n};
        CentreParams cp{};
        cp.tmid = b->tmid;
        for (int i = 0; i < 3; ++i) {
            cp.xm[i] = b->xyz_mid[i];
            cp.vm[i] = b->vel_mid[i];
        }
        cp.wvl = b->wvl;
        cp.angc0 = b->angc0;
        cp.angc1 = b->angc1;
        cp.prf = b->prf;
        cp.pi = ref_pi();
        NA_CK(launch_line_centres(make_burst_dev(*b, d_coef), orb, cp, d_coef, st));
        coef = d_coef;
    }
    BurstDev B = make_burst_dev(*b, coef);
    if (o.spin_limit > 0) B.spin = (unsigned)o.spin_limit;
    if ((rc = set_tiles(B, *ke, o.tile_shear))) return rc;
    B.tile_base = 0;
    const int total = B.tiles_x * B.tiles_y;
    CUtensorMap tm;
    std::memset(&tm, 0, sizeof tm);
    if (make_tmap(B, ke->shape.window, ke->shape.chunk, &tm) == 0) B.tmap = 0;
    NA_CK(cudaMemcpyAsync(d_burst, &B, sizeof B, cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(d_tmap, &tm, sizeof tm, cudaMemcpyHostToDevice, st));
    if (total > 0) {
        const int idx = kernel_index(ke);
        ensure_attrs(*c, idx);
        const int smem = shared_bytes(*ke);
        int per_sm = 0;
        NA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ke->fn, ke->shape.threads, smem));
        if (per_sm < 1) return fail(SRG_E_UNSUPPORTED, "kernel shape %d does not fit an SM", idx);
        NA_CK(launch_tiles(*ke, std::min(total, per_sm * c->sms), smem, st, d_burst, 1, total, d_tmap,
                           flags, flags + 1));
    }
    int h[2] = {0, 0};
    NA_CK(cudaMemcpyAsync(h, flags, sizeof h, cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
#undef NA_CK
    if (h[1]) return fail(SRG_E_TIMEOUT, "device error word 0x%x (TMA wait timed out)", h[1]);
    return SRG_OK;
}
