// capi.cu -- the C ABI of libsrg_bp.so (declared in include/srg_bp.h).
//
// Host orchestration of one burst mirrors sentinel/azimuth_compress.cu:
// line/pixel limits from latlons (295-301, 378-379), DEM slab read from the
// caller's descriptor (399-408), per-line azimuth centres (438-481), the
// per-pixel sum (500), and the read-modify-write merge of the output rows
// into the .geo raster (510-537).  Differences: every CUDA call is checked
// and reported; device scratch is cached per device and reused across calls
// instead of being allocated and freed on every burst; only the pixel box
// [firstpix, min(lastpix, W-1)] of the DEM rows is read (the only columns the
// sum touches) and only that box of the output rows is merged, row by row with
// pread/pwrite on the descriptors (instead of an fdopen() stream that is never
// flushed or closed), by a persistent pool of host threads; the DEM read and
// the azimuth centres overlap the upload of the burst, and the merge of each
// block of rows starts as soon as that block is copied back.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <unistd.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/srg_bp.h"
#include "host_internal.h"
#include "host_pool.h"
#include "kernels.h"

using namespace srg;

namespace srg {
namespace detail {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(SRG_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

// SRG_DROPIN_OVERLAP=1 in the environment: drop-in calls overlap by default
int env_overlap() {
    static const int v = [] {
        const char *e = std::getenv("SRG_DROPIN_OVERLAP");
        return e && e[0] == '1' ? 1 : 0;
    }();
    return v;
}
srg_bp_options g_default_opts = {SRG_FORM_SPLIT, -1, -1, 0, 0, 0, 0, 0, env_overlap(), 0};
std::mutex g_opts_mu;

DevCtx g_ctx[64];
std::mutex g_ctx_mu;

int get_ctx(int device, DevCtx **out) {
    int dev = device;
    if (dev < 0) CK(cudaGetDevice(&dev));
    if (dev >= 64) return fail(SRG_E_ARG, "device ordinal %d out of range", dev);
    CK(cudaSetDevice(dev));
    std::lock_guard<std::mutex> g(g_ctx_mu);
    DevCtx &c = g_ctx[dev];
    if (c.dev < 0) {
        CK(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
        c.dev = dev;
    }
    *out = &c;
    return SRG_OK;
}

// Drop-in contexts of a device: two, used in turn by overlapped calls (a
// call's tail still holds its context while the next call fills the other),
// and the worker thread that runs the overlapped calls' tails in call order.
struct DropinDev {
    std::mutex call_mu;  // one drop-in call at a time on the device
    DevCtx slot[2];
    int next = 0;
    std::mutex q_mu;
    std::condition_variable q_cv;
    std::deque<std::function<void()>> q;
    bool busy[2] = {false, false};  // a queued or running tail holds the slot
    bool worker = false;
    int pending_rc = SRG_OK;  // first failure of a tail not yet returned
    std::string pending_err;
    long long last_h2d = 0, last_d2h = 0;
};
// Never destroyed: the worker threads wait on these at exit (destroying a
// condition variable with a waiter blocks the exit).
DropinDev *const g_dropin = new DropinDev[64];
std::mutex g_dropin_mu;

int get_dropin(int device, DropinDev **out) {
    int dev = device;
    if (dev < 0) CK(cudaGetDevice(&dev));
    if (dev >= 64) return fail(SRG_E_ARG, "device ordinal %d out of range", dev);
    CK(cudaSetDevice(dev));
    std::lock_guard<std::mutex> g(g_dropin_mu);
    DropinDev &d = g_dropin[dev];
    for (DevCtx &c : d.slot) {
        if (c.dev < 0) {
            CK(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
            c.dev = dev;
        }
    }
    *out = &d;
    return SRG_OK;
}

// Waits until no tail is queued or running on the device.
void dropin_wait_idle(DropinDev &d) {
    std::unique_lock<std::mutex> lk(d.q_mu);
    d.q_cv.wait(lk, [&] { return d.q.empty() && !d.busy[0] && !d.busy[1]; });
}

// The first failure of an overlapped call's tail not yet returned (cleared).
int dropin_take_pending(DropinDev &d) {
    std::lock_guard<std::mutex> lk(d.q_mu);
    const int rc = d.pending_rc;
    if (rc) {
        g_err = d.pending_err;
        d.pending_rc = SRG_OK;
        d.pending_err.clear();
    }
    return rc;
}

void dropin_flush_all();

// Queues an overlapped call's tail for the device's worker thread (started
// on first use), which runs the tails one after the other; false, with
// nothing queued, when the worker cannot be started.
bool dropin_enqueue(DropinDev &d, int slot, std::function<void()> job) {
    static std::once_flag at_exit;
    std::call_once(at_exit, [] { std::atexit(dropin_flush_all); });
    std::lock_guard<std::mutex> lk(d.q_mu);
    if (!d.worker) {
        try {
            std::thread([&d] {
                for (;;) {
                    std::function<void()> f;
                    {
                        std::unique_lock<std::mutex> lk2(d.q_mu);
                        d.q_cv.wait(lk2, [&] { return !d.q.empty(); });
                        f = std::move(d.q.front());
                    }
                    f();  // the entry stays queued while it runs
                    {
                        std::lock_guard<std::mutex> g(d.q_mu);
                        d.q.pop_front();
                    }
                    d.q_cv.notify_all();
                }
            }).detach();
        } catch (...) {
            return false;
        }
        d.worker = true;
    }
    d.busy[slot] = true;
    d.q.push_back([&d, slot, job = std::move(job)] {
        job();
        std::lock_guard<std::mutex> g(d.q_mu);
        d.busy[slot] = false;
    });
    d.q_cv.notify_all();
    return true;
}

void dropin_flush_all() {
    for (int i = 0; i < 64; ++i) {
        DropinDev &d = g_dropin[i];
        bool started;
        {
            std::lock_guard<std::mutex> lk(d.q_mu);
            started = d.worker;
        }
        if (started) dropin_wait_idle(d);
    }
}

// A row block of a drop-in call's output box.
struct OutBlock {
    int r0, r1;  // rows [r0, r1) of the box
    int rb;      // row block whose stored count came back with it, or -1
};

// What the end of a drop-in call needs once its copies back are queued.
struct DropinTail {
    OutBlock blk[DevCtx::kOutBlocks];
    int nblk = 0, ntask = 1, ncols = 0, fl = 0, W = 0, fp_eff = 0, fdout = -1;
    bool overlapped = false;  // runs behind the caller (worker thread)
};

// The end of a drop-in call: each row block of the output box is merged into
// the .geo rows as soon as it is back (azimuth_compress.cu:510-537; pixels
// outside the box are never replaced, so only the box is read and written);
// then the call's streams are waited for and its status reported.
int dropin_tail(DevCtx *c, const DropinTail &t) {
    constexpr int K = DevCtx::kRowBlocks;
    cudaStream_t st = c->s_main;
    const float *win = static_cast<const float *>(c->host_stage);
    HostPool &pool = HostPool::get();
    std::atomic<int> cuda_err{0}, io_err{0};
    const int ncols = t.ncols;
    // merge rows [r0, r1) of the box (azimuth_compress.cu:510-537)
    auto merge_rows = [&](int r0, int r1) {
        std::vector<float> cur(2 * (size_t)ncols);
        auto replaced = [](const float *v) { return std::fabs((double)v[0]) > 1.e-18; };
        for (int r = r0; r < r1; ++r) {
            // only the span [i0, i1] of replaced pixels is read and written back
            // (most rows of a burst's box have none: they are left untouched)
            const float *o2 = win + 2 * (size_t)r * ncols;
            int i0 = 0;
            while (i0 < ncols && !replaced(o2 + 2 * i0)) ++i0;
            if (i0 == ncols) continue;
            int i1 = ncols - 1;
            while (!replaced(o2 + 2 * i1)) --i1;
            const ssize_t want = (ssize_t)(i1 - i0 + 1) * 8;
            const off_t off = ((off_t)(t.fl + r) * t.W + t.fp_eff + i0) * 8;
            const ssize_t got = pread(t.fdout, cur.data(), want, off);
            if (got < 0) {
                io_err = 1;
                return;
            }
            if (got < want) std::memset(reinterpret_cast<char *>(cur.data()) + got, 0, want - got);
            for (int i = i0; i <= i1; ++i) {
                if (replaced(o2 + 2 * i)) {
                    cur[2 * (i - i0)] = o2[2 * i];
                    cur[2 * (i - i0) + 1] = o2[2 * i + 1];
                }
            }
            if (pwrite(t.fdout, cur.data(), want, off) != want) {
                io_err = 2;
                return;
            }
        }
    };
    // a block is merged once it is back: a row block that came back with
    // every kept tile stored at once; any other block after the kernel's end,
    // and only with the error word clear
    auto mergeable = [&](int k) {
        if (cudaEventSynchronize(c->ev_blk[k]) != cudaSuccess) return false;
        const bool whole = t.blk[k].rb >= 0 && c->host_rb[2 * K + t.blk[k].rb] == c->host_rb[t.blk[k].rb];
        return whole || (cudaEventSynchronize(c->ev_flags) == cudaSuccess && !c->host_flags[1]);
    };
    if (!t.overlapped) {
        // every block's tasks at once on the pool, each waiting for its block
        const int per_blk = std::max(1, t.ntask / std::max(t.nblk, 1));
        if (t.nblk > 0) pool.run(t.nblk * per_blk, [&](int task) {
            const int k = task / per_blk, part = task % per_blk;
            if (!mergeable(k)) {
                cuda_err = 1;
                return;
            }
            const int b0 = t.blk[k].r0, b1 = t.blk[k].r1;
            merge_rows(b0 + (int)((long long)(b1 - b0) * part / per_blk),
                       b0 + (int)((long long)(b1 - b0) * (part + 1) / per_blk));
        });
    } else {
        // Overlapped calls: the blocks are waited for here, in the order they
        // come back, and only the merge of a block that is back goes to the
        // pool, so no pool thread waits on the device while the next call's
        // DEM read needs the pool.
        for (int k = 0; k < t.nblk; ++k) {
            if (!mergeable(k)) {
                cuda_err = 1;
                continue;
            }
            const int b0 = t.blk[k].r0, b1 = t.blk[k].r1;
            const int parts = std::max(1, std::min(b1 - b0, std::max(1, t.ntask / 4)));
            pool.run(parts, [&](int part) {
                merge_rows(b0 + (int)((long long)(b1 - b0) * part / parts),
                           b0 + (int)((long long)(b1 - b0) * (part + 1) / parts));
            });
        }
    }
    // the upload may end after the last chunk that needed it: the caller's
    // buffer stays in use until then
    const cudaError_t e1 = cudaStreamSynchronize(st), e2 = cudaStreamSynchronize(c->s_copy),
                      e3 = cudaStreamSynchronize(c->s_back);
    const cudaError_t e = e1 ? e1 : e2 ? e2 : e3 ? e3 : cudaGetLastError();
    if (e != cudaSuccess) return fail(SRG_E_CUDA, "drop-in streams: %s", cudaGetErrorString(e));
    if (c->host_flags[1]) {  // only row blocks whose every tile was stored were merged
        const int word = c->host_flags[1];
        cudaMemsetAsync(static_cast<int *>(c->flags.p) + 1, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return fail(SRG_E_TIMEOUT, "device error word 0x%x (a bounded device wait gave up)", word);
    }
    if (cuda_err) return fail(SRG_E_CUDA, "copy of the output box failed");
    if (io_err == 1) return fail(SRG_E_IO, "output read failed (fd %d)", t.fdout);
    if (io_err == 2) return fail(SRG_E_IO, "output write failed (fd %d)", t.fdout);
    return SRG_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// Stream memory operations of the driver API (a stream waits for, or writes,
// a 32-bit device word), or nulls where the driver offers none.
StreamValueOps stream_value_ops() {
    static StreamValueOps ops;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q1, q2;
        void *w = nullptr, *r = nullptr;
        if (cudaGetDriverEntryPoint("cuStreamWaitValue32", &w, cudaEnableDefault, &q1) ==
                cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuStreamWriteValue32", &r, cudaEnableDefault, &q2) ==
                cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            ops.wait = reinterpret_cast<StreamValueFn>(w);
            ops.write = reinterpret_cast<StreamValueFn>(r);
        } else {
            cudaGetLastError();
        }
    });
    return ops;
}

// Kernel entry for a form and shape index (-1: the default of that form).
const KernelEntry *pick_kernel(int form, int cfg) {
    if (cfg >= 0) {
        if (cfg >= kNumKernels || kKernels[cfg].form != form) return nullptr;
        return &kKernels[cfg];
    }
    for (int i = 0; i < kNumKernels; ++i)
        if (kKernels[i].form == form) return &kKernels[i];
    return nullptr;
}

// Reference line/pixel limits (azimuth_compress.cu:295-301, 378-379).
void ref_limits(const double *latlons, double firstlat, double deltalat, double firstlon,
                double deltalon, int W, int L, int *fl, int *ll, int *fp, int *lp) {
    int lastline = (int)((latlons[0] - firstlat) / deltalat);
    int firstline = (int)((latlons[1] - firstlat) / deltalat);
    if (firstline < 0) firstline = 0;
    if (lastline < 0) lastline = 0;
    if (firstline > L - 1) firstline = L - 1;
    if (lastline > L - 1) lastline = L - 1;
    int firstpix = (int)((latlons[2] - firstlon) / deltalon);
    if (firstpix < 0) firstpix = 0;
    int lastpix = (int)((latlons[3] - firstlon) / deltalon);
    if (lastpix > W) lastpix = W;
    *fl = firstline;
    *ll = lastline;
    *fp = firstpix;
    *lp = lastpix;
}

double ref_pi() { return 4.0 * atan2(1.0, 1.0); }

// R_k^2 = |x - s_k|^2 has the second difference
//   |ds_k|^2 + |ds_{k-1}|^2 - 2 (x - s_k) . d2s_k
// (ds_k = s_{k+1} - s_k, d2s_k = s_{k+1} - 2 s_k + s_{k-1}), positive at every
// pulse for every point x within rbound of it when
// |ds_k|^2 + |ds_{k-1}|^2 > 2 rbound |d2s_k|.  A pixel with a term in range
// lies within rngend of that term's pulse, so within rngend + the track's
// length of every pulse of its window; the test takes twice that bound.  On
// an orbit the left side is ~40 m^2 and the right ~10 m^2.
bool pulses_convex(const double *s, int P, double rngend) {
    if (P < 3) return true;
    double track = 0.0;
    for (int k = 0; k + 1 < P; ++k) {
        const double a = s[3 * k + 3] - s[3 * k], b = s[3 * k + 4] - s[3 * k + 1],
                     c = s[3 * k + 5] - s[3 * k + 2];
        track += std::sqrt(a * a + b * b + c * c);
    }
    const double rbound = std::fabs(rngend) + track;
    for (int k = 1; k + 1 < P; ++k) {
        double n1 = 0.0, n0 = 0.0, n2 = 0.0;
        for (int q = 0; q < 3; ++q) {
            const double d1 = s[3 * (k + 1) + q] - s[3 * k + q];
            const double d0 = s[3 * k + q] - s[3 * (k - 1) + q];
            const double d2 = d1 - d0;
            n1 += d1 * d1;
            n0 += d0 * d0;
            n2 += d2 * d2;
        }
        if (!(n1 + n0 > 4.0 * rbound * std::sqrt(n2))) return false;
    }
    return true;
}

bool all_finite(const double *v, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

int validate_desc(const srg_burst_desc &d) {
    if (!d.burst || !d.satloc || !d.dem || !d.out)
        return fail(SRG_E_ARG, "null device pointer in burst descriptor");
    const int nbins = d.nbins > 0 ? d.nbins : d.S;
    if (d.P < 1 || d.S < 2 || d.ldb < nbins || d.demwidth < 1 || d.nlines < 1)
        return fail(SRG_E_ARG, "bad sizes: P=%d S=%d ldb=%lld nbins=%d W=%d nlines=%d", d.P, d.S,
                    (long long)d.ldb, nbins, d.demwidth, d.nlines);
    if (d.bin0 < 0 || (d.bin0 & 1) || d.nbins < 0 || (long long)d.bin0 + nbins > d.S)
        return fail(SRG_E_ARG, "bad bin window bin0=%d nbins=%d of S=%d (bin0 even)", d.bin0,
                    d.nbins, d.S);
    if (d.P > 100000000 || d.S > (1 << 28))
        return fail(SRG_E_ARG, "burst too large: P=%d S=%d", d.P, d.S);
    if (!(d.dmrg > 0) || !(d.wvl > 0) || d.aperture < 0)
        return fail(SRG_E_ARG, "bad radar scalars: dmrg=%g wvl=%g aperture=%d", d.dmrg, d.wvl,
                    d.aperture);
    if (!d.coef && (!d.timeorbit || !d.xx || !d.vv || d.numstatevec < 4))
        return fail(SRG_E_ARG, "no coef and no orbit (numstatevec=%d, need >= 4)", d.numstatevec);
    if (d.firstpix < 0 || d.out_pix0 > d.firstpix)
        return fail(SRG_E_ARG, "bad pixel window firstpix=%d out_pix0=%d", d.firstpix, d.out_pix0);
    return SRG_OK;
}

// Azimuth-centre and range slopes of a burst per grid line and per column,
// at the grid's centre at height 0 on the WGS-84 ellipsoid: a ground step dx
// moves a point's time of closest approach by about (v . dx) / |v|^2
// (mid-burst velocity v), and its range by about e . dx (e the unit vector
// from the mid-burst position).  Zero without a velocity, position and PRF (a
// caller that passes its own azimuth centres need not give them).
static void centre_slopes(const srg_burst_desc &d, BurstDev &B) {
    B.slope_line = B.slope_col = B.rbin_line = B.rbin_col = 0.0;
    const double *v = d.vel_mid, *s = d.xyz_mid;
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (!(vv > 0.0) || !std::isfinite(vv) || !(d.prf > 0.0) || !std::isfinite(d.prf) ||
        !(d.dmrg > 0.0))
        return;
    auto ecef = [](double lat_deg, double lon_deg, double x[3]) {
        const double a = 6378137.0, e2 = 0.0066943799901499996, r = M_PI / 180.0;
        const double sl = std::sin(lat_deg * r), cl = std::cos(lat_deg * r);
        const double n = a / std::sqrt(1.0 - e2 * sl * sl);
        x[0] = n * cl * std::cos(lon_deg * r);
        x[1] = n * cl * std::sin(lon_deg * r);
        x[2] = n * (1.0 - e2) * sl;
    };
    const double lat = d.firstlat + (d.firstline + 0.5 * d.nlines) * d.deltalat;
    const double lon = d.firstlon + 0.5 * (d.firstpix + d.lastpix) * d.deltalon;
    double p0[3], pl[3], pc[3];
    ecef(lat, lon, p0);
    ecef(lat + d.deltalat, lon, pl);
    ecef(lat, lon + d.deltalon, pc);
    auto dot = [](const double *a, const double *p, const double *q) {
        return a[0] * (p[0] - q[0]) + a[1] * (p[1] - q[1]) + a[2] * (p[2] - q[2]);
    };
    const double k = d.prf / vv;
    const double r = std::sqrt((p0[0] - s[0]) * (p0[0] - s[0]) + (p0[1] - s[1]) * (p0[1] - s[1]) +
                               (p0[2] - s[2]) * (p0[2] - s[2]));
    const double e[3] = {(p0[0] - s[0]) / r, (p0[1] - s[1]) / r, (p0[2] - s[2]) / r};
    const double sl = k * dot(v, pl, p0), sc = k * dot(v, pc, p0);
    const double rl = dot(e, pl, p0) / d.dmrg, rc = dot(e, pc, p0) / d.dmrg;
    if (std::isfinite(sl) && std::isfinite(sc) && std::isfinite(rl) && std::isfinite(rc)) {
        B.slope_line = sl;
        B.slope_col = sc;
        B.rbin_line = rl;
        B.rbin_col = rc;
    }
}

BurstDev make_burst_dev(const srg_burst_desc &d, const double *coef) {
    BurstDev B{};
    B.burst = reinterpret_cast<const float2 *>(d.burst);
    B.satloc = d.satloc;
    B.dem = reinterpret_cast<const short *>(d.dem);
    B.out = reinterpret_cast<float2 *>(d.out);
    B.coef = coef;
    B.ldb = d.ldb;
    B.bin0 = d.bin0;
    B.nbins = d.nbins > 0 ? d.nbins : d.S;
    B.dem_ld = d.dem_ld;
    B.out_ld = d.out_ld;
    B.P = d.P;
    B.S = d.S;
    B.W = d.demwidth;
    B.firstline = d.firstline;
    B.nlines = d.nlines;
    B.firstpix = d.firstpix;
    B.lastpix = d.lastpix;
    B.lastpix_eff = std::min(d.lastpix, d.demwidth - 1);
    B.out_pix0 = d.out_pix0;
    B.aperture = d.aperture;
    B.ap2 = d.aperture / 2;
    B.tmap = -1;
    B.spin = kSpinLimit;
    const double pi = ref_pi();
    B.firstlat = d.firstlat;
    B.deltalat = d.deltalat;
    B.firstlon = d.firstlon;
    B.deltalon = d.deltalon;
    B.deg2rad = pi / 180.;
    B.rngstart = d.rngstart;
    B.rmax = d.rngend - d.dmrg;
    B.dmrg = d.dmrg;
    B.k4pi = 4. * pi / d.wvl;
    B.K = 2.0 / d.wvl;
    B.inv_dmrg = 1.0 / d.dmrg;
    B.K_hi = (float)B.K;
    B.K_lo = (float)(B.K - (double)B.K_hi);
    B.K_f = B.K_hi;
    B.inv_dmrg_f = (float)B.inv_dmrg;
    centre_slopes(d, B);
    return B;
}

int set_tiles(BurstDev &B, const KernelEntry &ke, int shear) {
    static_assert(kMaxShear == SRG_MAX_TILE_SHEAR, "shear limit");
    const int tx = ke.shape.tx, ty = ke.shape.ty;
    if (shear != SRG_TILE_SHEAR_AUTO &&
        (shear < -kMaxShear || shear > kMaxShear || tile_span(shear, tx) >= ty))
        return fail(SRG_E_ARG, "tile_shear %d: outside [-%d, %d] or a line offset of %d over a "
                    "tile of %d x %d", shear, kMaxShear, kMaxShear, tile_span(shear, tx), tx, ty);
    const int nx = B.lastpix_eff - B.firstpix + 1;
    int best = 0;
    if (ke.shears && shear != SRG_TILE_SHEAR_AUTO) {
        best = shear;
    } else if (ke.shears && nx > 0 && B.nlines > 0) {
        // A tile's pixels span aperture + spread pulses, the spread of their
        // azimuth centres; its tile rows need span more lines.  A shear of s
        // lines per 32 columns turns the per-column slopes by s / 32 of the
        // per-line ones.  Shears that widen a tile's range-bin window by more
        // than kShearBins are passed over (the staged window is fixed).
        constexpr double kShearBins = 8.0;
        auto slots = [&](int s) {
            const double spread = std::fabs(B.slope_col + s / 32.0 * B.slope_line) * (tx - 1) +
                                  std::fabs(B.slope_line) * (ty - 1);
            return (B.aperture + spread) * (double)(B.nlines + tile_span(s, tx));
        };
        auto bins = [&](int s) { return std::fabs(B.rbin_col + s / 32.0 * B.rbin_line) * (tx - 1); };
        double least = slots(0);
        for (int m = 1; m <= kMaxShear; ++m) {
            for (const int s : {-m, m}) {
                if (tile_span(s, tx) >= ty || bins(s) > bins(0) + kShearBins) continue;
                const double v = slots(s);
                if (v < least * (1.0 - 1e-9)) {
                    least = v;
                    best = s;
                }
            }
        }
    }
    B.shear = best;
    B.tiles_x = nx > 0 ? (nx + tx - 1) / tx : 0;
    B.tiles_y = B.nlines > 0 ? (B.nlines + tile_span(best, tx) + ty - 1) / ty : 0;
    return SRG_OK;
}

int make_tmap(const BurstDev &B, int box_x, int box_y, CUtensorMap *out) {
    auto enc = get_encode();
    if (!enc) return -1;
    const uintptr_t base = reinterpret_cast<uintptr_t>(B.burst);
    if ((base & 15) || ((B.ldb * 8) & 15) || (box_x & 1) || (B.bin0 & 1)) return -1;
    cuuint64_t dims[2] = {(cuuint64_t)B.nbins, (cuuint64_t)B.P};
    cuuint64_t strides[1] = {(cuuint64_t)(B.ldb * 8)};
    cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_y};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, (void *)B.burst, dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

// Device line centres for one descriptor into `coef` (device).
int centres_device(DevCtx &c, const srg_burst_desc &d, const BurstDev &B, double *coef,
                   cudaStream_t st) {
    const int n = d.numstatevec;
    int rc = c.orbit.ensure(sizeof(double) * 7 * (size_t)n);
    if (rc) return rc;
    double *ob = static_cast<double *>(c.orbit.p);
    std::vector<double> host(7 * (size_t)n);
    std::memcpy(host.data(), d.timeorbit, sizeof(double) * n);
    std::memcpy(host.data() + n, d.xx, sizeof(double) * 3 * n);
    std::memcpy(host.data() + 4 * n, d.vv, sizeof(double) * 3 * n);
    CK(cudaMemcpyAsync(ob, host.data(), sizeof(double) * 7 * n, cudaMemcpyHostToDevice, st));
    Orbit o{ob, ob + n, ob + 4 * n, n};
    CentreParams cp{};
    cp.tmid = d.tmid;
    for (int i = 0; i < 3; ++i) {
        cp.xm[i] = d.xyz_mid[i];
        cp.vm[i] = d.vel_mid[i];
    }
    cp.wvl = d.wvl;
    cp.angc0 = d.angc0;
    cp.angc1 = d.angc1;
    cp.prf = d.prf;
    cp.pi = ref_pi();
    // a pageable source is staged before cudaMemcpyAsync returns, so `host`
    // may go out of scope now
    CK(launch_line_centres(B, o, cp, coef, st));
    return SRG_OK;
}

void ensure_attrs(DevCtx &c, int idx) {
    std::lock_guard<std::mutex> g(c.attrs_mu);
    if (c.attrs_done[idx]) return;
    const KernelEntry &e = kKernels[idx];
    cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, shared_bytes(e));
    c.attrs_done[idx] = true;
}

int ensure_gated_attrs(DevCtx &c, const KernelEntry &twin) {
    std::lock_guard<std::mutex> g(c.attrs_mu);
    const int i = (int)(&twin - kGatedKernels);
    if (c.gated_attrs_done[i]) return SRG_OK;
    CK(cudaFuncSetAttribute(twin.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            shared_bytes(twin)));
    c.gated_attrs_done[i] = true;
    return SRG_OK;
}

int kernel_index(const KernelEntry *e) { return (int)(e - kKernels); }

int ensure_dropin(DevCtx &c) {
    if (c.dropin_ready) return SRG_OK;
    CK(cudaStreamCreateWithFlags(&c.s_main, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c.s_copy, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c.ev_burst, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ev_flags, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ev_band, cudaEventDisableTiming));
    for (int i = 0; i < DevCtx::kOutBlocks; ++i)
        CK(cudaEventCreateWithFlags(&c.ev_blk[i], cudaEventDisableTiming));
    if (cudaMallocHost(&c.host_flags, 64) != cudaSuccess) {
        cudaGetLastError();
        return fail(SRG_E_NOMEM, "pinned error word allocation failed");
    }
    CK(cudaStreamCreateWithFlags(&c.s_back, cudaStreamNonBlocking));
    if (cudaMallocHost(&c.host_rb, 4 * DevCtx::kRowBlocks * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return fail(SRG_E_NOMEM, "pinned row-block words allocation failed");
    }
    int rc = c.rb.ensure(4 * DevCtx::kRowBlocks * sizeof(int));  // zeroed
    if (rc) return rc;
    c.dropin_ready = true;
    return SRG_OK;
}

}  // namespace detail
}  // namespace srg

using namespace srg::detail;

namespace {

// Copy of n bytes whose stores bypass the CPU caches (16-byte streaming
// stores where the target is aligned; plain bytes at the two ends).  The
// stores are ordered against later ones only after store_fence().
void copy_nontemporal(char *dst, const char *src, size_t n) {
#if defined(__x86_64__)
    size_t i = 0;
    const size_t head = std::min(n, (16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15);
    for (; i < head; ++i) dst[i] = src[i];
    for (; i + 16 <= n; i += 16)
        _mm_stream_si128(reinterpret_cast<__m128i *>(dst + i),
                         _mm_loadu_si128(reinterpret_cast<const __m128i *>(src + i)));
    for (; i < n; ++i) dst[i] = src[i];
#else
    std::memcpy(dst, src, n);
#endif
}

void store_fence() {
#if defined(__x86_64__)
    _mm_sfence();
#endif
}

// Range lines that are still being copied in granules of `rows` pulse rows:
// the copy stream raises `*word` to base + n once the first n granules are in.
struct UploadGate {
    const int *word;
    int base, rows;
    // row blocks finished while the sum runs (null: none): the DevCtx::rb
    // words, tile rows per block, the value of a finished block's word, and
    // the pinned copy of the kept counts and the order word
    int *rb = nullptr;
    int rb_tile_rows = 0, rb_seq = 0;
    int *rb_host = nullptr;
};

// Core: launch the tiled kernel over n prepared bursts.
// Azimuth centres (for descriptors without them) and one backprojection
// launch over `descs` on `st`; with `before_sum` the launch also waits for
// that event (the azimuth centres need no range lines, so they may overlap
// the upload the event marks).  With `gate` (one burst) and a shape that has
// a gated twin (kGatedKernels), the twin starts at once and its producer waits
// for each chunk's rows instead; other shapes still wait for `before_sum`.
// `band` (optional): see launch_tile_list; with `band_host` the two words are
// also copied there right after the work list and `band_ready` is recorded,
// ahead of the backprojection.
int run_bursts(DevCtx &c, const srg_burst_desc *descs, int n, const srg_bp_options &o,
               cudaStream_t st, cudaEvent_t before_sum = nullptr,
               const UploadGate *gate = nullptr, int *band = nullptr, int *band_host = nullptr,
               cudaEvent_t band_ready = nullptr) {
    const KernelEntry *ke = pick_kernel(o.form, o.tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", o.form, o.tile_cfg);
    const KernelEntry *twin = gate && n == 1 ? gated_twin(*ke) : nullptr;
    const bool gated = twin != nullptr;
    const int TX = ke->shape.tx, TY = ke->shape.ty;
    // coefficient scratch
    size_t coef_total = 0;
    for (int i = 0; i < n; ++i) {
        int rc = validate_desc(descs[i]);
        if (rc) return rc;
        if (!descs[i].coef) coef_total += 3 * (size_t)descs[i].nlines;
    }
    int rc = c.coef.ensure(sizeof(double) * std::max<size_t>(coef_total, 3));
    if (rc) return rc;
    rc = c.bursts.ensure(sizeof(BurstDev) * n);
    if (rc) return rc;
    rc = c.tmaps.ensure(sizeof(CUtensorMap) * n);
    if (rc) return rc;
    rc = c.flags.ensure(64);
    if (rc) return rc;
    std::vector<BurstDev> hb(n);
    std::vector<CUtensorMap> hm(n);
    double *coef_base = static_cast<double *>(c.coef.p);
    size_t coef_off = 0;
    int total = 0, max_burst_tiles = 0;
    for (int i = 0; i < n; ++i) {
        const srg_burst_desc &d = descs[i];
        const double *coef = d.coef;
        if (!coef) {
            double *dst = coef_base + coef_off;
            coef_off += 3 * (size_t)d.nlines;
            BurstDev tmp = make_burst_dev(d, dst);
            if (o.centres_on_host)
                return fail(SRG_E_UNSUPPORTED, "host centres need host DEM (use the file entry)");
            rc = centres_device(c, d, tmp, dst, st);
            if (rc) return rc;
            coef = dst;
        }
        BurstDev B = make_burst_dev(d, coef);
        if (o.spin_limit > 0) B.spin = (unsigned)o.spin_limit;
        // row blocks copied back while the sum runs count whole tile rows of
        // rectangular tiles
        if ((rc = set_tiles(B, *ke, gated && gate->rb ? 0 : o.tile_shear))) return rc;
        B.tile_base = total;
        total += B.tiles_x * B.tiles_y;
        max_burst_tiles = std::max(max_burst_tiles, B.tiles_x * B.tiles_y);
        if (make_tmap(B, ke->shape.window, ke->shape.chunk, &hm[i]) == 0) B.tmap = i;
        if (gated) {
            B.ready = gate->word;
            B.ready_base = gate->base;
            B.ready_rows = gate->rows;
            if (gate->rb) {
                constexpr int K = DevCtx::kRowBlocks;
                B.rb_count = gate->rb;
                B.rb_expect = gate->rb + K;
                B.rb_order = gate->rb + 2 * K;
                B.rb_done = gate->rb + 3 * K;
                B.rb_tile_rows = gate->rb_tile_rows;
                B.rb_seq = gate->rb_seq;
            }
        }
        hb[i] = B;
    }
    if (total == 0) return SRG_OK;
    rc = c.tiles.ensure(tile_list_bytes(total));
    if (rc) return rc;
    CK(cudaMemcpyAsync(c.bursts.p, hb.data(), sizeof(BurstDev) * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c.tmaps.p, hm.data(), sizeof(CUtensorMap) * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(c.flags.p, 0, sizeof(int), st));  // work counter only
    const int idx = kernel_index(ke);
    ensure_attrs(c, idx);
    if (gated && (rc = ensure_gated_attrs(c, *twin))) return rc;
    const KernelEntry &run = gated ? *twin : *ke;
    const int smem = shared_bytes(run);
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, run.fn, run.shape.threads, smem));
    if (per_sm < 1) return fail(SRG_E_UNSUPPORTED, "kernel shape %d does not fit an SM", idx);
    const int grid = std::min(total, per_sm * c.sms);
    int *flags = static_cast<int *>(c.flags.p);
    if (before_sum && !gated) CK(cudaStreamWaitEvent(st, before_sum, 0));
    const BurstDev *d_bursts = static_cast<const BurstDev *>(c.bursts.p);
    CK(launch_tile_list(d_bursts, n, max_burst_tiles, total, TX, TY, c.tiles.p, st, band));
    if (band && band_host) {
        CK(cudaMemcpyAsync(band_host, band, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        if (gated && gate->rb && gate->rb_host)
            CK(cudaMemcpyAsync(gate->rb_host, gate->rb + DevCtx::kRowBlocks,
                               (DevCtx::kRowBlocks + 1) * sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(band_ready, st));
    }
    CK(launch_tiles(run, grid, smem, st, d_bursts, n, total,
                    static_cast<const CUtensorMap *>(c.tmaps.p), flags, flags + 1,
                    static_cast<const int *>(c.tiles.p)));
    // host vectors hb/hm were copied from pageable memory: the copies are
    // complete (staged) when cudaMemcpyAsync returns for pageable sources.
    return SRG_OK;
}

int check_flags(DevCtx &c, cudaStream_t st) {
    int h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, c.flags.p, sizeof h, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h[1]) {
        cudaMemsetAsync(static_cast<int *>(c.flags.p) + 1, 0, sizeof(int), st);
        return fail(SRG_E_TIMEOUT, "device error word 0x%x (TMA wait timed out)", h[1]);
    }
    return SRG_OK;
}

}  // namespace

extern "C" {

void srg_bp_default_options(srg_bp_options *o) {
    if (!o) return;
    o->form = SRG_FORM_SPLIT;
    o->tile_cfg = -1;
    o->device = -1;
    o->centres_on_host = 0;
    o->verbose = 0;
    o->spin_limit = 0;
    o->full_lines = 0;
    o->scratch_limit = 0;
    o->overlap = env_overlap();
    o->tile_shear = 0;
}

const char *srg_last_error(void) { return g_err.c_str(); }

void srg_set_default_options(const srg_bp_options *o) {
    std::lock_guard<std::mutex> g(g_opts_mu);
    if (o) g_default_opts = *o;
    else srg_bp_default_options(&g_default_opts);
}

int srg_tile_config_count(void) { return kNumKernels; }

int srg_tile_shear(const srg_burst_desc *b, int tile_cfg, int tile_shear, int *shear,
                   int *tiles_x, int *tiles_y) {
    if (!b || !shear || !tiles_x || !tiles_y) return fail(SRG_E_ARG, "null argument");
    const KernelEntry *ke = tile_cfg < 0 ? pick_kernel(SRG_FORM_SPLIT, -1)
                            : tile_cfg < kNumKernels ? &kKernels[tile_cfg] : nullptr;
    if (!ke) return fail(SRG_E_ARG, "shape index %d", tile_cfg);
    BurstDev B = make_burst_dev(*b, nullptr);
    if (const int rc = set_tiles(B, *ke, tile_shear)) return rc;
    *shear = B.shear;
    *tiles_x = B.tiles_x;
    *tiles_y = B.tiles_y;
    return SRG_OK;
}

const char *srg_tile_config_name(int idx) {
    if (idx < 0 || idx >= kNumKernels) return "";
    return kKernels[idx].name;
}

int srg_tile_config(int idx, int *tile_x, int *tile_y, int *threads, int *chunk, int *window) {
    if (idx < 0 || idx >= kNumKernels) return fail(SRG_E_ARG, "shape index %d", idx);
    const TileShape &s = kKernels[idx].shape;
    if (tile_x) *tile_x = s.tx;
    if (tile_y) *tile_y = s.ty;
    if (threads) *threads = s.threads;
    if (chunk) *chunk = s.chunk;
    if (window) *window = s.window;
    return kKernels[idx].form;
}

int srg_bp_bursts_device(const srg_burst_desc *bursts, int n, const srg_bp_options *opts,
                         void *stream) {
    if (!bursts || n < 1) return fail(SRG_E_ARG, "no bursts");
    srg_bp_options o;
    srg_bp_default_options(&o);
    if (opts) o = *opts;
    DevCtx *c = nullptr;
    int rc = get_ctx(o.device, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    return run_bursts(*c, bursts, n, o, static_cast<cudaStream_t>(stream));
}

int srg_bp_burst_device_gated(const srg_burst_desc *b, const int *ready_word, int ready_base,
                              int ready_rows, const srg_bp_options *opts, void *stream) {
    if (!b || !ready_word || ready_rows < 1 || ready_base < 0)
        return fail(SRG_E_ARG, "bad arguments (ready_word %p, base %d, rows %d)",
                    (const void *)ready_word, ready_base, ready_rows);
    if ((long long)ready_base + (b->P + ready_rows - 1) / ready_rows > INT_MAX)
        return fail(SRG_E_ARG, "ready_base %d leaves no room for the granule count", ready_base);
    srg_bp_options o;
    srg_bp_default_options(&o);
    if (opts) o = *opts;
    const KernelEntry *ke = pick_kernel(o.form, o.tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", o.form, o.tile_cfg);
    if (!gated_twin(*ke))
        return fail(SRG_E_UNSUPPORTED, "kernel shape %s has no twin that waits for arriving lines",
                    ke->name);
    DevCtx *c = nullptr;
    int rc = get_ctx(o.device, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    UploadGate gate{ready_word, ready_base, ready_rows};
    return run_bursts(*c, b, 1, o, static_cast<cudaStream_t>(stream), nullptr, &gate);
}

int srg_dropin_last_bytes(int device, long long *h2d, long long *d2h) {
    DropinDev *D = nullptr;
    int rc = get_dropin(device, &D);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(D->call_mu);
    if (h2d) *h2d = D->last_h2d;
    if (d2h) *d2h = D->last_d2h;
    return SRG_OK;
}

int srg_dropin_flush(int device) {
    if (device >= 0) {
        DropinDev *D = nullptr;
        int rc = get_dropin(device, &D);
        if (rc) return rc;
        dropin_wait_idle(*D);
        return dropin_take_pending(*D);
    }
    int first = SRG_OK;
    std::string msg;
    for (int i = 0; i < 64; ++i) {
        DropinDev &d = g_dropin[i];
        bool started;
        {
            std::lock_guard<std::mutex> lk(d.q_mu);
            started = d.worker;
        }
        if (!started) continue;
        dropin_wait_idle(d);
        const int rc = dropin_take_pending(d);
        if (rc && !first) {
            first = rc;
            msg = g_err;
        }
    }
    if (first) g_err = msg;
    return first;
}

int srg_test_set_dropin_sequence(int device, int seq) {
    if (seq < 0 || seq > DevCtx::kSeqLimit)
        return fail(SRG_E_ARG, "sequence %d outside [0, %d]", seq, DevCtx::kSeqLimit);
    DropinDev *D = nullptr;
    int rc = get_dropin(device, &D);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(D->call_mu);
    dropin_wait_idle(*D);
    for (DevCtx &c : D->slot) c.upload_seq = seq;
    return SRG_OK;
}

int srg_sync_check(void *stream) {
    DevCtx *c = nullptr;
    int rc = get_ctx(-1, &c);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    if (!c->flags.p) return SRG_OK;
    return check_flags(*c, st);
}

int srg_count_terms_device(const srg_burst_desc *bursts, int n, int64_t *terms, void *stream) {
    if (!bursts || n < 1 || !terms) return fail(SRG_E_ARG, "bad arguments");
    DevCtx *c = nullptr;
    int rc = get_ctx(-1, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = c->flags.ensure(64);
    if (rc) return rc;
    unsigned long long *cnt = reinterpret_cast<unsigned long long *>(static_cast<int *>(c->flags.p) + 2);
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
    size_t coef_total = 0;
    for (int i = 0; i < n; ++i) {
        rc = validate_desc(bursts[i]);
        if (rc) return rc;
        if (!bursts[i].coef) coef_total += 3 * (size_t)bursts[i].nlines;
    }
    rc = c->coef.ensure(sizeof(double) * std::max<size_t>(coef_total, 3));
    if (rc) return rc;
    double *coef_base = static_cast<double *>(c->coef.p);
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        const double *coef = bursts[i].coef;
        if (!coef) {
            double *dst = coef_base + off;
            off += 3 * (size_t)bursts[i].nlines;
            rc = centres_device(*c, bursts[i], make_burst_dev(bursts[i], dst), dst, st);
            if (rc) return rc;
            coef = dst;
        }
        BurstDev B = make_burst_dev(bursts[i], coef);
        CK(launch_count_terms(B, cnt, c->sms, st));
    }
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, cnt, sizeof h, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *terms = (int64_t)h;
    return SRG_OK;
}

int srg_merge_device(float *dst, int64_t dst_ld, const float *src, int64_t src_ld, int rows,
                     int cols, void *stream) {
    if (!dst || !src || rows < 0 || cols < 0) return fail(SRG_E_ARG, "bad merge arguments");
    DevCtx *c = nullptr;
    int rc = get_ctx(-1, &c);
    if (rc) return rc;
    CK(launch_merge(reinterpret_cast<float2 *>(dst), dst_ld, reinterpret_cast<const float2 *>(src),
                    src_ld, rows, cols, c->sms, static_cast<cudaStream_t>(stream)));
    return SRG_OK;
}

int srg_line_centres_device(const srg_burst_desc *b, double *coef_out, void *stream) {
    if (!b || !coef_out) return fail(SRG_E_ARG, "bad arguments");
    int rc = validate_desc(*b);
    if (rc) return rc;
    DevCtx *c = nullptr;
    rc = get_ctx(-1, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    return centres_device(*c, *b, make_burst_dev(*b, coef_out), coef_out,
                          static_cast<cudaStream_t>(stream));
}

int srg_pulse_orbit_device(const double *times, int P, const double *timeorbit, const double *xx,
                           const double *vv, int numstatevec, double *pos, double *vel,
                           void *stream) {
    if (!times || !timeorbit || !xx || !vv || !pos || !vel || P < 0 || numstatevec < 4)
        return fail(SRG_E_ARG, "bad arguments");
    DevCtx *c = nullptr;
    int rc = get_ctx(-1, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = numstatevec;
    rc = c->orbit.ensure(sizeof(double) * 7 * (size_t)n);
    if (rc) return rc;
    double *ob = static_cast<double *>(c->orbit.p);
    std::vector<double> host(7 * (size_t)n);
    std::memcpy(host.data(), timeorbit, sizeof(double) * n);
    std::memcpy(host.data() + n, xx, sizeof(double) * 3 * n);
    std::memcpy(host.data() + 4 * n, vv, sizeof(double) * 3 * n);
    CK(cudaMemcpyAsync(ob, host.data(), sizeof(double) * 7 * n, cudaMemcpyHostToDevice, st));
    Orbit o{ob, ob + n, ob + 4 * n, n};
    CK(launch_pulse_orbit(times, P, o, pos, vel, st));
    CK(cudaStreamSynchronize(st));
    return SRG_OK;
}

int srg_forward_project_device(const srg_burst_desc *b, const float *refl, int64_t refl_ld,
                               const double *satvel, double antenna_m, const float *range_offset,
                               void *stream) {
    if (!b || !refl || !satvel) return fail(SRG_E_ARG, "bad arguments");
    int rc = validate_desc(*b);
    if (rc) return rc;
    if (b->bin0 != 0 || (b->nbins != 0 && b->nbins != b->S))
        return fail(SRG_E_ARG, "forward projection writes whole lines (bin0 0, nbins 0 or S)");
    DevCtx *c = nullptr;
    rc = get_ctx(-1, &c);
    if (rc) return rc;
    BurstDev B = make_burst_dev(*b, nullptr);
    CK(launch_forward_project(B, reinterpret_cast<const float2 *>(refl), refl_ld, satvel,
                              antenna_m, range_offset, static_cast<cudaStream_t>(stream)));
    return SRG_OK;
}

int srg_measure_fma_peak(int fp64, double *tflops) {
    if (!tflops) return fail(SRG_E_ARG, "null output");
    DevCtx *c = nullptr;
    int rc = get_ctx(-1, &c);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(c->mu);
    rc = c->orbit.ensure(sizeof(double) * 64 * 1024);
    if (rc) return rc;
    const int blocks = c->sms * 8;   // 8 x 256 threads = full occupancy
    const int iters = fp64 ? 4096 : 8192;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(launch_fma_peak(fp64, blocks, iters, c->orbit.p, 0));  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        CK(cudaEventRecord(e0, 0));
        CK(launch_fma_peak(fp64, blocks, iters, c->orbit.p, 0));
        CK(cudaEventRecord(e1, 0));
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * 8.0 * (double)iters * 256.0 * (double)blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SRG_OK;
}

int srg_azimuth_compress(const float *burstdata, const double *satloc, int rawdatalines,
                         int samplesPerBurst, int demwidth, int demlength, int fdout, int fddem,
                         double deltalat, double deltalon, double firstlat, double firstlon,
                         const double *latlons, const double *timeorbit, const double *xx,
                         const double *vv, int numstatevec, double rngstart, double rngend,
                         double tmid, const double *xyz_mid, const double *vel_mid, double dmrg,
                         double wvl, int aperture, double angc0, double angc1, double prf,
                         const srg_bp_options *opts) {
    if (!burstdata || !satloc || !latlons || !timeorbit || !xx || !vv || !xyz_mid || !vel_mid)
        return fail(SRG_E_ARG, "null argument");
    if (rawdatalines < 1 || samplesPerBurst < 2 || demwidth < 1 || demlength < 1 ||
        numstatevec < 4 || !(dmrg > 0) || !(wvl > 0) || aperture < 0)
        return fail(SRG_E_ARG, "bad sizes or scalars (P=%d S=%d W=%d L=%d n=%d)", rawdatalines,
                    samplesPerBurst, demwidth, demlength, numstatevec);
    // Non-finite geometry would leave every pixel unformed without a word
    // (NaN fails every range and window test): refuse it before any work.
    {
        const double sc[] = {deltalat, deltalon, firstlat, firstlon, rngstart, rngend, tmid,
                             dmrg, wvl, angc0, angc1, prf};
        const char *bad = !all_finite(sc, sizeof sc / sizeof sc[0]) ? "a scalar argument"
                          : !all_finite(latlons, 4)                 ? "latlons"
                          : !all_finite(xyz_mid, 3) || !all_finite(vel_mid, 3) ? "xyz_mid / vel_mid"
                          : !all_finite(timeorbit, numstatevec)     ? "timeorbit"
                          : !all_finite(xx, 3 * (size_t)numstatevec) ? "xx"
                          : !all_finite(vv, 3 * (size_t)numstatevec) ? "vv"
                          : !all_finite(satloc, 3 * (size_t)rawdatalines) ? "satloc"
                                                                    : nullptr;
        if (bad) return fail(SRG_E_ARG, "non-finite value in %s", bad);
    }
    srg_bp_options o;
    if (opts) o = *opts;
    else {
        std::lock_guard<std::mutex> g(g_opts_mu);
        o = g_default_opts;
    }
    if (o.centres_on_host)
        return fail(SRG_E_UNSUPPORTED, "azimuth centres are solved on the device only");
    int fl, ll, fp_, lp_;
    ref_limits(latlons, firstlat, deltalat, firstlon, deltalon, demwidth, demlength, &fl, &ll, &fp_,
               &lp_);
    const int nl = ll - fl + 1;
    if (o.verbose) printf("Burst line limits, size (first,last,nlines) %d %d %d\n", fl, ll, nl);
    if (nl < 1)
        return fail(SRG_E_ARG, "latlons select no grid line (first line %d, last line %d)", fl, ll);
    const int W = demwidth;
    const int fp = fp_, lp = lp_;

    const int fp_eff = std::max(fp, 0);
    const int lp_eff = std::min(lp, W - 1);
    const int ncols = lp_eff >= fp_eff ? lp_eff - fp_eff + 1 : 0;
    if (ncols == 0) return SRG_OK;  // no pixel of the grid in the burst's box
    // pinned staging: the DEM box in, the output box back
    const size_t dem_bytes = (size_t)nl * ncols * 2;
    const size_t win_bytes = (size_t)nl * ncols * 8;
    if (o.scratch_limit > 0) {
        // device scratch of this call: range lines, orbit, DEM box, output box,
        // parabolas, work list (for the smallest tiles of any shape) and descriptors
        const KernelEntry *kc = pick_kernel(o.form, o.tile_cfg);
        const int tx = kc ? kc->shape.tx : 32, ty = kc ? kc->shape.ty : 4;
        const long long tiles = (long long)((ncols + tx - 1) / tx) * ((nl + ty - 1) / ty);
        const long long need = (long long)rawdatalines * ((samplesPerBurst + 1) & ~1) * 8 +
                               24LL * rawdatalines + (long long)dem_bytes + (long long)win_bytes +
                               24LL * nl + 56LL * numstatevec +
                               (long long)tile_list_bytes((int)std::min<long long>(tiles, INT_MAX)) +
                               4096;
        if (need > o.scratch_limit)
            return fail(SRG_E_NOMEM, "the call needs %lld bytes of device scratch, the limit is %lld",
                        need, (long long)o.scratch_limit);
    }
    DropinDev *D = nullptr;
    int rc = get_dropin(o.device, &D);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(D->call_mu);
    // An overlapped call takes the context the call before last used, once
    // that call's tail is done; a call without overlap waits for every tail.
    int si = 0;
    if (o.overlap) {
        si = D->next;
        D->next ^= 1;
        std::unique_lock<std::mutex> lk(D->q_mu);
        D->q_cv.wait(lk, [&] { return !D->busy[si]; });
    } else {
        dropin_wait_idle(*D);
    }
    DevCtx *c = &D->slot[si];
    if ((rc = ensure_dropin(*c))) return rc;
    cudaStream_t st = c->s_main;
    const size_t stage_bytes = std::max(dem_bytes, win_bytes) + 64;
    if (stage_bytes > c->host_cap) {
        if (c->host_stage) cudaFreeHost(c->host_stage);
        c->host_stage = nullptr;
        c->host_cap = 0;
        if (cudaMallocHost(&c->host_stage, stage_bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(SRG_E_NOMEM, "pinned staging of %zu bytes failed", stage_bytes);
        }
        c->host_cap = stage_bytes;
    }
    // room for whole lines at an even row pitch (the range band needs less)
    const size_t bbytes = (size_t)rawdatalines * (size_t)((samplesPerBurst + 1) & ~1) * 8;
    if ((rc = c->in_burst.ensure(bbytes)) || (rc = c->in_sat.ensure(24 * (size_t)rawdatalines)) ||
        (rc = c->in_dem.ensure(dem_bytes)) || (rc = c->out.ensure(win_bytes)) ||
        (rc = c->flags.ensure(64)))
        return rc;
    HostPool &pool = HostPool::get();
    // Once the first copy is queued, a failure waits for the three streams
    // before it returns: queued copies may still read the caller's buffers.
    auto drain = [&] {
        cudaStreamSynchronize(c->s_copy);
        cudaStreamSynchronize(c->s_back);
        cudaStreamSynchronize(st);
    };
#define CKD(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            drain();                                                                   \
            return fail(SRG_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
        }                                                                              \
    } while (0)
    // The range lines upload on their own stream in blocks of pulse rows; after
    // each block the copy stream raises a device word, and the backprojection,
    // launched without waiting for the whole upload, takes a chunk of pulses as
    // soon as its rows are in.  The orbit, the DEM box and the azimuth centres
    // (which need no range lines) proceed meanwhile.  The word counts granules
    // of P/32 pulse rows; the blocks shrink toward the end (6, 6, 5, 5, 4, 3,
    // 2, 1 granules), so that little of the sum waits for the last one.  The
    // word grows from call to call (call number x 64 + granules), so a value
    // left by an earlier call never satisfies a later one; the row blocks'
    // done words hold the call number.  When the call number restarts, both
    // are cleared first (every earlier call on this context has finished its
    // GPU work: a call's tail waits for its three streams, and a call takes a
    // context only once the tail of the call that last held it is done).
    int *ready_word = static_cast<int *>(c->flags.p) + DevCtx::kReadyWord;
    constexpr int kGranules = 32;
    static const int kBlockEnd[DevCtx::kUploadBlocks] = {6, 12, 17, 22, 26, 29, 31, 32};
    const int nup = DevCtx::kUploadBlocks;
    const int up_rows = (rawdatalines + kGranules - 1) / kGranules;  // rows per granule
    const int ngran = (rawdatalines + up_rows - 1) / up_rows;
    if (c->upload_seq >= DevCtx::kSeqLimit) {
        CK(cudaMemsetAsync(ready_word, 0, sizeof(int), st));
        CK(cudaMemsetAsync(static_cast<int *>(c->rb.p) + 3 * DevCtx::kRowBlocks, 0,
                           DevCtx::kRowBlocks * sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        c->upload_seq = 0;
    }
    ++c->upload_seq;
    const int ready_base = c->upload_seq * 64;
    // The lines go up cropped to the range bins the sum can read (the range
    // band, known once the DEM box and the azimuth centres are on the device):
    // rows of nbins samples from bin bin0, row pitch ldbc samples.
    int bin0 = 0, nbins = samplesPerBurst;
    long long ldbc = (samplesPerBurst + 1) & ~1;
    auto upload = [&](int kb, int ke) -> int {
        const size_t spitch = (size_t)samplesPerBurst * 8, dpitch = (size_t)ldbc * 8;
        const size_t width = (size_t)nbins * 8;
        for (int k = kb; k < ke; ++k) {
            const int g0 = k ? std::min(kBlockEnd[k - 1], ngran) : 0, g1 = std::min(kBlockEnd[k], ngran);
            const int r0 = std::min(rawdatalines, g0 * up_rows), r1 = std::min(rawdatalines, g1 * up_rows);
            if (r0 < r1) {
                char *dst = static_cast<char *>(c->in_burst.p) + (size_t)r0 * dpitch;
                const char *src = reinterpret_cast<const char *>(burstdata) + (size_t)r0 * spitch +
                                  (size_t)bin0 * 8;
                if (dpitch == spitch && width == spitch)
                    CK(cudaMemcpyAsync(dst, src, (size_t)(r1 - r0) * spitch, cudaMemcpyHostToDevice,
                                       c->s_copy));
                else
                    CK(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, r1 - r0,
                                         cudaMemcpyHostToDevice, c->s_copy));
            }
            c->host_flags[DevCtx::kReadyHost + k] = ready_base + g1;
            CK(cudaMemcpyAsync(ready_word, c->host_flags + DevCtx::kReadyHost + k, sizeof(int),
                               cudaMemcpyHostToDevice, c->s_copy));
        }
        return SRG_OK;
    };
    UploadGate gate{ready_word, ready_base, up_rows};
    // Host-to-device copies leave the copy engine in the order they are
    // issued, whatever their stream: the small inputs and the DEM box go
    // first; with a gated kernel then the first block and the launch, and the
    // other blocks last; without one, every block before the launch, which
    // waits for them all.
    const KernelEntry *ke0 = pick_kernel(o.form, o.tile_cfg);
    const bool pipelined = ke0 && gated_twin(*ke0) != nullptr;
    // With the gated kernel the output also comes back while the sum runs: the
    // grid lines are cut into row blocks of whole tile rows; the kernel counts
    // the stored tiles of each block and raises the block's done word when the
    // count reaches the block's kept tiles, and a stream of its own waits for
    // that word before it copies the block back.  Every done word is also
    // written on the main stream after the kernel, so each wait ends even when
    // the kernel gives up early (the block then merges only if the error word
    // is clear).
    constexpr int K = DevCtx::kRowBlocks;
    const StreamValueOps svo = stream_value_ops();
    const int tile_ty = ke0 ? ke0->shape.ty : 1;
    const int tiles_y = (nl + tile_ty - 1) / tile_ty;
    const int rb_tiles = std::max(1, (tiles_y + K - 1) / K);
    const int nrb = (tiles_y + rb_tiles - 1) / rb_tiles;
    const bool rows_back = pipelined && svo.wait && svo.write;
    int *rbw = static_cast<int *>(c->rb.p);
    if (rows_back) {
        gate.rb = rbw;
        gate.rb_tile_rows = rb_tiles;
        gate.rb_seq = c->upload_seq;
        gate.rb_host = c->host_rb;
        for (int k = 0; k <= K; ++k) c->host_rb[k] = 0;
        CK(cudaMemsetAsync(rbw, 0, (2 * K + 1) * sizeof(int), st));
    }
    CK(cudaMemcpyAsync(c->in_sat.p, satloc, 24 * (size_t)rawdatalines, cudaMemcpyHostToDevice, st));
    // DEM box of rows [fl, fl + nl) (azimuth_compress.cu:399-408), read by the
    // pool's threads; a file that ends before the box does is an error (the
    // reference would use whatever its buffer held)
    int16_t *slab = static_cast<int16_t *>(c->host_stage);
    std::atomic<int> io_err{0};
    const int ntask = std::max(1, std::min(nl, 4 * HostPool::threads()));
    // Each row is read into a small buffer of the thread's own and moved into
    // the pinned slab with non-temporal stores: a slab written through the CPU
    // caches leaves its lines dirty in many cores' caches, and the DMA that
    // follows then copies at about a seventh of the rate it reaches on lines
    // held in memory only (0.7 ms against 0.1 ms for a 5 MB box).  The box is
    // copied to the device in kDemBlocks blocks of rows, each queued by the
    // thread that stores its last row, so the copies overlap the reads.
    constexpr int kDemBlocks = 4;
    const int ndb = std::min(kDemBlocks, nl);
    auto dem_block_row = [&](int b) { return (int)((long long)nl * b / ndb); };
    std::atomic<int> rows_left[kDemBlocks];
    for (int b = 0; b < ndb; ++b) rows_left[b] = dem_block_row(b + 1) - dem_block_row(b);
    std::atomic<int> copy_err{0};
    const int dev = c->dev;
    pool.run(ntask, [&](int t) {
        const size_t want = (size_t)ncols * 2;
        std::vector<char> row(want);
        for (int r = (int)((long long)nl * t / ntask); r < (int)((long long)nl * (t + 1) / ntask); ++r) {
            size_t done = 0;
            while (done < want) {   // pread may return fewer bytes than asked
                const ssize_t got = pread(fddem, row.data() + done, want - done,
                                          ((off_t)(fl + r) * W + fp_eff) * 2 + (off_t)done);
                if (got <= 0) {
                    io_err = got < 0 ? 1 : 2;
                    return;
                }
                done += (size_t)got;
            }
            copy_nontemporal(reinterpret_cast<char *>(slab + (size_t)r * ncols), row.data(), want);
            store_fence();  // the row's stores before its count (and the block's copy)
            int b = (int)((long long)r * ndb / nl);  // the block whose rows hold r
            while (b + 1 < ndb && dem_block_row(b + 1) <= r) ++b;
            while (b > 0 && dem_block_row(b) > r) --b;
            if (rows_left[b].fetch_sub(1) == 1 && !io_err) {
                const size_t off = (size_t)dem_block_row(b) * ncols;
                const size_t n = (size_t)(dem_block_row(b + 1) - dem_block_row(b)) * ncols * 2;
                cudaError_t e = cudaSetDevice(dev);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(static_cast<int16_t *>(c->in_dem.p) + off, slab + off, n,
                                        cudaMemcpyHostToDevice, st);
                if (e != cudaSuccess) copy_err = (int)e;
            }
        }
    });
    if (io_err) {
        drain();
        return fail(SRG_E_IO, io_err == 1 ? "DEM read failed (fd %d)"
                                          : "DEM file (fd %d) ends before the burst's rows do",
                    fddem);
    }
    CKD((cudaError_t)copy_err.load());

    srg_burst_desc d{};
    d.burst = static_cast<const float *>(c->in_burst.p);
    d.satloc = static_cast<const double *>(c->in_sat.p);
    // the sum reads DEM columns [firstpix, lastpix_eff] only: the descriptor's
    // column 0 lies fp_eff entries before the box
    d.dem = static_cast<const int16_t *>(c->in_dem.p) - fp_eff;
    d.out = static_cast<float *>(c->out.p);
    d.coef = nullptr;
    d.ldb = ldbc;
    d.dem_ld = ncols;
    d.out_ld = ncols;
    d.P = rawdatalines;
    d.S = samplesPerBurst;
    d.demwidth = W;
    d.firstline = fl;
    d.nlines = nl;
    d.firstpix = fp;
    d.lastpix = lp;
    d.out_pix0 = fp_eff;
    d.aperture = aperture;
    d.firstlat = firstlat;
    d.deltalat = deltalat;
    d.firstlon = firstlon;
    d.deltalon = deltalon;
    d.rngstart = rngstart;
    d.rngend = rngend;
    d.dmrg = dmrg;
    d.wvl = wvl;
    d.timeorbit = timeorbit;
    d.xx = xx;
    d.vv = vv;
    d.numstatevec = numstatevec;
    d.tmid = tmid;
    for (int i = 0; i < 3; ++i) {
        d.xyz_mid[i] = xyz_mid[i];
        d.vel_mid[i] = vel_mid[i];
    }
    d.angc0 = angc0;
    d.angc1 = angc1;
    d.prf = prf;
    // azimuth centres (azimuth_compress.cu:438-481) on the device, before the
    // lines: the range band needs them, and so does the sum
    if ((rc = c->coef.ensure(sizeof(double) * 3 * (size_t)nl))) {
        drain();
        return rc;
    }
    double *coef = static_cast<double *>(c->coef.p);
    if ((rc = centres_device(*c, d, make_burst_dev(d, coef), coef, st))) {
        drain();
        return rc;
    }
    d.coef = coef;
    // The range band: every bin a term of a formed pixel can read, with a
    // margin; the whole line unless the pulses satisfy the convexity test
    // the band's bisection relies on (pulses_convex).
    if (!o.full_lines && pulses_convex(satloc, rawdatalines, rngend)) {
        int *rw = static_cast<int *>(c->flags.p) + DevCtx::kRangeWord;
        CKD(cudaMemsetAsync(rw, 0x7f, sizeof(int), st));      // INT_MAX-like
        CKD(cudaMemsetAsync(rw + 1, 0x80, sizeof(int), st));  // INT_MIN-like
        CKD(launch_range_band(make_burst_dev(d, coef), rw, c->sms, st));
        CKD(cudaMemcpyAsync(c->host_flags + DevCtx::kRangeHost, rw, 2 * sizeof(int),
                            cudaMemcpyDeviceToHost, st));
        CKD(cudaStreamSynchronize(st));
        const int lo = c->host_flags[DevCtx::kRangeHost], hi = c->host_flags[DevCtx::kRangeHost + 1];
        if (lo <= hi) {
            const long long b0 = std::max<long long>(0, (long long)lo - kBandMargin) & ~1LL;
            const long long b1 = std::min<long long>(samplesPerBurst - 1, (long long)hi + kBandMargin);
            if (b1 > b0 && b0 < samplesPerBurst) {
                bin0 = (int)b0;
                nbins = (int)(b1 - b0 + 1);
            }
        } else {  // no formed pixel: nothing is read
            bin0 = 0;
            nbins = std::min(samplesPerBurst, 2);
        }
        ldbc = (nbins + 1) & ~1;
    }
    d.ldb = ldbc;
    d.bin0 = bin0;
    d.nbins = nbins;
    c->last_h2d = (long long)rawdatalines * nbins * 8 + 24LL * rawdatalines + (long long)dem_bytes +
                  56LL * numstatevec;
    c->last_d2h = 0;
    if ((rc = upload(0, pipelined ? 1 : nup))) {
        drain();  // the caller's buffer stays in use until then
        return rc;
    }
    if (!pipelined) CKD(cudaEventRecord(c->ev_burst, c->s_copy));
    // rows of the kept tiles (the band): rows outside it have no formed pixel
    int *band = static_cast<int *>(c->flags.p) + DevCtx::kBandWord;
    CKD(cudaMemsetAsync(band, 0x7f, sizeof(int), st));      // INT_MAX-like
    CKD(cudaMemsetAsync(band + 1, 0xff, sizeof(int), st));  // -1
    c->host_flags[DevCtx::kBandWord] = INT_MAX;  // an empty band unless the list reports one
    c->host_flags[DevCtx::kBandWord + 1] = -1;
    CKD(cudaEventRecord(c->ev_band, st));
    rc = run_bursts(*c, &d, 1, o, st, pipelined ? nullptr : c->ev_burst, pipelined ? &gate : nullptr,
                    band, c->host_flags + DevCtx::kBandWord, c->ev_band);
    if (!rc && pipelined) {
        rc = upload(1, nup);
        if (!rc && cudaEventRecord(c->ev_burst, c->s_copy) != cudaSuccess)
            rc = fail(SRG_E_CUDA, "event record failed");
    }
    if (rc) {
        drain();
        return rc;
    }
    // The done words' writes after the kernel, issued after every upload copy
    // (a stream's wait for the kernel must not hold copies the kernel needs,
    // should two streams share a hardware queue).  Blocks [0, nfall) have one.
    int nfall = 0;
    if (rows_back) {
        while (nfall < nrb &&
               svo.write(st, reinterpret_cast<CUdeviceptr>(rbw + 3 * K + nfall),
                         (cuuint32_t)c->upload_seq, 0) == CUDA_SUCCESS)
            ++nfall;
    }
    // The band is known once the work list is built, ahead of the backprojection.
    // Without row blocks its rows' copies back are queued behind the sum at
    // once, after the error word, in up to kOutBlocks blocks; the merge of a
    // block starts as soon as that block is back and the error word is clear.
    CKD(cudaEventSynchronize(c->ev_band));
    CKD(cudaMemcpyAsync(c->host_flags, c->flags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CKD(cudaEventRecord(c->ev_flags, st));
    const int band_lo = std::max(0, c->host_flags[DevCtx::kBandWord]);
    const int band_hi = std::min(nl - 1, c->host_flags[DevCtx::kBandWord + 1]);
    const int nband = band_hi >= band_lo ? band_hi - band_lo + 1 : 0;
    float *win = static_cast<float *>(c->host_stage);
    OutBlock blk[DevCtx::kOutBlocks];
    int nblk = 0;
    auto copy_back = [&](int r0, int r1, cudaStream_t s) {
        const size_t off = (size_t)r0 * ncols * 2, n = (size_t)(r1 - r0) * ncols * 8;
        c->last_d2h += (long long)n;
        return cudaMemcpyAsync(win + off, static_cast<float *>(c->out.p) + off, n,
                               cudaMemcpyDeviceToHost, s);
    };
    if (rows_back) {
        // in the order the kernel finishes them (it takes the tiles from the
        // last line back when the lines run against the pulses)
        const bool from_last = c->host_rb[K] != 0;
        for (int i = 0; i < nrb; ++i) {
            const int k = from_last ? nrb - 1 - i : i;
            const int r0 = std::max(band_lo, k * rb_tiles * tile_ty);
            const int r1 = std::min(band_hi + 1, std::min(nl, (k + 1) * rb_tiles * tile_ty));
            if (r0 >= r1 || c->host_rb[k] == 0) continue;  // no kept tile: nothing formed
            OutBlock &b = blk[nblk];
            b.r0 = r0;
            b.r1 = r1;
            b.rb = -1;
            if (k < nfall &&
                svo.wait(c->s_back, reinterpret_cast<CUdeviceptr>(rbw + 3 * K + k),
                         (cuuint32_t)c->upload_seq, CU_STREAM_WAIT_VALUE_EQ) == CUDA_SUCCESS) {
                CKD(copy_back(r0, r1, c->s_back));
                CKD(cudaMemcpyAsync(c->host_rb + 2 * K + k, rbw + k, sizeof(int),
                                   cudaMemcpyDeviceToHost, c->s_back));
                CKD(cudaEventRecord(c->ev_blk[nblk], c->s_back));
                b.rb = k;
            } else {
                CKD(copy_back(r0, r1, st));
                CKD(cudaEventRecord(c->ev_blk[nblk], st));
            }
            ++nblk;
        }
    } else {
        const int n = std::min(nband, (int)DevCtx::kOutBlocks);
        for (int k = 0; k < n; ++k) {
            OutBlock &b = blk[nblk++];
            b.r0 = band_lo + (int)((long long)nband * k / n);
            b.r1 = band_lo + (int)((long long)nband * (k + 1) / n);
            b.rb = -1;
            CKD(copy_back(b.r0, b.r1, st));
            CKD(cudaEventRecord(c->ev_blk[k], st));
        }
    }

    DropinTail tail;
    std::copy(blk, blk + nblk, tail.blk);
    tail.nblk = nblk;
    tail.ntask = ntask;
    tail.ncols = ncols;
    tail.fl = fl;
    tail.W = W;
    tail.fp_eff = fp_eff;
    tail.fdout = fdout;
    D->last_h2d = c->last_h2d;
    D->last_d2h = c->last_d2h;
    if (o.overlap) {
        // the caller's buffers are read by the upload only: free once it is
        // done; the tail merges through a descriptor of its own
        CKD(cudaStreamSynchronize(c->s_copy));
        tail.fdout = dup(fdout);
        tail.overlapped = true;
        if (tail.fdout >= 0) {
            // failures of earlier calls' tails only: this call's comes later
            const int earlier = dropin_take_pending(*D);
            const std::string earlier_msg = g_err;
            const int dev = c->dev;
            const bool queued = dropin_enqueue(*D, si, [D, c, tail, dev] {
                int r = cudaSetDevice(dev) == cudaSuccess ? dropin_tail(c, tail)
                                                          : fail(SRG_E_CUDA, "cudaSetDevice failed");
                close(tail.fdout);
                if (r) {
                    std::lock_guard<std::mutex> lk(D->q_mu);
                    if (!D->pending_rc) {
                        D->pending_rc = r;
                        D->pending_err = g_err;
                    }
                }
            });
            if (queued) {
                if (earlier) g_err = earlier_msg;
                return earlier;
            }
            // no worker thread to be had: the tail runs here after all
            close(tail.fdout);
            tail.fdout = fdout;
            tail.overlapped = false;
            rc = dropin_tail(c, tail);
            if (!rc && earlier) g_err = earlier_msg;
            return rc ? rc : earlier;
        }
        tail.fdout = fdout;  // no descriptor to spare: the tail runs here
        tail.overlapped = false;
    }
    rc = dropin_tail(c, tail);
    return rc ? rc : dropin_take_pending(*D);
#undef CKD
}

void azimuth_compress_(float *burstdata, double *satloc, int *rawdatalines, int *samplesPerBurst,
                       int *demwidth, int *demlength, int *fdout, int *fddem, double *deltalat,
                       double *deltalon, double *firstlat, double *firstlon, double *latlons,
                       double *timeorbit, double *xx, double *vv, int *numstatevec,
                       double *rngstart, double *rngend, double *tstart, double *tend, double *tmid,
                       double *xyz_mid, double *vel_mid, double *t, double *dtaz, double *dmrg,
                       double *wvl, int *aperture, int *iaperture, double *angc0, double *angc1,
                       double *prf) {
    (void)tstart;
    (void)tend;
    (void)t;
    (void)dtaz;
    (void)iaperture;
    const int rc = srg_azimuth_compress(
        burstdata, satloc, *rawdatalines, *samplesPerBurst, *demwidth, *demlength, *fdout, *fddem,
        *deltalat, *deltalon, *firstlat, *firstlon, latlons, timeorbit, xx, vv, *numstatevec,
        *rngstart, *rngend, *tmid, xyz_mid, vel_mid, *dmrg, *wvl, *aperture, *angc0, *angc1, *prf,
        nullptr);
    if (rc) fprintf(stderr, "azimuth_compress_: error %d: %s\n", rc, g_err.c_str());
}

}  // extern "C"
