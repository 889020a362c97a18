// scene.cu -- reusable plans for batched scenes (srg_scene_* in srg_bp.h).
//
// A plan holds, in device memory, everything one pass over a set of bursts
// needs besides the caller's inputs and outputs: the burst descriptors, one
// TMA descriptor per burst, the orbit state vectors and centre parameters of
// every burst, the per-line azimuth-centre parabolas and the work counter.
// A pass is a short chain of launches -- azimuth centres of every line of
// every burst (one launch), the counter reset, the work list of tiles with a
// formed pixel (a mask and an ordered compaction), the persistent
// backprojection (one launch for all bursts) and, when a scene raster is
// given, the ordered merge of every burst into it (one launch).  On a non-default stream the
// first pass is captured into a CUDA graph and later passes replay it.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "host_internal.h"

using namespace srg;
using namespace srg::detail;

struct srg_scene {
    int dev = -1;
    int n = 0;
    srg_bp_options opts{};
    int kernel = -1;                 // index into kKernels
    std::vector<srg_burst_desc> descs;
    std::vector<BurstDev> hb;        // host copy (tiles depend on the kernel shape)
    int total_tiles = 0;
    int total_lines = 0;
    int64_t terms = -1;
    float2 *scene = nullptr;
    long long scene_ld = 0;
    int scene_lines = 0, scene_cols = 0;
    // device memory owned by the plan
    BurstDev *d_bursts = nullptr;
    CUtensorMap *d_tmaps = nullptr;
    CentreJob *d_jobs = nullptr;
    double *d_coef = nullptr;
    double *d_orbit = nullptr;
    int *d_flags = nullptr;          // [0] work counter, [1] error word, [2..3] u64 term counter
    void *d_tiles = nullptr;         // work list of the backprojection (tile_list_bytes)
    size_t tiles_cap = 0;
    int max_burst_tiles = 0;
    bool mask_valid = false;         // d_tiles holds the mask of the outputs' last backprojection
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    // range interpolation: SRG_INTERP_LINEAR on the caller's lines, or
    // SRG_INTERP_OVERSAMPLED2 on 2x-oversampled copies the plan makes in
    // every pass (os_lines: one [P][os_ld] buffer per burst)
    int interp = SRG_INTERP_LINEAR;
    std::vector<float2 *> os_lines;
    std::vector<long long> os_ld;
};

namespace {

#define SCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(SRG_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

int alloc(void **p, size_t bytes) {
    const size_t n = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(p, n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(SRG_E_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    // zeroed: the flag words are read before any kernel has written them; the
    // zeroing (legacy stream) is finished before the caller's streams use it
    if (cudaMemset(*p, 0, n) != cudaSuccess || cudaStreamSynchronize(0) != cudaSuccess) {
        cudaGetLastError();
        return fail(SRG_E_CUDA, "zeroing of plan memory failed");
    }
    return SRG_OK;
}

void drop_graph(srg_scene *s) {
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->graph_stream = nullptr;
}

// (Re)build the burst table and TMA descriptors for kernel shape `idx`.
int set_kernel(srg_scene *s, int idx) {
    const KernelEntry &ke = kKernels[idx];
    std::vector<CUtensorMap> hm(s->n);
    int total = 0, max_burst_tiles = 0;
    for (int i = 0; i < s->n; ++i) {
        BurstDev &B = s->hb[i];
        if (const int e = set_tiles(B, ke, s->opts.tile_shear)) return e;
        B.tile_base = total;
        total += B.tiles_x * B.tiles_y;
        max_burst_tiles = std::max(max_burst_tiles, B.tiles_x * B.tiles_y);
        std::memset(&hm[i], 0, sizeof(CUtensorMap));
        B.tmap = make_tmap(B, ke.shape.window, ke.shape.chunk, &hm[i]) == 0 ? i : -1;
    }
    // An earlier pass of the plan may still read the descriptors on a caller's
    // non-blocking stream, which the legacy stream's copies below do not wait
    // for: wait for the device first.  The copies are from pageable memory and
    // may still be in flight when cudaMemcpy returns: wait for them too.
    SCK(cudaDeviceSynchronize());
    SCK(cudaMemcpy(s->d_bursts, s->hb.data(), sizeof(BurstDev) * s->n, cudaMemcpyHostToDevice));
    SCK(cudaMemcpy(s->d_tmaps, hm.data(), sizeof(CUtensorMap) * s->n, cudaMemcpyHostToDevice));
    SCK(cudaStreamSynchronize(0));
    const size_t need = tile_list_bytes(total);
    if (need > s->tiles_cap) {
        cudaFree(s->d_tiles);
        s->d_tiles = nullptr;
        s->tiles_cap = 0;
        const int rc = alloc(&s->d_tiles, need);
        if (rc) return rc;
        s->tiles_cap = need;
    }
    s->total_tiles = total;
    s->max_burst_tiles = max_burst_tiles;
    s->mask_valid = false;
    s->kernel = idx;
    drop_graph(s);
    return SRG_OK;
}

// Burst descriptor of burst i as the kernels see it: the caller's lines, or
// the plan's oversampled copy (2S - 1 samples at dmrg / 2 over the same
// rngstart .. rngend, as srg_oversample_range_device documents).
srg_burst_desc kernel_desc(const srg_scene *s, int i) {
    srg_burst_desc d = s->descs[i];
    if (s->interp == SRG_INTERP_OVERSAMPLED2) {
        d.burst = reinterpret_cast<const float *>(s->os_lines[i]);
        d.ldb = s->os_ld[i];
        d.S = 2 * s->descs[i].S - 1;
        d.dmrg = s->descs[i].dmrg / 2.0;
        d.bin0 = d.nbins = 0;
    }
    return d;
}

// The 2x oversampling of every burst's lines into the plan's copies.
int enqueue_oversample(srg_scene *s, cudaStream_t st) {
    if (s->interp != SRG_INTERP_OVERSAMPLED2) return SRG_OK;
    for (int i = 0; i < s->n; ++i) {
        const srg_burst_desc &d = s->descs[i];
        const int rc = srg_oversample_range_device(d.burst, d.ldb, d.P, d.S,
                                                   reinterpret_cast<float *>(s->os_lines[i]),
                                                   s->os_ld[i], st);
        if (rc) return rc;
    }
    return SRG_OK;
}

int enqueue_centres(srg_scene *s, cudaStream_t st) {
    SCK(launch_line_centres_batch(s->d_bursts, s->d_jobs, s->n, s->total_lines, st));
    return SRG_OK;
}

int enqueue_backprojection(srg_scene *s, cudaStream_t st) {
    if (s->total_tiles == 0) return SRG_OK;
    DevCtx *c = nullptr;
    int rc = get_ctx(s->dev, &c);
    if (rc) return rc;
    const KernelEntry &ke = kKernels[s->kernel];
    ensure_attrs(*c, s->kernel);
    int per_sm = 0;
    SCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ke.fn, ke.shape.threads, ke.smem));
    if (per_sm < 1) return fail(SRG_E_UNSUPPORTED, "kernel shape %d does not fit an SM", s->kernel);
    SCK(cudaMemsetAsync(s->d_flags, 0, sizeof(int), st));
    SCK(launch_tile_list(s->d_bursts, s->n, s->max_burst_tiles, s->total_tiles, ke.shape.tx,
                         ke.shape.ty, s->d_tiles, st));
    s->mask_valid = true;
    SCK(launch_tiles(ke, std::min(s->total_tiles, per_sm * c->sms), ke.smem, st, s->d_bursts, s->n,
                     s->total_tiles, s->d_tmaps, s->d_flags, s->d_flags + 1,
                     static_cast<const int *>(s->d_tiles)));
    return SRG_OK;
}

// the ordered merge into the scene raster, skipping the tiles the last
// backprojection found without a formed pixel
cudaError_t merge(srg_scene *s, cudaStream_t st) {
    const KernelEntry &ke = kKernels[s->kernel];
    const unsigned char *tm =
        s->mask_valid && s->total_tiles > 0 ? tile_list_mask(s->d_tiles, s->total_tiles) : nullptr;
    return launch_merge_scene(s->d_bursts, s->n, s->scene, s->scene_ld, s->scene_lines,
                              s->scene_cols, st, tm, ke.shape.tx, ke.shape.ty);
}

int enqueue_pass(srg_scene *s, cudaStream_t st) {
    int rc = enqueue_centres(s, st);
    if (rc) return rc;
    rc = enqueue_oversample(s, st);
    if (rc) return rc;
    rc = enqueue_backprojection(s, st);
    if (rc) return rc;
    if (s->scene) SCK(merge(s, st));
    return SRG_OK;
}

// Rebuild the kernels' burst table for the plan's interpolation (keeps the
// azimuth-centre pointers and the poll limit) and the shape's tiles.
int rebuild_bursts(srg_scene *s) {
    for (int i = 0; i < s->n; ++i) {
        const double *coef = s->hb[i].coef;
        const unsigned spin = s->hb[i].spin;
        s->hb[i] = make_burst_dev(kernel_desc(s, i), coef);
        s->hb[i].spin = spin;
    }
    s->terms = -1;
    return set_kernel(s, s->kernel);
}

int set_interp(srg_scene *s, int interp) {
    if (interp != SRG_INTERP_LINEAR && interp != SRG_INTERP_OVERSAMPLED2)
        return fail(SRG_E_ARG, "unknown interpolation %d", interp);
    if (interp == s->interp) return SRG_OK;
    if (interp == SRG_INTERP_OVERSAMPLED2) {
        for (int i = 0; i < s->n; ++i)
            if (s->descs[i].bin0 != 0 || (s->descs[i].nbins != 0 && s->descs[i].nbins != s->descs[i].S))
                return fail(SRG_E_UNSUPPORTED, "burst %d: oversampling needs whole lines", i);
        if (s->os_lines.empty()) {
            s->os_lines.assign(s->n, nullptr);
            s->os_ld.assign(s->n, 0);
            for (int i = 0; i < s->n; ++i) {
                const long long ld = 2LL * s->descs[i].S;  // even: 16-byte rows for TMA
                void *p = nullptr;
                const int rc = alloc(&p, sizeof(float2) * (size_t)s->descs[i].P * (size_t)ld);
                if (rc) return rc;
                s->os_lines[i] = static_cast<float2 *>(p);
                s->os_ld[i] = ld;
            }
        }
    }
    s->interp = interp;
    return rebuild_bursts(s);
}

// Tuning results of this process (and, with SRG_TUNE_CACHE naming a file, of
// earlier ones): the best shape per form, interpolation and scene shape.
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

const char *tune_file() {
    const char *f = std::getenv("SRG_TUNE_CACHE");
    return f && *f ? f : nullptr;
}

// Scene shape: the multiset of (pulses / 64, samples / 1024, lines / 64,
// columns / 64) of its bursts, with the form and the interpolation.
std::string tune_key(const srg_scene *s) {
    std::vector<std::string> parts;
    for (int i = 0; i < s->n; ++i) {
        const BurstDev &B = s->hb[i];
        char buf[96];
        snprintf(buf, sizeof buf, "%d/%d/%d/%d", B.P / 64, B.S / 1024, B.nlines / 64,
                 (B.lastpix_eff - B.firstpix + 1) / 64);
        parts.emplace_back(buf);
    }
    std::sort(parts.begin(), parts.end());
    std::string k = "f" + std::to_string(s->opts.form) + ":i" + std::to_string(s->interp) + ":";
    for (const std::string &p : parts) k += p + ",";
    return k;
}

int tune_lookup(const std::string &key) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    if (!g_tune_loaded) {
        g_tune_loaded = true;
        if (const char *f = tune_file()) {
            if (FILE *fp = std::fopen(f, "r")) {
                char key_buf[4096];
                int cfg;
                while (std::fscanf(fp, "%4095s %d", key_buf, &cfg) == 2) g_tune[key_buf] = cfg;
                std::fclose(fp);
            }
        }
    }
    auto it = g_tune.find(key);
    return it == g_tune.end() ? -1 : it->second;
}

void tune_record(const std::string &key, int cfg) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[key] = cfg;
    if (const char *f = tune_file()) {
        if (FILE *fp = std::fopen(f, "a")) {
            std::fprintf(fp, "%s %d\n", key.c_str(), cfg);
            std::fclose(fp);
        }
    }
}

}  // namespace

extern "C" {

int srg_scene_create(const srg_burst_desc *bursts, int n, float *scene, int64_t scene_ld,
                     int scene_lines, int scene_cols, const srg_bp_options *opts,
                     srg_scene **out) {
    if (!out) return fail(SRG_E_ARG, "null output handle");
    *out = nullptr;
    if (!bursts || n < 1) return fail(SRG_E_ARG, "no bursts");
    if (scene && n > 256) return fail(SRG_E_ARG, "scene merge supports at most 256 bursts");
    srg_bp_options o;
    srg_bp_default_options(&o);
    if (opts) o = *opts;
    const KernelEntry *ke = pick_kernel(o.form, o.tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", o.form, o.tile_cfg);
    for (int i = 0; i < n; ++i) {
        int rc = validate_desc(bursts[i]);
        if (rc) return rc;
        if (bursts[i].coef)
            return fail(SRG_E_ARG, "burst %d: a scene plan solves its own azimuth centres (coef must be NULL)", i);
        if (bursts[i].numstatevec < 4 || bursts[i].numstatevec > 4096)
            return fail(SRG_E_ARG, "burst %d: numstatevec %d", i, bursts[i].numstatevec);
    }
    DevCtx *c = nullptr;
    int rc = get_ctx(o.device, &c);
    if (rc) return rc;
    srg_scene *s = new srg_scene();
    s->dev = c->dev;
    s->n = n;
    s->opts = o;
    s->descs.assign(bursts, bursts + n);
    s->scene = reinterpret_cast<float2 *>(scene);
    s->scene_ld = scene_ld;
    s->scene_lines = scene_lines;
    s->scene_cols = scene_cols;
    size_t lines = 0, orbit = 0;
    for (int i = 0; i < n; ++i) {
        lines += (size_t)bursts[i].nlines;
        orbit += 7 * (size_t)bursts[i].numstatevec;
    }
    if ((rc = alloc((void **)&s->d_bursts, sizeof(BurstDev) * n)) ||
        (rc = alloc((void **)&s->d_tmaps, sizeof(CUtensorMap) * n)) ||
        (rc = alloc((void **)&s->d_jobs, sizeof(CentreJob) * n)) ||
        (rc = alloc((void **)&s->d_coef, sizeof(double) * 3 * lines)) ||
        (rc = alloc((void **)&s->d_orbit, sizeof(double) * orbit)) ||
        (rc = alloc((void **)&s->d_flags, 64))) {
        srg_scene_destroy(s);
        return rc;
    }
    std::vector<double> horb(orbit);
    std::vector<CentreJob> jobs(n);
    s->hb.resize(n);
    size_t lo = 0, oo = 0;
    for (int i = 0; i < n; ++i) {
        const srg_burst_desc &d = bursts[i];
        const int k = d.numstatevec;
        std::memcpy(&horb[oo], d.timeorbit, sizeof(double) * k);
        std::memcpy(&horb[oo + k], d.xx, sizeof(double) * 3 * k);
        std::memcpy(&horb[oo + 4 * k], d.vv, sizeof(double) * 3 * k);
        CentreJob &J = jobs[i];
        J.orbit = Orbit{s->d_orbit + oo, s->d_orbit + oo + k, s->d_orbit + oo + 4 * k, k};
        J.cp.tmid = d.tmid;
        for (int q = 0; q < 3; ++q) {
            J.cp.xm[q] = d.xyz_mid[q];
            J.cp.vm[q] = d.vel_mid[q];
        }
        J.cp.wvl = d.wvl;
        J.cp.angc0 = d.angc0;
        J.cp.angc1 = d.angc1;
        J.cp.prf = d.prf;
        J.cp.pi = ref_pi();
        J.coef = s->d_coef + 3 * lo;
        J.line_base = (int)lo;
        s->hb[i] = make_burst_dev(d, J.coef);
        if (o.spin_limit > 0) s->hb[i].spin = (unsigned)o.spin_limit;
        lo += (size_t)d.nlines;
        oo += 7 * (size_t)k;
    }
    s->total_lines = (int)lines;
    if (cudaMemcpy(s->d_orbit, horb.data(), sizeof(double) * orbit, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->d_jobs, jobs.data(), sizeof(CentreJob) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaStreamSynchronize(0) != cudaSuccess) {  // (pageable copies may still be in flight)
        cudaGetLastError();
        srg_scene_destroy(s);
        return fail(SRG_E_CUDA, "plan upload failed");
    }
    rc = set_kernel(s, kernel_index(ke));
    if (rc) {
        srg_scene_destroy(s);
        return rc;
    }
    *out = s;
    return SRG_OK;
}

int srg_scene_run(srg_scene *s, void *stream) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    int rc = cudaSetDevice(s->dev) == cudaSuccess ? SRG_OK : fail(SRG_E_CUDA, "cudaSetDevice");
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (st == nullptr) return enqueue_pass(s, st);  // the legacy stream cannot be captured
    if (!s->graph || s->graph_stream != st) {
        drop_graph(s);
        // make sure attributes and lazily loaded kernels are settled outside capture
        DevCtx *c = nullptr;
        if ((rc = get_ctx(s->dev, &c))) return rc;
        ensure_attrs(*c, s->kernel);
        cudaGraph_t g = nullptr;
        SCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_pass(s, st);
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return fail(SRG_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            s->graph = nullptr;
            return fail(SRG_E_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
        }
        s->graph_stream = st;
    }
    SCK(cudaGraphLaunch(s->graph, st));
    return SRG_OK;
}

int srg_scene_run_stages(srg_scene *s, int stages, void *stream) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = SRG_OK;
    if (stages & 1) rc = enqueue_centres(s, st);
    if (!rc && (stages & 2)) rc = enqueue_oversample(s, st);
    if (!rc && (stages & 2)) rc = enqueue_backprojection(s, st);
    if (!rc && (stages & 4) && s->scene) SCK(merge(s, st));
    return rc;
}

int srg_scene_sync(srg_scene *s, void *stream) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SCK(cudaStreamSynchronize(st));
    int h[2] = {0, 0};
    SCK(cudaMemcpy(h, s->d_flags, sizeof h, cudaMemcpyDeviceToHost));
    if (h[1]) {
        cudaMemsetAsync(s->d_flags + 1, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return fail(SRG_E_TIMEOUT, "device error word 0x%x (TMA wait timed out)", h[1]);
    }
    return SRG_OK;
}

int srg_scene_terms(srg_scene *s, int64_t *terms) {
    if (!s || !terms) return fail(SRG_E_ARG, "bad arguments");
    if (s->terms < 0) {
        DevCtx *c = nullptr;
        int rc = get_ctx(s->dev, &c);
        if (rc) return rc;
        rc = enqueue_centres(s, 0);
        if (rc) return rc;
        unsigned long long *cnt = reinterpret_cast<unsigned long long *>(s->d_flags + 2);
        SCK(cudaMemset(cnt, 0, sizeof(unsigned long long)));
        for (int i = 0; i < s->n; ++i) SCK(launch_count_terms(s->hb[i], cnt, c->sms, 0));
        unsigned long long h = 0;
        SCK(cudaMemcpy(&h, cnt, sizeof h, cudaMemcpyDeviceToHost));
        s->terms = (int64_t)h;
    }
    *terms = s->terms;
    return SRG_OK;
}

int srg_scene_autotune(srg_scene *s, const srg_tune_request *req, srg_tune_result *res) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    srg_tune_request q{};
    q.iters = 3;
    q.use_cache = 1;
    if (req) q = *req;
    if (q.iters < 1) q.iters = 3;
    srg_tune_result r{};
    r.tile_cfg = -1;
    r.ms = -1.0;
    r.err_linear = r.err_oversampled = -1.0;
    cudaStream_t st = nullptr;
    SCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = SRG_OK;
    // Interpolation: the reference's linear interpolation of the original
    // lines when its estimated phase error is within the budget, else the
    // 2x-oversampled lines (srg_interp_error, from a sample of every burst's
    // lines; the error powers of the bursts are averaged).
    if (q.interp_budget > 0.0) {
        double pl = 0.0, po = 0.0;
        for (int i = 0; i < s->n && rc == SRG_OK; ++i) {
            const srg_burst_desc &d = s->descs[i];
            const int S = d.nbins > 0 ? d.nbins : d.S;
            double el = 0.0, eo = 0.0;
            rc = srg_interp_error(d.burst, d.ldb, d.P, S, std::max(4, 64 / s->n), &el, &eo, st);
            pl += el * el;
            po += eo * eo;
        }
        if (rc == SRG_OK) {
            r.err_linear = std::sqrt(pl / s->n);
            r.err_oversampled = std::sqrt(po / s->n);
            rc = set_interp(s, r.err_linear <= q.interp_budget ? SRG_INTERP_LINEAR
                                                               : SRG_INTERP_OVERSAMPLED2);
        }
    }
    r.interp = s->interp;
    // The shape: every compiled shape of the form is timed, unless the cache
    // holds the best shape of a scene of the same sizes.  The tile shear
    // (rectangular tiles or the geometric shear) is timed on every call: it
    // pays or costs by the terrain (a tile's range window grows with the
    // relief it covers), which the cache key does not see.
    const std::string key = rc == SRG_OK ? tune_key(s) : std::string();
    const int cached = rc == SRG_OK && q.use_cache ? tune_lookup(key) : -1;
    const bool from_cache =
        cached >= 0 && cached < kNumKernels && kKernels[cached].form == s->opts.form;
    const int shear0 = s->opts.tile_shear;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    bool centres_done = false;
    int best = -1, best_shear = 0;
    float best_t = 1e30f;
    for (int idx = 0; idx < kNumKernels && rc == SRG_OK; ++idx) {
        if (from_cache ? idx != cached : kKernels[idx].form != s->opts.form) continue;
        // shear candidates: rectangular tiles, and the geometric shear where
        // it shears a burst
        bool geo = false;
        for (int i = 0; i < s->n && kKernels[idx].shears && !geo; ++i) {
            BurstDev probe = s->hb[i];
            geo = set_tiles(probe, kKernels[idx], SRG_TILE_SHEAR_AUTO) == SRG_OK && probe.shear != 0;
        }
        if (from_cache && !geo) {  // nothing to time
            best = idx;
            break;
        }
        for (const int shear : {0, SRG_TILE_SHEAR_AUTO}) {
            if (shear != 0 && !geo) continue;
            s->opts.tile_shear = shear;
            if ((rc = set_kernel(s, idx))) break;
            if (!centres_done) {
                if ((rc = enqueue_centres(s, st)) || (rc = enqueue_oversample(s, st))) break;
                if (cudaStreamSynchronize(st) != cudaSuccess) {
                    rc = fail(SRG_E_CUDA, "azimuth centres failed: %s",
                              cudaGetErrorString(cudaGetLastError()));
                    break;
                }
                centres_done = true;
            }
            if ((rc = enqueue_backprojection(s, st))) break;  // warm-up
            float tot = 0.f;
            for (int it = 0; it < q.iters && rc == SRG_OK; ++it) {
                cudaEventRecord(e0, st);
                rc = enqueue_backprojection(s, st);
                cudaEventRecord(e1, st);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                tot += ms;
            }
            if (rc) break;
            const float t = tot / q.iters;
            if (t < best_t) {
                best_t = t;
                best = idx;
                best_shear = shear;
            }
        }
    }
    if (rc == SRG_OK && cudaStreamSynchronize(st) != cudaSuccess)
        rc = fail(SRG_E_CUDA, "tuning launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (rc || best < 0) {
        s->opts.tile_shear = shear0;
        if (rc) return rc;
        return fail(SRG_E_UNSUPPORTED, "no kernel shape of form %d", s->opts.form);
    }
    s->opts.tile_shear = best_shear;
    rc = set_kernel(s, best);
    if (rc) return rc;
    s->opts.tile_cfg = best;
    if (!from_cache) tune_record(key, best);
    r.tile_cfg = best;
    r.tile_shear = best_shear;
    r.from_cache = from_cache ? 1 : 0;
    r.ms = best_t < 1e30f ? best_t : -1.0;
    if (res) *res = r;
    return SRG_OK;
}

int srg_scene_tune(srg_scene *s, int iters, int *best_cfg, double *best_ms) {
    srg_tune_request q{};
    q.iters = iters;
    q.use_cache = 1;
    srg_tune_result r{};
    const int rc = srg_scene_autotune(s, &q, &r);
    if (rc) return rc;
    if (best_cfg) *best_cfg = r.tile_cfg;
    if (best_ms) *best_ms = r.ms;
    return SRG_OK;
}

int srg_scene_set_interp(srg_scene *s, int interp) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    return set_interp(s, interp);
}

int srg_scene_interp(const srg_scene *s) { return s ? s->interp : -1; }

int srg_scene_set_shape(srg_scene *s, int tile_cfg) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    const KernelEntry *ke = pick_kernel(s->opts.form, tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", s->opts.form, tile_cfg);
    s->opts.tile_cfg = tile_cfg;
    return set_kernel(s, kernel_index(ke));
}

int srg_scene_set_form(srg_scene *s, int form, int tile_cfg) {
    if (!s) return fail(SRG_E_ARG, "null plan");
    const KernelEntry *ke = pick_kernel(form, tile_cfg);
    if (!ke) return fail(SRG_E_ARG, "no kernel for form %d shape %d", form, tile_cfg);
    s->opts.form = form;
    s->opts.tile_cfg = tile_cfg;
    return set_kernel(s, kernel_index(ke));
}

int srg_scene_shape(const srg_scene *s) { return s ? s->kernel : -1; }

int srg_scene_tile_shear(const srg_scene *s, int burst, int *shear) {
    if (!s || !shear || burst < 0 || burst >= s->n) return fail(SRG_E_ARG, "bad arguments");
    *shear = s->hb[burst].shear;
    return SRG_OK;
}

void srg_scene_destroy(srg_scene *s) {
    if (!s) return;
    drop_graph(s);
    for (float2 *p : s->os_lines) cudaFree(p);
    cudaFree(s->d_bursts);
    cudaFree(s->d_tmaps);
    cudaFree(s->d_jobs);
    cudaFree(s->d_coef);
    cudaFree(s->d_orbit);
    cudaFree(s->d_flags);
    cudaFree(s->d_tiles);
    delete s;
}

}  // extern "C"
