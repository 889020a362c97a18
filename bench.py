"""Benchmark of the B200 backprojection (one JSON line on stdout, rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: executed pixel.pulse terms per second (Gpixel.pulses/s), the split
FP32 form being the headline and the plain FP64 form timed on the same scene
beside it, with the split form's phase error against it.  A step is one pass
of the hot path over the workload: the per-line azimuth-centre solve plus the
per-pixel aperture sums of every burst.  `value` is device time (CUDA events
on the launching stream, max over ranks) with inputs resident in HBM; `e2e`
goes through the reference-facing C ABI (azimuth_compress_: host burst
buffer in pinned memory, DEM and .geo files on tmpfs, every host<->device
copy and the .geo merge inside the timed region).  The workload's range
lines are larger than L2, so no flush is needed between steps.

--impl reference times the reference's own CPU backprojection
(sentinel/azimuth_compress_cpu.c compiled from source into oracle/_ref,
OpenMP over all host cores) on whole bursts of the same workload, one burst
per step, built on the host (neither the GPU nor the CUDA library is used).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpixel·pulses/s on 1 B200: split-FP32 vs FP64 form at ≤1 mrad RMS phase error"
UNIT = "Gpixel·pulses/s"
FLOPS_PER_TERM = 29  # fixed convention: 3+5+1+2+1+6+1+2+8 (diff, norm, sqrt, bin, frac, lerp, phase, sincos, cmac)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def load_traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of `kernel` on `workload` from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    try:
        return json.load(open(path)).get(f"{kernel}/{workload}")
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
# our arm


def e2e_dropin(torch, wl, steps, form, separate=False, bursts=None, overlap=0):
    """End to end through azimuth_compress_ (the drop-in C ABI), one call per
    burst in acquisition order as the reference's driver makes them: burst
    lines in pinned host memory, the DEM and the .geo raster as files on tmpfs
    (when it has room, else the temp dir); `separate`: one .geo file per burst
    (a stack of passes) instead of one scene raster; `bursts`: the bursts to
    run (default: all of the workload's); `overlap`: calls overlap (each
    returns once its lines are on the device; srg_dropin_flush at the end of
    every step, inside the timed region, waits for the last merges).  Returns
    (s per step, h2d, d2h bytes per step)."""
    from srg_b200 import api
    api.set_default_form(form, overlap=overlap)
    bursts = wl.bursts if bursts is None else bursts
    if not bursts:
        return 0.0, 0, 0
    b0 = bursts[0].b
    geo_bytes = b0.demlength * b0.demwidth * 8
    dem_bytes = b0.demlength * b0.demwidth * 2
    nfiles = len(bursts) if separate else 1
    tmp = None
    if os.path.isdir("/dev/shm"):
        st = os.statvfs("/dev/shm")
        if st.f_bavail * st.f_frsize > 2 * (nfiles * geo_bytes + dem_bytes):
            tmp = "/dev/shm"
    h2d = d2h = 0
    with tempfile.TemporaryDirectory(dir=tmp) as td:
        dem_path = os.path.join(td, "elevation.dem")
        np.ascontiguousarray(b0.dem, np.int16).tofile(dem_path)
        fd_dem = os.open(dem_path, os.O_RDWR)
        fds = []
        for i in range(nfiles):
            geo_path = os.path.join(td, f"scene{i}.geo")
            with open(geo_path, "wb") as f:
                f.truncate(geo_bytes)
            fds.append(os.open(geo_path, os.O_RDWR))
        fd_of = (lambda i: fds[i]) if separate else (lambda i: fds[0])
        hosts = []
        try:
            for db in bursts:
                host = torch.empty(tuple(db.burst.shape), dtype=torch.complex64, pin_memory=True)
                host.copy_(db.burst)
                hosts.append(host)
            # each call's arguments built once, as a Fortran caller holds them
            calls = [api.prepare_azimuth_compress(db.b, fd_of(i), fd_dem, burst=host.numpy())
                     for i, (db, host) in enumerate(zip(bursts, hosts))]
            for call in calls:   # warm-up; the bytes each call copies, as it reports them
                call()
                h, d = api.dropin_last_bytes()
                h2d += h
                d2h += d
            if overlap:
                # overlapped calls take the device's two drop-in contexts in turn: a
                # second pass gives each context the bursts the first gave the other
                # (its buffers grow to the largest burst before the timed steps)
                for call in calls:
                    call()
            api.dropin_flush()
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_push("e2e_overlapped" if overlap else "e2e_waiting")
            t0 = time.perf_counter()
            for _ in range(steps):
                for call in calls:
                    call()
                api.dropin_flush()
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) / steps
            torch.cuda.nvtx.range_pop()
        finally:
            api.dropin_flush()
            api.set_default_form(form, overlap=0)
            os.close(fd_dem)
            for fd in fds:
                os.close(fd)
            del hosts
    return dt, h2d, d2h


def time_plan(torch, plan, steps, warmup, stream, stages=None, label="timed"):
    """K passes of a scene plan on `stream` (graph replay), or of chosen
    stages; returns ms per pass (CUDA events on the stream).  The timed
    passes sit in an NVTX range named `label` (for ncu --nvtx-include)."""
    sp = stream.cuda_stream
    run = (lambda: plan.run(sp)) if stages is None else (lambda: plan.run_stages(stages, sp))
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    torch.cuda.nvtx.range_push(label)
    for e0, e1 in ev:
        e0.record(stream)
        run()
        e1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    plan.sync(sp)
    return sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps


def stack_interferograms(torch, wl, s_slcs, d_slcs, stream, steps, exchange=None):
    """Crossmul of the stack's sequential pairs (one stack call, timed with
    CUDA events on `stream`), the interferometric phase error of the split
    images against the FP64 images, and of the FP64 interferograms against
    the injected deformation (4 pi / lambda times the pair's range change).
    `exchange` (a stack dealt in blocks over ranks): extends this rank's image
    list by the next block's first image, inside the timed region."""
    from srg_b200 import api
    sp = stream.cuda_stream
    ext = exchange if exchange is not None else (lambda images: list(images))
    with torch.cuda.stream(stream):
        pairs = ext(s_slcs)
    outs = api.crossmul_stack(pairs, stream=sp)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for e0, e1 in ev:
        e0.record(stream)
        with torch.cuda.stream(stream):
            pairs = ext(s_slcs)
        api.crossmul_stack(pairs, stream=sp, sync=False, outs=outs)
        e1.record(stream)
    torch.cuda.synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    with torch.cuda.stream(stream):
        d_pairs = ext(d_slcs)
    igd, _ = api.crossmul_stack(d_pairs, stream=sp)
    igs = torch.stack(outs[0]).to(torch.complex128)
    igd = torch.stack(igd).to(torch.complex128)
    amp = igd.abs()
    rms = torch.sqrt((amp[amp > 0] ** 2).mean())
    m = amp > 0.05 * rms
    ph = torch.angle(igs[m] * igd[m].conj()) * 1e3
    n = wl.extra["acquisitions"]
    want = torch.from_numpy(wl.extra["range_change"]).to(igd.device, torch.float64)
    want = want * (4.0 * np.pi / wl.extra["wvl"] / max(1, n - 1))
    dt = torch.angle(igd * torch.exp(-1j * want)[None]) * 1e3
    return {"ms_per_stack": ms, "pairs": len(outs[0]), "looks": [1, 1],
            "ifg_phase_error_vs_fp64": {"ph_rms_mrad": float(torch.sqrt((ph ** 2).mean())),
                                        "ph_max_mrad": float(ph.abs().max()),
                                        "pixels": int(ph.numel())},
            "injected_deformation_phase_rms_mrad": float(torch.sqrt((want[m[0]] ** 2).mean()) * 1e3),
            "fp64_ifg_vs_injected_deformation_rms_mrad": float(torch.sqrt((dt[m] ** 2).mean()))}


def oversampled_lines(torch, wl, stream):
    """Configuration 2: the config-1 burst on 2x-oversampled range lines
    (8-tap windowed-sinc half samples, then the backprojection's linear
    interpolation on the finer line).  Keeps the plain-line FP64 output for
    the comparison with configuration 1, swaps the workload's bursts for the
    oversampled ones and times the oversampling."""
    from srg_b200 import _lib, api
    plain = []
    for db, c in zip(wl.bursts, wl.coefs):
        api.backproject([db], form=_lib.FORM_FP64, coefs=[c])
        plain.append(db.out.clone())
    api.oversample2(wl.bursts[0], stream=stream.cuda_stream)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bursts = [api.oversample2(db, stream=stream.cuda_stream, sync=False) for db in wl.bursts]
    e1.record(stream)
    torch.cuda.synchronize()
    wl.bursts = bursts
    wl.terms = api.count_terms(bursts)
    wl.description += ("; range lines oversampled 2x (8-tap Hann-windowed sinc half samples) "
                       "before the linear interpolation")
    return {"oversample_ms": e0.elapsed_time(e1), "plain_fp64": plain}


def vs_plain_lines(torch, wl, plain):
    """FP64 images of the oversampled lines against those of the plain lines."""
    from srg_b200 import _lib, api
    api.backproject(wl.bursts, form=_lib.FORM_FP64, coefs=wl.coefs)
    return raster_phase_error(torch, torch.cat([db.out for db in wl.bursts]), torch.cat(plain))


def pinned_h2d_gbs(torch, mib: int = 256, reps: int = 5) -> float:
    """Host-to-device copy bandwidth from pinned memory (GB/s), the bound of
    the end-to-end path, whose step uploads every burst's range lines."""
    n = mib * 1024 * 1024 // 8
    h = torch.ones(n, dtype=torch.complex64).pin_memory()
    d = torch.empty(n, dtype=torch.complex64, device="cuda")
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        d.copy_(h, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    return reps * n * 8 / (e0.elapsed_time(e1) * 1e-3) / 1e9


def raster_phase_error(torch, a, ref):
    a = a.to(torch.complex128)
    r = ref.to(torch.complex128)
    amp = r.abs()
    rms = torch.sqrt((amp[amp > 0] ** 2).mean())
    m = amp > 0.05 * rms
    ph = torch.angle(a[m] * r[m].conj()) * 1e3
    ar = (a[m].abs() - amp[m]).abs() / amp[m]
    return {"ph_rms_mrad": float(torch.sqrt((ph ** 2).mean())), "ph_max_mrad": float(ph.abs().max()),
            "amp_rel_rms": float(torch.sqrt((ar ** 2).mean())), "pixels": int(ph.numel())}


# ---------------------------------------------------------------------------
# reference (CPU) arm


class quiet_stdout:
    """Silence C-level stdout (the reference prints its line limits) so that
    the JSON line stays the only output."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        __import__("ctypes").CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def combine_ranks(torch, dist, device, maxes, sums):
    """Max over ranks of `maxes` and sum over ranks of `sums` (lists of
    numbers); identity without a process group (dist None)."""
    if dist is None:
        return list(maxes), list(sums)
    t = torch.tensor([float(x) for x in maxes], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([float(x) for x in sums], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return t.tolist(), u.tolist()


WORKLOADS = {
    "c1": ("IW1 burst 1500x21000 complex64 -> 2400x1200 grid at 1e-4 deg, volcano DEM "
           "(0-2500 m cone + fBm, Hurst 0.8, 30 m RMS)", 1),
    "c2": ("IW1 burst 1500x21000 complex64 on 2x-oversampled range lines (8-tap windowed sinc) "
           "-> 2400x1200 grid at 1e-4 deg, volcano DEM", 1),
    "c3": ("IW scene: 3 subswaths x 9 bursts (P 1380-1620, S 18000/21500/25600 complex64), "
           "sub-grids 2000-2600 x 1000-1300 at 1e-4 deg on a shared 16504x6646 volcano DEM, "
           "merged in burst order", 27),
    "c4": ("repeat-pass stack: 32 passes of 1500x21000 complex64 onto a common 2400x1200 grid "
           "at 1e-4 deg, perpendicular baselines U[+-150 m], along-track U[+-5 m], Mogi source "
           "3 km deep, 10 cm max LOS; then crossmul of 31 sequential pairs", 32),
}
STEPS = {
    "c3": "one pass over the scene: azimuth centres of every line, work list of the tiles with "
          "a formed pixel, one persistent backprojection launch for all bursts, ordered merge "
          "into the scene raster",
    "c4": "one pass over the stack: azimuth centres of every pass, work list, one persistent "
          "backprojection launch for all passes onto the common grid",
    "c1": "one pass over the burst: azimuth centres of every line, work list, one "
          "backprojection launch",
    "c2": "one pass over the burst: azimuth centres of every line, work list, one "
          "backprojection launch (lines oversampled once, beforehand)",
}


def workload_config(workload: str, world: int) -> dict:
    """The `config` of the JSON line, identical in both arms."""
    desc, nb = WORKLOADS[workload]
    if world == 1:
        par = "1 GPU"
    elif workload == "c3":
        par = (f"scene partition over {world} GPUs: bursts dealt by estimated terms (LPT), "
               "ordered merge of the ranks' rasters in burst order")
    else:
        par = f"replicas x{world} (one workload per GPU)"
    return {"workload": desc, "bursts": nb, "step": STEPS[workload],
            "l2": "range lines of every burst > 126 MB L2; no flush between steps",
            "parallelism": par}


def host_bursts(workload: str):
    """The workload's bursts on the host for the CPU runs, built without the
    GPU or the CUDA library: the same geometry as the device workload (orbit,
    grid, volcano DEM synthesised with numpy), range lines drawn per burst by
    ``scene.host_clutter_samples`` when a burst is used.  Returns a list of
    (burst, sample seed, line length)."""
    from srg_b200 import scene
    if workload == "c3":
        _, bursts = scene.iw_scene(seed=1003)   # acquisition order, host DEM
        return [(b, 1003 * 100 + i, b.samples) for i, b in enumerate(bursts)]
    seed = {"c1": 1001, "c2": 1001, "c4": 1004}[workload]
    b = scene.config1_geometry(seed=seed)
    if workload == "c2":   # the 2x-oversampled line: 2S - 1 samples at dmrg / 2
        b.dmrg = b.dmrg / 2.0
        return [(b, seed, 2 * b.samples - 1)]
    return [(b, seed, b.samples)]


def reference_cpu(workload: str, steps: int, warmup: int):
    """Time the reference CPU backprojection (sentinel/azimuth_compress_cpu.c
    compiled from source, unmodified, in oracle/_ref; OpenMP over every host
    core) end to end through its 33-argument entry, one whole burst per step
    (the workload's bursts in acquisition order, cycling), with DEM and .geo
    files on tmpfs.  Terms per burst come from the oracle's exact count
    (liboracle.so, the reference's window and range test), outside the timed
    call.  Neither the GPU nor the CUDA library is touched.  Returns
    (terms/s over the timed steps, cores, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    import oracle as O
    from srg_b200 import scene
    ref, orc = O.RefCPU(), O.Oracle()
    bursts = host_bursts(workload)
    tmp = "/dev/shm" if os.path.isdir("/dev/shm") else None
    terms_tot, secs_tot, used = 0, 0.0, []
    for step in range(warmup + steps):
        k = step % len(bursts)
        b, seed, S = bursts[k]
        scene.host_clutter_samples(b, seed, samples=S)
        with quiet_stdout():
            timing = {}
            O.run_33_files(ref.lib.azimuth_compress_cpu_, b, timing=timing, tmpdir=tmp,
                               read_back=False)
        if step >= warmup:
            terms_tot += orc.count_terms(b, nthreads=cores)
            secs_tot += timing["call_s"]
            used.append(k)
        b.burst = np.zeros((0, S), np.complex64)   # free the lines
    desc = (f"reference azimuth_compress_cpu_ (OpenMP, {cores} threads) end to end on whole "
            f"bursts {used} of the workload, one per step ({terms_tot} terms, {secs_tot:.1f} s)")
    return terms_tot / secs_tot, cores, desc, secs_tot / max(1, len(used))


# ---------------------------------------------------------------------------
# profiling driver


def profile_shapes(torch, workload: str, shapes, samples: str = "random", seed=None,
                   tile_shear=None):
    """A fixed workload and a list of kernel shapes: one warm-up launch, then
    one measured launch per shape, nothing else on the GPU (the command line
    of the committed ncu summaries).  c1: one IW1-sized burst (random or
    forward-projected samples); c3: the 27-burst IW scene, azimuth centres
    and backprojection stages of its scene plan.  Under ncu, select the
    backprojection kernels by name (regex:bp_) and skip the warm-up launches
    with -s <number of shapes>.  tile_shear: srg_bp_options.tile_shear (None:
    the default, rectangular tiles)."""
    from srg_b200 import _lib, api, scene, workloads
    cfgs = _lib.tile_configs()
    if workload == "c3":
        wl = workloads.config3(seed=1003 if seed is None else seed)
        plan = wl.plan if tile_shear is None else api.Scene(wl.bursts, raster=None,
                                                             tile_shear=tile_shear)
        for rep in range(2):  # warm-up, then measured
            for s in shapes:
                plan.set_form(cfgs[s][1], s)
                plan.run_stages(1 | 2, 0)
        plan.sync(0)
        return
    seed = 1001 if seed is None else seed
    if samples == "forward":
        wl = workloads.config1(seed=seed)
        db, coef = wl.bursts[0], wl.coefs[0]
    else:
        b = scene.config1_geometry(seed=seed)
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        bt = torch.complex(torch.randn(b.rawdatalines, b.samples, device="cuda", generator=g),
                           torch.randn(b.rawdatalines, b.samples, device="cuda", generator=g))
        db = api.to_device(b, burst_tensor=bt)
        coef = api.line_centres(db)
    for rep in range(2):  # warm-up, then measured
        for s in shapes:
            api.backproject([db], form=cfgs[s][1], tile_cfg=s, coefs=[coef],
                            tile_shear=tile_shear)
    torch.cuda.synchronize()


def hbm_peak_gbs():
    """(HBM copy bandwidth in GB/s, where it comes from): the measured figure of
    MEASURED_PEAKS.json when present, else the pool's earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (6.65 TB/s, an earlier measurement on this pool)"


def range_compression_bench(torch, steps: int, warmup: int):
    """Range compression of one IW1-sized burst of decoded lines on the device
    (sentinel/processsub.f90:86-123: each line times the conjugate chirp
    replica spectrum over 32,768-point FFTs, whose kept samples the library
    forms by overlap-save with 8,192-point segments in one fused kernel;
    srg_range_compress_device): 1,500
    lines of 24,000 complex64 samples, seeded Gaussian samples (the timing does
    not depend on them), the IW pulse of the tests (64.3 MHz sampling, 52.4 us,
    0.7792 MHz/us).  Lines resident in HBM; a step compresses the burst once.
    Algorithmic bytes: every input sample read once and every output sample
    written once.  CPU baseline: the oracle's numpy restatement (one thread)
    on 32 lines (parity of the two is tests/test_rangecomp.py's)."""
    from srg_b200 import api
    fs = float(np.float32(3.0 / 7.0 * 4.0 * 37.53472224))
    pulse = dict(samplefreq=fs, startfreq=-20.2, ramprate=0.7792, pulselength=52.4)
    nlines, nsamps = 1500, 24000
    g = torch.Generator(device="cuda")
    g.manual_seed(1005)
    lines = torch.complex(torch.randn((nlines, nsamps), device="cuda", generator=g),
                          torch.randn((nlines, nsamps), device="cuda", generator=g))
    _, npts = api.range_replica(**pulse)
    nvalid = nsamps - npts
    out = torch.empty((nlines, nvalid), dtype=torch.complex64, device="cuda")
    st = torch.cuda.Stream()
    for _ in range(warmup):
        api.range_compress(lines, **pulse, out=out, stream=st.cuda_stream, sync=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        api.range_compress(lines, **pulse, out=out, stream=st.cuda_stream, sync=False)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    alg_bytes = nlines * (nsamps + nvalid) * 8
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    peak, peak_src = hbm_peak_gbs()
    # the CPU baseline leg: the oracle's restatement on a sample of the lines
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import rangecomp as orc
    sample = lines[:32].cpu().numpy()
    t0 = time.perf_counter()
    orc.range_compress(sample, **pulse)
    cpu_s = time.perf_counter() - t0
    line = {
        "metric": "range-compressed lines/s (IW1 burst, the 32,768-point matched filter)",
        "workload": "rc",
        "value": nlines / (ms * 1e-3), "unit": "lines/s", "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "c64 (f32)",
        "data": "synthetic, seeded Gaussian decoded lines",
        "config": {"workload": "range compression of one IW1-sized burst: 1500 lines x 24000 "
                               f"complex64 samples, replica of {npts} points; the kept samples "
                               "of the 32768-point filter, formed by overlap-save with "
                               "8192-point segments in one fused kernel",
                   "l2": "lines (288 MB) > 126 MB L2; no flush between steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                     "bytes_per_line": (nsamps + nvalid) * 8},
        "cpu_baseline": {"value": len(sample) / cpu_s, "unit": "lines/s", "cores": 1,
                         "kind": "port", "sample": "oracle numpy restatement, 32 lines"},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "rc"],
                    help="c1-c4: backprojection workloads; rc: range compression of one burst")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shapes", default=None,
                    help="SPLIT,FP64 kernel shape indices (srg_tile_config; -1: the form's "
                         "default shape); default: tuned")
    ap.add_argument("--profile-shapes", default=None,
                    help="comma-separated kernel shape indices: run the profiling driver on "
                         "--workload c1 or c3 instead of the benchmark")
    ap.add_argument("--tile-shear", default=None,
                    help="with --profile-shapes: tile shear, lines per 32 columns, or 'auto' "
                         "(the geometric choice); default rectangular tiles")
    ap.add_argument("--samples", default="random", choices=["random", "forward"],
                    help="profiling driver, c1: random or forward-projected range lines")
    ap.add_argument("--e2e-only", default=None, choices=["overlapped", "waiting"],
                    help="only the drop-in end to end on --workload c1, c3 or c4, calls "
                         "overlapped or waiting (NVTX ranges e2e_overlapped / e2e_waiting); not "
                         "for ncu: its serialised launches hold the range lines of the gated "
                         "kernel back")
    args = ap.parse_args()
    if args.profile_shapes is not None:
        import torch
        from srg_b200 import _lib
        shear = (None if args.tile_shear is None else _lib.TILE_SHEAR_AUTO
                 if args.tile_shear == "auto" else int(args.tile_shear))
        profile_shapes(torch, args.workload, [int(x) for x in args.profile_shapes.split(",")],
                       args.samples, tile_shear=shear)
        print("ok", args.profile_shapes)
        return
    if args.workload == "rc":
        import torch
        range_compression_bench(torch, max(1, args.steps), max(1, args.warmup))
        return
    if args.e2e_only is not None:
        import torch
        from srg_b200 import _lib, workloads
        wl = {"c1": workloads.config1, "c3": workloads.config3,
              "c4": workloads.config4}[args.workload]()
        dt, h2d, d2h = e2e_dropin(torch, wl, max(1, args.e2e_steps), _lib.FORM_SPLIT,
                                  separate=args.workload == "c4",
                                  overlap=1 if args.e2e_only == "overlapped" else 0)
        print(json.dumps({"e2e_only": args.e2e_only, "workload": args.workload,
                          "s_per_step": dt, "value": wl.terms / dt / 1e9, "unit": UNIT,
                          "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}))
        return
    pinned = [int(x) for x in args.shapes.split(",")] if args.shapes else None
    rank, world, local = dist_env()
    config = workload_config(args.workload, world)
    if args.impl == "reference":
        if rank != 0:
            return  # the reference arm runs on rank 0 only
        # host only: neither torch.cuda nor the CUDA library is loaded here
        value, cores, sample, s_step = reference_cpu(args.workload, max(1, args.steps), args.warmup)
        value /= 1e9
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": s_step * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    from srg_b200 import _lib, workloads

    build = {"c1": workloads.config1, "c2": workloads.config1, "c3": workloads.config3,
             "c4": workloads.config4}[args.workload]
    # N > 1, the IW scene: one scene partitioned over the ranks (every rank
    # builds the same scene); the repeat-pass stack: its acquisitions dealt in
    # date-order blocks; the one-burst workloads: one replica per rank
    partitioned = world > 1 and args.workload == "c3"
    stack_blocks = world > 1 and args.workload == "c4"
    wl = build(device=f"cuda:{local}",
               seed={"c1": 1001, "c2": 1001, "c3": 1003, "c4": 1004}[args.workload] +
               (0 if partitioned or stack_blocks else rank))
    if partitioned:
        from srg_b200 import api, partition
        weights = [api.count_terms([db]) for db in wl.bursts]
        wl.plan.close()   # the one-rank plan gives way to this rank's share
        wl.plan = partition.PartitionedScene(wl.bursts, wl.raster, rank, world, dist, weights,
                                             _lib.FORM_SPLIT)
        own_bursts, terms_rank = wl.plan.mine, int(wl.plan.own_weight())

    exchange = None
    if stack_blocks:
        from srg_b200 import api, partition
        block = partition.block_partition(len(wl.bursts), world)[rank]
        own_bursts = [wl.bursts[i] for i in block]
        wl.plan.close()   # the whole-stack plan gives way to this rank's block
        wl.plan = api.Scene(own_bursts, raster=None, form=_lib.FORM_SPLIT)
        terms_rank = wl.plan.terms()
        recv = torch.empty_like(own_bursts[0].out)

        def exchange(images):
            """This rank's images and, but on the last rank, the next block's
            first (the pair across the block's end)."""
            nxt = partition.exchange_boundary(images[0], recv, rank, world, dist)
            return list(images) + ([nxt] if nxt is not None else [])

    stream = torch.cuda.Stream()
    c2 = oversampled_lines(torch, wl, stream) if args.workload == "c2" else None
    if not partitioned and not stack_blocks:
        own_bursts, terms_rank = wl.bursts, wl.terms
    fp32_peak = _lib.measure_fma_peak(False)
    fp64_peak = _lib.measure_fma_peak(True)
    tuned = {}
    ifg = None
    if getattr(wl, "plan", None) is None:  # single bursts: a plan without a scene raster
        from srg_b200 import api
        wl.plan = api.Scene(wl.bursts, raster=None, form=_lib.FORM_SPLIT)
    plan = wl.plan
    if pinned:
        plan.set_form(_lib.FORM_SPLIT, pinned[0])
        tuned["split"] = (plan.shape(), None)
    else:
        tuned["split"] = plan.tune(iters=2)
    split_shears = sorted(set(plan.tile_shears()))
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        s_ms = time_plan(torch, plan, args.steps, args.warmup, stream, label="timed_split")
        if world > 1:
            dist.barrier()
    s_kern = time_plan(torch, plan, args.steps, 1, stream, stages=2)
    if wl.raster is not None:
        split_out = wl.raster.clone()
    else:
        split_out = torch.stack([db.out for db in own_bursts])
    if pinned:
        plan.set_form(_lib.FORM_FP64, pinned[1])
        tuned["fp64"] = (plan.shape(), None)
    else:
        plan.set_form(_lib.FORM_FP64)
        tuned["fp64"] = plan.tune(iters=1)
    d_ms = time_plan(torch, plan, max(3, args.steps // 3), 1, stream)
    d_kern = d_ms
    if wl.raster is not None:
        perr = raster_phase_error(torch, split_out, wl.raster) if rank == 0 else None
    else:
        fp64_out = torch.stack([db.out for db in own_bursts])
        perr = raster_phase_error(torch, split_out, fp64_out)
        if "range_change" in wl.extra:
            ifg = stack_interferograms(torch, wl, list(split_out), list(fp64_out), stream,
                                       max(3, args.steps), exchange=exchange)
        del fp64_out
    del split_out
    plan.set_form(_lib.FORM_SPLIT, tuned["split"][0])
    # azimuth centres, work-list mask and compaction, backprojection (and the
    # ordered merge): one graph per pass
    launches = 5 if wl.raster is not None else 4
    if partitioned:   # own plan (4) and, on rank 0, one merge per burst
        launches = (4 if own_bursts else 0) + (len(wl.bursts) if rank == 0 else 0)
    if c2 is not None:
        c2["vs_config1_fp64"] = vs_plain_lines(torch, wl, c2.pop("plain_fp64"))
    # the drop-in with its calls overlapped (SRG_DROPIN_OVERLAP), and with every
    # call returning after its merge, as the reference's does; the headline
    # overlaps them where a step makes more than one call (one call has
    # nothing to overlap with)
    e2e_ov_s, h2d, d2h = e2e_dropin(torch, wl, args.e2e_steps, _lib.FORM_SPLIT,
                                    separate=args.workload == "c4", bursts=own_bursts, overlap=1)
    e2e_seq_s, _, _ = e2e_dropin(torch, wl, args.e2e_steps, _lib.FORM_SPLIT,
                                 separate=args.workload == "c4", bursts=own_bursts, overlap=0)
    h2d_gbs = pinned_h2d_gbs(torch)
    # whole job: the slowest rank's times, every rank's terms and bytes
    (s_ms, d_ms, e2e_ov_s, e2e_seq_s), (terms_all, h2d, d2h) = combine_ranks(
        torch, dist if world > 1 else None, "cuda", [s_ms, d_ms, e2e_ov_s, e2e_seq_s],
        [terms_rank, h2d, d2h])
    overlapped = len(wl.bursts) > 1
    e2e_s = e2e_ov_s if overlapped else e2e_seq_s
    terms_all, h2d, d2h = int(terms_all), int(h2d), int(d2h)
    value = terms_all / (s_ms * 1e-3) / 1e9
    fp64_value = terms_all / (d_ms * 1e-3) / 1e9
    achieved = FLOPS_PER_TERM * terms_rank / (s_kern * 1e-3) / 1e12
    traffic = load_traffic("bp_split", wl.name)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(
            os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")):
        # a bounded sample: one whole burst per subswath (c3) or the burst
        v, cores, sample, _ = reference_cpu(args.workload, 3 if args.workload == "c3" else 1, 0)
        cpu = {"value": v / 1e9, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": s_ms, "higher_is_better": True,
        "scaling": "strong" if partitioned or stack_blocks else "weak",
        "vs_baseline": None, "dtype": "f32 (split; FP64 orbit/ECEF/reference range)",
        "data": {"c3": "synthetic, seeded: complex Gaussian clutter + forward-projected point targets",
                 "c4": "synthetic, seeded: forward-projected scatterers + point targets, Mogi "
                       "deformation, repeat-pass baselines",
                 "c1": "synthetic, seeded: forward-projected scatterers",
                 "c2": "synthetic, seeded: forward-projected scatterers"}[args.workload],
        "config": config,
        "workload_detail": wl.description,
        "terms_per_step": terms_all,
        "kernel_shapes": {k: _lib.tile_config_name(v[0]) for k, v in tuned.items()},
        "tile_shear_split": split_shears,
        "fp64_form": {"value": fp64_value, "ms_per_step": d_ms, "kernel_ms": d_kern,
                      "split_over_fp64": value / fp64_value},
        "phase_error_vs_fp64": perr,
        **({"oversampled_lines": c2} if c2 is not None else {}),
        **({"crossmul": ifg} if ifg is not None else {}),
        "roofline": {"bound": "fp32-issue", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": traffic, "flops_per_term": FLOPS_PER_TERM,
                     "peak_source": "measured in-run: FFMA-chain kernel (srg_measure_fma_peak)",
                     "fp64_peak": fp64_peak,
                     "fp64_form_frac_of_fp64_peak": FLOPS_PER_TERM * terms_rank / (d_kern * 1e-3) / 1e12 / fp64_peak,
                     "kernel_ms": s_kern},
        "cpu_baseline": cpu,
        "e2e": {"value": terms_all / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "s_per_step": e2e_s,
                "pinned_h2d_gbs": h2d_gbs,
                "h2d_bound_s_per_step": h2d / world / (h2d_gbs * 1e9),
                "path": "azimuth_compress_ (33-arg C ABI), pinned host burst, tmpfs DEM/.geo"
                        + (", calls overlapped (SRG_DROPIN_OVERLAP=1: a call returns once its "
                           "lines are on the device; srg_dropin_flush ends every step)"
                           if overlapped else ", one call per step (not overlapped)")
                        + (" (one .geo per pass)" if args.workload == "c4" else ""),
                "calls_overlapped": {"value": terms_all / e2e_ov_s / 1e9, "s_per_step": e2e_ov_s},
                "calls_not_overlapped": {"value": terms_all / e2e_seq_s / 1e9,
                                         "s_per_step": e2e_seq_s}},
        "gpu_launches": launches * args.steps,
        "clocks": clk.summary(),
        "setup_s": wl.setup_s,
    }
    print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
