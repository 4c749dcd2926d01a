"""Benchmark of the B200 heliostat-field tracer: rays/s on the 1000-heliostat field.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload mid|small|large] [--impl b200|reference]

One step = one pass of the hot path over one batch: aim the field for the
step's sun position, rebuild the grid, the per-heliostat occluder
candidates and the per-point candidate masks on the GPU, trace 2^28 rays (Buie sampling, shadow and block tests,
receiver deposition), scale the flux map and smooth the count map (trimmed
mean).  Every step uses a fresh Philox stream
and a slightly moved sun, so no output or geometry is reused.  Under torchrun
each rank traces its own 2^28 rays (weak scaling) and the count/energy maps
are summed across ranks with one NCCL all-reduce per step (the only exchange
the path has).

`--impl reference` times the reference algorithm's CPU implementation (the
FP64 oracle port, all host cores) on a bounded sample of the same workload.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "rays/s (shadow+block+hit)"
UNIT = "rays/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="mid", choices=["small", "mid", "large"])
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU work budget of the oracle sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--rays", type=int, default=0, help="override rays per step (profiling runs; multiple of 256)")
    ap.add_argument("--variant", type=int, default=0, help="trace kernel variant (qmcrt_trace_params.kernel_variant)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-versus-sequential section")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint section")
    ap.add_argument("--cell", type=float, default=0.0, help="override the grid cell size (m; the coarse cell of a two-level grid)")
    ap.add_argument("--fine-div", type=int, default=-1, help="override the two-level grid split (1 = one level)")
    ap.add_argument("--sun-elev", type=float, default=None, help="override the sun elevation (degrees)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ------------------------------------------------------------------ oracle
def oracle_sample(w, seconds, threads=0):
    """Time the FP64 oracle on ray ranges spread over the whole field."""
    from oracle import oracle as O
    # the oracle walks one uniform grid with the fine cell size
    cell = w.grid.cell[0] / max(w.grid.fine_div, 1)
    sc = O.Scene(w.pos, w.size, w.sigma, w.receiver, cell, w.grid.margin, list(w.sun.dir), aim=w.aim)
    rpp = w.params.rays_per_point
    total = int(w.params.rays)
    xz, helio = O.points_poisson(w.size, total // rpp, w.params.point_spacing, w.params.seed)
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    cores = threads or os.cpu_count()

    def run(nranges, per):
        starts = np.linspace(0, total - per, nranges).astype(np.int64)
        st = np.zeros(7, np.uint64)
        t0 = time.perf_counter()
        for b in starts:
            cfg = sc.cfg(w.sun.csr, w.params.seed, total, rpp, xz, helio, weight, threads=cores,
                         ray_begin=int(b), ray_end=int(b) + per)
            r = sc.trace_philox(cfg, records=False, maps=False)
            st += np.array(r["stats"], np.uint64)
        return time.perf_counter() - t0, st

    dt, st = run(16, 4096)
    rate = st[0] / dt
    per = 8192
    nr = int(max(16, min(4096, seconds * rate / per)))
    dt, st = run(nr, per)
    return {"rays_per_s": float(st[0] / dt), "rays": int(st[0]), "seconds": dt, "cores": cores,
            "ranges": nr, "rays_per_range": per, "stats": [int(x) for x in st]}


def flux_rmse(sc, w, p, ranges=512, per=8192):
    """Flux error of the benchmark configuration.

    Monte Carlo: two independent ray sets of the configuration's size (Philox
    items 0 and 1) give maps F0, F1; one map's RMSE is RMS(F0 - F1) / sqrt 2,
    stated in W/m^2 and relative to the peak and to the mean over lit pixels.
    Against the FP64 oracle on identical rays (item 0, the oracle's sun and
    points): `ranges` ray ranges of `per` rays spread over the field, per-ray
    agreement of flags and receiver pixels, and the RMSE of the count map of
    those rays relative to the oracle's RMS count."""
    import torch
    from oracle import oracle as O
    rays = int(p.rays)
    item0 = p.item
    p.item = 0
    r0 = sc.trace(w.sun, p, records=True, stats=False)
    p.item = 1
    r1 = sc.trace(w.sun, p, records=False, stats=False)
    p.item = item0
    f0 = r0["flux"].double()
    f1 = r1["flux"].double()
    mc = float(torch.sqrt(torch.mean((f0 - f1) ** 2) / 2.0))
    mean = 0.5 * (f0 + f1)
    lit = mean > 0
    starts = np.linspace(0, rays - per, ranges).astype(np.int64)
    idx = torch.as_tensor((starts[:, None] + np.arange(per)[None, :]).ravel(), device=r0["flags"].device)
    gf = r0["flags"][idx].cpu().numpy()
    gp = r0["pixel"][idx].cpu().numpy()
    del r0, r1
    cell = w.grid.cell[0] / max(w.grid.fine_div, 1)
    osc = O.Scene(w.pos, w.size, w.sigma, w.receiver, cell, w.grid.margin, list(w.sun.dir), aim=w.aim)
    rpp = p.rays_per_point
    xz, helio = O.points_poisson(w.size, rays // rpp, p.point_spacing, p.seed)
    of = np.empty_like(gf)
    op = np.empty_like(gp)
    oc = np.zeros(w.res[0] * w.res[1], np.float64)
    for i, b in enumerate(starts):
        cfg = osc.cfg(w.sun.csr, p.seed, rays, rpp, xz, helio, threads=os.cpu_count(), ray_begin=int(b),
                      ray_end=int(b) + per)
        r = osc.trace_philox(cfg, records=True, maps=True)
        of[i * per:(i + 1) * per] = r["flags"]
        op[i * per:(i + 1) * per] = r["pixel"]
        oc += r["counts"]
    gc = np.bincount(gp[gp >= 0], minlength=oc.size).astype(np.float64)
    same = (gf == of) & (gp == op)
    return {"mc_rmse_w_m2": mc, "mc_rmse_rel_peak": mc / float(mean.max()),
            "mc_rmse_rel_lit_mean": mc / float(mean[lit].mean()),
            "mc_method": "two independent %d-ray maps (Philox items 0, 1): RMS(F0 - F1) / sqrt 2" % rays,
            "oracle_rays": int(gf.size), "oracle_ray_agreement": float(same.mean()),
            "oracle_rays_differing": int((~same).sum()),
            "oracle_count_map_rmse_rel": float(np.sqrt(np.mean((gc - oc) ** 2)) / np.sqrt(np.mean(oc ** 2))),
            "oracle_method": "%d ray ranges x %d rays spread over the field, identical rays traced by the FP64 "
                             "oracle" % (ranges, per)}


def flops_per_ray(stats):
    """Algorithmic FP32 flops per ray of the reference algorithm: fixed per-ray
    work 192, 30 per traversal set-up (one traversal for shadowed rays, two
    otherwise), 54 per rectangle test and 4 per DDA cell step."""
    rays, shadowed, rect, cells = stats[0], stats[1], stats[5], stats[6]
    return 192.0 + 30.0 * (2.0 - shadowed / rays) + 54.0 * rect / rays + 4.0 * cells / rays


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu_id)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self, window=None):
        """Summary of the samples that arrived within window = (t0, t1) (host
        clock; all samples when none arrived there or no window is given)."""
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        return self.summarise(self.lines, window)

    @staticmethod
    def summarise(lines, window=None):
        """Median SM clock, max clock and the throttle reasons seen in
        (arrival time, csv line) samples of FIELDS, keeping those that arrived
        in window (a sample arrives at most one interval after it was taken)."""
        inside = [ln for ts, ln in lines if window is None or window[0] <= ts <= window[1] + 0.05]
        scope = "timed region"
        if not inside:
            inside, scope = [ln for _, ln in lines], "whole run (no sample inside the timed region)"
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "scope": scope}


# ------------------------------------------------------------------ arms
def reference_arm(a, rank, world):
    if rank != 0:
        return
    from onemirror_b200 import workloads as W
    w = W.BUILDERS[a.workload]()
    per_step = max(1.0, 60.0 / max(1, a.steps + a.warmup))
    for _ in range(a.warmup):
        oracle_sample(w, min(per_step, 2.0))
    vals, rays, secs = [], 0, 0.0
    for _ in range(a.steps):
        r = oracle_sample(w, per_step)
        vals.append(r["rays_per_s"])
        rays += r["rays"]
        secs += r["seconds"]
    v = rays / secs
    sample = ("%d ray ranges x %d rays spread over the %s field's %d rays per step (FP64 oracle, %d threads)"
              % (r["ranges"], r["rays_per_range"], a.workload, int(w.params.rays), r["cores"]))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * secs / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(w), "rays_per_step": int(w.params.rays)},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_section(reps=3):
    """The batched form against sequential plain launches on the equinox day:
    3 fields (300, 1000, 4000 heliostats) x 45 sun positions x 2^24 rays.
    Batched: one captured CUDA graph (aiming, grids, one persistent trace
    kernel, flux scaling) per pass.  Sequential: one qmcrt_trace per item
    (its own aiming, grid, trace and scaling launches) plus a copy of the
    item's flux map out of the scene.  Both timed with CUDA events."""
    import torch
    from onemirror_b200.scene import Batch, SolarScene
    from onemirror_b200 import workloads as W
    fields, suns, items, params = W.batched()
    scenes = [SolarScene.from_workload(f) for f in fields]
    b = Batch(scenes, items, params)
    tuning = b.autotune()
    b.capture()
    b.launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        b.launch()
    e1.record()
    e1.synchronize()
    batched_ms = e0.elapsed_time(e1) / reps
    rays = len(items) * int(params.rays)
    outs = [torch.empty((256, 256), dtype=torch.float32, device="cuda") for _ in items]
    ps = []
    for i in range(len(items)):
        p = W.params(int(params.rays), params.rays_per_point, params.point_spacing, seed=params.seed)
        p.item = i
        ps.append(p)

    def sequential():
        for i, (si, sun) in enumerate(items):
            r = scenes[si].trace(sun, ps[i], stats=False, outputs=seq_out[si])
            outs[i].copy_(r["flux"])

    seq_out = [scenes[k]._outputs(0, False) for k in range(len(scenes))]
    sequential()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        sequential()
    e1.record()
    e1.synchronize()
    seq_ms = e0.elapsed_time(e1) / reps

    # The reference's structure (ray_tracing.cu:23-27): one launch and one
    # device synchronisation per heliostat.  Each heliostat's rays are one
    # range of the item's rays; timed on the host clock for the day's middle
    # sun position on all three fields, then scaled to the 45 positions.
    mid_sun = suns[len(suns) // 2][3]
    ph_out = [scenes[k]._outputs(0, False) for k in range(len(scenes))]
    ph = []
    for k, sc in enumerate(scenes):
        _, helio = sc.read_points()
        bounds = np.concatenate([[0], np.cumsum(np.bincount(helio, minlength=sc.n))]) * params.rays_per_point
        p = W.params(int(params.rays), params.rays_per_point, params.point_spacing, seed=params.seed)
        p.accumulate = 1
        ph.append((sc, bounds, p))

    def per_heliostat():
        for k, (sc, bounds, p) in enumerate(ph):
            for h in range(sc.n):
                p.ray_begin, p.ray_end = int(bounds[h]), int(bounds[h + 1])
                sc.trace(mid_sun, p, stats=False, outputs=ph_out[k])
                torch.cuda.synchronize()

    per_heliostat()
    t0 = time.perf_counter()
    per_heliostat()
    ph_ms = (time.perf_counter() - t0) * 1e3 * len(suns)
    b.close()
    for s in scenes:
        s.close()
    return {"items": len(items), "sun_positions": len(suns), "fields": [f.n for f in fields],
            "rays_per_item": int(params.rays), "batched_ms": batched_ms, "sequential_ms": seq_ms,
            "batched_rays_per_s": rays / (batched_ms * 1e-3), "sequential_rays_per_s": rays / (seq_ms * 1e-3),
            "speedup_vs_sequential": seq_ms / batched_ms,
            "per_heliostat_ms": ph_ms, "speedup_vs_per_heliostat": ph_ms / batched_ms,
            "per_heliostat_launches": sum(f.n for f in fields) * len(suns),
            "per_heliostat_method": "one qmcrt_trace of a heliostat's ray range + device synchronise per heliostat "
                                    "(the reference's launch structure), host clock, the middle sun position on all "
                                    "3 fields x %d positions" % len(suns),
            "tuning": {"chunk_rays": tuning.chunk_rays, "ctas_per_sm": tuning.ctas_per_sm, "tile": tuning.tile}}


def adjoint_section(reps=5):
    """Adjoint cost on the differentiable field (2000 heliostats, 128x128,
    2^26 rays): plain trace, adjoint forward (bilinear deposit + tape + loss)
    and backward, CUDA events after warm-up."""
    import torch
    from onemirror_b200.scene import SolarScene
    from onemirror_b200 import workloads as W
    w = W.differentiable()
    sc = SolarScene(w.pos, w.size, w.receiver, w.grid, sigma=w.sigma, aim=w.aim, tilt=w.extra["tilt"])
    target = torch.as_tensor(w.extra["target"], device="cuda")
    plain_p = W.params(int(w.params.rays), 256, 0.5, seed=w.params.seed)
    outs = sc._outputs(0, False)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    tf, tb, tp = [], [], []
    tape = None  # one tape for all iterations, as an optimisation loop would keep it
    for it in range(reps + 2):
        ev[0].record()
        sc.trace(w.sun, plain_p, stats=False, outputs=outs)
        ev[1].record()
        tape, _, _ = sc.adjoint_forward(w.sun, w.params, target, want_loss=False, flux=False, tape=tape)
        ev[2].record()
        sc.adjoint_backward(tape)
        ev[3].record()
        ev[3].synchronize()
        if it >= 2:
            tp.append(ev[0].elapsed_time(ev[1]))
            tf.append(ev[1].elapsed_time(ev[2]))
            tb.append(ev[2].elapsed_time(ev[3]))
    SolarScene.tape_free(tape)
    sc.close()
    f, b, p = statistics.median(tf), statistics.median(tb), statistics.median(tp)
    return {"heliostats": w.n, "rays": int(w.params.rays), "params": 4 * w.n, "plain_trace_ms": p,
            "adjoint_forward_ms": f, "adjoint_backward_ms": b, "backward_over_forward": b / f,
            "adjoint_over_plain_forward": (f + b) / p}


def workload_name(w):
    return {"small": "100 heliostats 2x2 m, flat 5x5 m receiver 128x128, 409600 rays",
            "mid": "1000 heliostats 10x10 m to 600 m, flat 12x12 m receiver 256x256, 2^28 rays",
            "large": "10000 heliostats 11x11 m to 1300 m, cylinder 8x18 m 512x256, 2^31 rays"}[w.name]


def grid_name(g):
    if g.fine_div > 1:
        return "two-level: %g m coarse / %g m fine cells" % (g.cell[0], g.cell[0] / g.fine_div)
    return "%g m cells" % g.cell[0]


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def read_traffic(name):
    """dram bytes per launch of the trace kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "trace_kernel_%s.md" % name)
    try:
        for ln in open(p):
            if ln.startswith("traffic_bytes_per_launch:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


def b200_arm(a, rank, world, local):
    import torch
    from onemirror_b200 import capi, workloads as W
    from onemirror_b200 import dist as D
    from onemirror_b200.scene import SolarScene, image_smooth

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    w = W.BUILDERS[a.workload](rays=a.rays) if a.rays else W.BUILDERS[a.workload]()
    if a.cell > 0:
        w.grid.cell[:] = [a.cell] * 3
    if a.fine_div >= 0:
        w.grid.fine_div = a.fine_div
    sc = SolarScene.from_workload(w)
    p = w.params
    p.kernel_variant = a.variant
    rays = int(p.rays)
    base_az = 180.0
    sun_elev = a.sun_elev if a.sun_elev is not None else {"small": 45.0, "mid": 30.0, "large": 20.0}[a.workload]
    if a.sun_elev is not None:  # the oracle sample follows the same sun
        w.sun = W.make_sun(sun_elev, base_az, w.sun.dni, w.sun.csr)

    # FP32 issue-rate peak, measured live (best of 5 bursts)
    sink = torch.zeros(8192, device=dev)
    flops = C.c_double()
    best = 0.0
    for it in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        capi.check(capi.lib().qmcrt_fp32_peak_probe(C.c_void_p(sink.data_ptr()), 4096, C.byref(flops),
                                                    C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        e1.record()
        torch.cuda.synchronize()
        if it:
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)

    outs = sc._outputs(rays, False)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def one(k, item, want_stats=False):
        el, az = sun_elev, base_az + 0.01 * k
        sun = W.make_sun(el, az, w.sun.dni, w.sun.csr)
        p.item = item
        r = sc.trace(sun, p, stats=want_stats, outputs=outs)
        sm = image_smooth(r["counts"], w.smooth_radius, w.smooth_ratio, capi.TRIM_SORTED)
        if world > 1:
            D.reduce_maps(r["counts"], r["energy"])  # the one exchange: sum of the ranks' maps
        return r, sm

    for k in range(a.warmup):
        one(k, D.shard_item(rank, 1000 + k))
    r, _ = one(a.warmup, D.shard_item(rank, 5000), want_stats=True)
    gst = r["stats"]
    gpu_stats = [gst.rays, gst.shadowed, gst.blocked, gst.hit, gst.offmap, gst.rect_tests, gst.dda_cells]
    torch.cuda.synchronize()

    # timed region
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local if "CUDA_VISIBLE_DEVICES" not in os.environ else
                       os.environ["CUDA_VISIBLE_DEVICES"].split(",")[local])
    clk.start()
    time.sleep(0.3)  # nvidia-smi's first samples; the summary keeps only the timed region's
    t_begin = time.time()
    step_ms, kern_ms, setup_ms = [], [], []
    for k in range(a.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one(a.warmup + 1 + k, D.shard_item(rank, k))
        e1.record()
        t = sc.timing()
        kern_ms.append(t.trace_kernel_ms)
        setup_ms.append(t.setup_ms)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.stop((t_begin, time.time()))
    total_ms = float(sum(step_ms))
    if world > 1:
        tt = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    value = rays * world * a.steps / (total_ms * 1e-3)

    # end to end through the host-buffer entry point (pinned host memory)
    e2e = None
    if a.e2e_steps > 0:
        pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
               for k, v in (("pos", w.pos), ("size", w.size), ("aim", w.aim)) if v is not None}
        counts = torch.zeros(w.res, dtype=torch.int32).pin_memory().numpy()
        flux = torch.zeros(w.res, dtype=torch.float32).pin_memory().numpy()
        f = capi.Field()
        f.n = w.n
        f.pos, f.size = capi.as_fp(pin["pos"]), capi.as_fp(pin["size"])
        f.aim = capi.as_fp(pin["aim"]) if "aim" in pin else None
        f.sigma = w.sigma
        h2d = sum(v.nbytes for v in pin.values())
        d2h = counts.nbytes + flux.nbytes
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for k in range(a.e2e_steps + 1):
            if k == 1:
                if world > 1:
                    dist.barrier()
                t0 = time.perf_counter()
            sun = W.make_sun(sun_elev, base_az - 0.01 * (k + 1),
                             w.sun.dni, w.sun.csr)
            p.item = D.shard_item(rank, 9000 + k)
            capi.check(capi.lib().qmcrt_trace_host(sc.h, C.byref(f), C.byref(sun), C.byref(p),
                                                   counts.ctypes.data_as(capi.u32p), capi.as_fp(flux), None, stream))
        dt = time.perf_counter() - t0
        if world > 1:
            tt = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            dt = float(tt.item())
        e2e = {"value": rays * world * a.e2e_steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "call": "qmcrt_trace_host"}

    batch = adj = None
    if rank == 0 and world == 1 and a.workload == "mid" and not a.rays:
        if not a.no_batch:
            batch = batch_section()
        if not a.no_adjoint:
            adj = adjoint_section()
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        ob = oracle_sample(w, a.cpu_seconds)
        cpu = {"value": ob["rays_per_s"], "unit": UNIT, "cores": ob["cores"], "kind": "port",
               "sample": "%d ray ranges x %d rays spread over the field (%d rays, %.1f s), FP64 oracle"
                         % (ob["ranges"], ob["rays_per_range"], ob["rays"], ob["seconds"])}
        ref_stats = ob["stats"]
        accuracy = flux_rmse(sc, w, p)
    else:
        ref_stats = None
        accuracy = None
    # Algorithmic flops per ray: the per-ray figure of the reference algorithm
    # (fixed work + traversal set-ups + 54 per rectangle test + 4 per DDA cell)
    # with the oracle's counts of rectangle tests and cells on a sample of the
    # same rays; without the oracle sample, the kernel's own counts.  The
    # kernel's own counts (after culling, or of its occluder candidates) give
    # the flops it executes, reported beside them.
    alg_stats = ref_stats if ref_stats else gpu_stats
    nbar_src = "oracle (reference traversal)" if ref_stats else "gpu (executed)"
    fpr = flops_per_ray(alg_stats)
    exe = flops_per_ray(gpu_stats)
    kern_s = statistics.mean(kern_ms) * 1e-3
    achieved = rays * fpr / kern_s / 1e12
    traffic = read_traffic(a.workload)
    peaks = measured_peaks()
    roof = {"bound": "fp32", "achieved": achieved, "peak": best, "unit": "TFLOP/s", "frac": achieved / best,
            "traffic": traffic, "kernel": "qm::trace_kernel", "kernel_ms": statistics.mean(kern_ms),
            "peak_source": "measured live: FFMA chains (qmcrt_fp32_peak_probe), best of 5",
            "flops_per_ray": fpr, "nbar_source": nbar_src,
            "reference_rect_tests_per_ray": alg_stats[5] / alg_stats[0],
            "reference_dda_cells_per_ray": alg_stats[6] / alg_stats[0],
            "executed_flops_per_ray": exe, "executed_tflops": rays * exe / kern_s / 1e12,
            "executed_frac": rays * exe / kern_s / 1e12 / best,
            "rect_tests_per_ray": gpu_stats[5] / gpu_stats[0], "dda_cells_per_ray": gpu_stats[6] / gpu_stats[0],
            "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
            "hbm_peak_source": "measured copy" if "hbm_gbs" in peaks else "fallback (6.65 TB/s, earlier copy on B200)"}
    if traffic is not None:
        roof["hbm_achieved_gbs"] = traffic / kern_s / 1e9
        roof["hbm_frac"] = roof["hbm_achieved_gbs"] / roof["hbm_peak_gbs"]
    per_step = {"aim": 1, "candidates": 1, "grid_scan": 1, "grid_fill": 1, "grid_cells": 1, "point_masks": 1,
                "trace": 1, "finalize": 1, "smooth": 1}
    if w.grid.fine_div > 1:
        per_step["grid_coarse"] = 1
    launches = sum(per_step.values())
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(w), "rays_per_step_per_gpu": rays, "heliostats": w.n,
                       "parallelism": "ray shards per GPU + NCCL all-reduce of maps" if world > 1 else "1 GPU",
                       "l2": "flushed between timed steps (256 MB write)",
                       "grid": grid_name(w.grid),
                       "step": "aim + occluder candidates + grid build + point masks + trace + flux scaling + trimmed-mean smoothing"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "flux_rmse": accuracy,
            "gpu_launches": launches * a.steps,
            "launches_per_step": per_step,
            "setup_ms": statistics.mean([s for s in setup_ms if s >= 0]) if any(s >= 0 for s in setup_ms) else None,
            "clocks": clocks,
            "batched": batch,
            "adjoint": adj,
            "stats": {"shadowed": gst.shadowed / gst.rays, "blocked": gst.blocked / gst.rays,
                      "hit": gst.hit / gst.rays, "intercept_ratio": gst.intercept_ratio}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sc.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    rank, world, local = dist_env()
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return
    b200_arm(a, rank, world, local)


if __name__ == "__main__":
    main()
