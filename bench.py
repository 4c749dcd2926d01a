"""Benchmark of the B200 heliostat-field tracer: rays/s on the 1000-heliostat field.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload mid|small|large] [--impl b200|reference]

One step = one pass of the hot path over one batch: aim the field for the
step's sun position, rebuild the per-heliostat occluder candidates (and the
grid, where a candidate list overflows) and the per-point candidate masks on
the GPU, trace 2^28 rays (Buie sampling, shadow and block tests,
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
    ap.add_argument("--no-fields", action="store_true", help="skip the small- and large-field sub-blocks")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip the timing of the reference's CUDA build")
    ap.add_argument("--ref-cuda-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--ref-cuda-reps", type=int, default=3, help=argparse.SUPPRESS)
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
STEP = ("aim + occluder candidates + grid build (its passes build only when a candidate list overflows) + point "
        "masks + trace + flux scaling + all-reduce of the maps "
        "(N > 1) + trimmed-mean smoothing of the summed count map; the Poisson sample points depend only on the "
        "mirror sizes and are sampled once per scene, before the timed steps")
SUN_ELEV = {"small": 45.0, "mid": 30.0, "large": 20.0}


def bench_config(w, world):
    """The `config` of both arms' lines (identical for the same workload)."""
    return {"workload": workload_name(w), "rays_per_step_per_gpu": int(w.params.rays), "heliostats": w.n,
            "parallelism": "ray shards per GPU + NCCL all-reduce of maps" if world > 1 else "1 GPU",
            "l2": "flushed between timed steps (256 MB write)", "grid": grid_name(w.grid), "step": STEP}


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
            "config": bench_config(w, world),
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


def adjoint_section(reps=5, check=True):
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
    # the gradients these timings produce, against the FP64 adjoint of the same rays
    err = None
    if check:
        from oracle import oracle as O
        _, loss, flux = sc.adjoint_forward(w.sun, w.params, target, tape=tape)
        ga, gt = sc.adjoint_backward(tape)
        g = np.concatenate([ga.cpu().numpy(), gt.cpu().numpy()], 1)
        gi = sc.grid_info()
        ref = O.Scene(w.pos, w.size, w.sigma, w.receiver, w.grid.cell[0], w.grid.margin, list(w.sun.dir), aim=sc.aim,
                      tilt=sc.tilt, grid_csr=sc.read_grid(), grid_bounds=(list(gi.origin), list(gi.cell), list(gi.dims)))
        sc.sample_points_count = int(w.params.rays) // w.params.rays_per_point
        xz, helio = sc.read_points()
        weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
        cfg = ref.cfg(w.sun.csr, w.params.seed, int(w.params.rays), w.params.rays_per_point, xz, helio, weight)
        pix = (w.receiver.size[0] / w.receiver.res_x) * (w.receiver.size[1] / w.receiver.res_y)
        scale = w.sun.dni * w.params.reflectivity / (w.params.rays_per_point * pix)
        oloss, oenergy, og = ref.adjoint(cfg, w.extra["target"], scale)
        flux = flux.cpu().numpy()
        oflux = oenergy * scale
        err = {"loss_rel": abs(loss - oloss) / oloss, "flux_rel_max": float(np.abs(flux - oflux).max() / oflux.max()),
               "gradients_rel_norm": float(np.linalg.norm(g - og) / np.linalg.norm(og)),
               "column_max_rel": [float(np.abs(g[:, k] - og[:, k]).max() / np.abs(og[:, k]).max()) for k in range(4)],
               "method": "the timed field's loss, flux map and 8000 gradients against the FP64 CPU adjoint of the same "
                         "2^26 rays (oracle/, per-ray central differences with visibility held)"}
    SolarScene.tape_free(tape)
    sc.close()
    f, b, p = statistics.median(tf), statistics.median(tb), statistics.median(tp)
    return {"heliostats": w.n, "rays": int(w.params.rays), "params": 4 * w.n, "plain_trace_ms": p,
            "adjoint_forward_ms": f, "adjoint_backward_ms": b, "backward_over_forward": b / f,
            "adjoint_over_plain_forward": (f + b) / p, "gradient_error_vs_fp64": err}


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


class FieldRun:
    """One workload traced step after step on this rank's GPU: the timed
    device step, and the same step end to end on host buffers."""

    def __init__(self, w, rank, world, dev, flush, sun_elev=None, variant=0):
        from onemirror_b200.scene import SolarScene
        self.w, self.rank, self.world, self.dev, self.flush = w, rank, world, dev, flush
        self.sc = SolarScene.from_workload(w)
        self.p = w.params
        self.p.kernel_variant = variant
        self.rays = int(self.p.rays)
        self.sun_elev = SUN_ELEV[w.name] if sun_elev is None else sun_elev
        self.base_az = 180.0
        self.outs = self.sc._outputs(self.rays, False)

    def sun(self, k):
        from onemirror_b200 import workloads as W
        return W.make_sun(self.sun_elev, self.base_az + 0.01 * k, self.w.sun.dni, self.w.sun.csr)

    def smooth(self, counts):
        from onemirror_b200 import capi
        from onemirror_b200.scene import image_smooth
        return image_smooth(counts, self.w.smooth_radius, self.w.smooth_ratio, capi.TRIM_SORTED)

    def step(self, k, item, want_stats=False, sun=None):
        """Trace with a sun moved by 0.01 deg per step, exchange the maps
        (N > 1), smooth the summed count map.  `sun`: the step's sun, when
        the caller has formed it already."""
        from onemirror_b200 import dist as D
        self.p.item = item
        r = self.sc.trace(sun if sun is not None else self.sun(k), self.p, stats=want_stats, outputs=self.outs)
        _, _, sm = D.step_maps(r["counts"], r["energy"], self.smooth)
        return r, sm

    def timed(self, steps, k0, stages=0):
        """`steps` device-timed steps, L2 flushed before each (outside the
        events); returns per-step ms, and the trace-kernel and setup ms of the
        stages the library timed (`stages`: capi.TIMING_* bits; a timed stage
        adds CUDA events to the step)."""
        import torch
        from onemirror_b200 import capi
        from onemirror_b200 import dist as D
        self.sc.set_timing(stages)
        step_ms, kern_ms, setup_ms = [], [], []
        for k in range(steps):
            # the step's sun and events are formed before the flush, so that the
            # host enqueues the step while the flush runs and the events time the
            # step's device work, not the host's preparation of it (as when
            # steps follow each other without a flush)
            sun, item = self.sun(k0 + k), D.shard_item(self.rank, k)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            self.flush.zero_()
            e0.record()
            self.step(k0 + k, item, sun=sun)
            e1.record()
            if stages & (capi.TIMING_TRACE | capi.TIMING_FINALIZE):
                t = self.sc.timing()
                if t.trace_kernel_ms >= 0:
                    kern_ms.append(t.trace_kernel_ms)
                if t.setup_ms >= 0:
                    setup_ms.append(t.setup_ms)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        self.sc.set_timing(0)
        return step_ms, kern_ms, setup_ms

    def e2e(self, steps):
        """The same step end to end on pinned host buffers, L2 flushed before
        each call (outside the timed span).  One GPU: one qmcrt_results_host
        call (field upload, trace, scaling, smoothing, download of counts,
        flux and smoothed map).  N GPUs: the field upload, qmcrt_trace, the
        map exchange and smoothing, then the download of the summed maps.
        Host clock per step, the slowest rank's total."""
        import torch
        from onemirror_b200 import capi
        from onemirror_b200 import dist as D
        sc, w = self.sc, self.w
        for name in ("pos", "size", "aim"):  # the field the call uploads, from pinned memory
            v = getattr(sc, name)
            if v is not None:
                setattr(sc, name, torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy())
        h2d = sum(getattr(sc, nm).nbytes for nm in ("pos", "size", "aim") if getattr(sc, nm) is not None)
        res = w.res
        if self.world == 1:
            out = {"counts": torch.zeros(res, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                   "flux": torch.zeros(res, dtype=torch.float32).pin_memory().numpy(),
                   "smoothed": torch.zeros(res, dtype=torch.float32).pin_memory().numpy()}
            d2h = sum(v.nbytes for v in out.values())
            call = "qmcrt_results_host (field upload, trace, flux scaling, smoothing, map downloads)"
        else:
            hc = torch.zeros(res, dtype=torch.int64).pin_memory()
            he = torch.zeros(res, dtype=torch.float64).pin_memory()
            hs = torch.zeros(res, dtype=torch.float32).pin_memory()
            d2h = hc.numel() * 8 + he.numel() * 8 + hs.numel() * 4
            call = "qmcrt_scene_set_field + qmcrt_trace + NCCL all-reduce + qmcrt_smooth_trimmed_u32 + map downloads"
        total = 0.0
        for k in range(steps + 1):
            self.flush.zero_()
            torch.cuda.synchronize()
            if self.world > 1:
                import torch.distributed as dist
                dist.barrier()
            t0 = time.perf_counter()
            self.p.item = D.shard_item(self.rank, 9000 + k)
            sun = self.sun(-(k + 1))
            if self.world == 1:
                sc.results_host(sun, self.p, w.smooth_radius, w.smooth_ratio, capi.TRIM_SORTED, capi.SMOOTH_COUNTS,
                                out=out)
            else:
                sc.update_field()
                r = sc.trace(sun, self.p, stats=False, outputs=self.outs)
                c, e, sm = D.step_maps(r["counts"], r["energy"], self.smooth)
                hc.copy_(c, non_blocking=True)
                he.copy_(e, non_blocking=True)
                hs.copy_(sm, non_blocking=True)
                torch.cuda.current_stream().synchronize()
            if k:
                total += time.perf_counter() - t0
        if self.world > 1:
            total = D.max_over_ranks(total, self.dev)
        return {"value": self.rays * self.world * steps / total, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "call": call, "ms_per_step": 1e3 * total / steps,
                "l2": "flushed before each step, outside the timed span"}

    def close(self):
        self.sc.close()


def field_block(name, rank, world, dev, flush, steps, e2e_steps, warmup=3):
    """Throughput of another field at its own configuration (a sub-block of
    the default line): device-timed steps and the end-to-end call."""
    import statistics as S
    from onemirror_b200 import capi
    from onemirror_b200 import workloads as W
    w = W.BUILDERS[name]()
    run = FieldRun(w, rank, world, dev, flush)
    for k in range(warmup):
        run.step(k, 60000 + k)
    step_ms, _, _ = run.timed(steps, warmup)
    # the trace kernel's time from further steps that time it (the events
    # would lengthen the small field's step)
    _, kern_ms, _ = run.timed(10, warmup + steps, capi.TIMING_TRACE)
    e2e = run.e2e(e2e_steps)
    run.close()
    total = sum(step_ms)
    return {"value": run.rays * steps / (total * 1e-3), "unit": UNIT, "steps": steps, "warmup": warmup,
            "ms_per_step": total / steps, "trace_kernel_ms": S.mean(kern_ms), "e2e": e2e,
            "config": bench_config(w, world)}


# ----------------------------------------------- the reference's CUDA build
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")


def aimed_normals(pos, aim, sun):
    """Unit bisectors of the reversed incident sun direction and the direction
    to each aim point (the reference's CRotate(focus, sun), heliostat.cpp:16-21)."""
    to_t = aim.astype(np.float64) - pos
    to_t /= np.linalg.norm(to_t, axis=1, keepdims=True)
    n = to_t - np.asarray(sun, np.float64)[None, :] / np.linalg.norm(sun)
    return (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)


def ref_cuda_scene(name):
    """Inputs of the reference's own pass (positions, sizes, normals, grid,
    receiver, sunshape), and the CPU checks that keep its out-of-range
    accesses from happening (see ref_cuda_child)."""
    from onemirror_b200 import workloads as W
    if name == "nine":
        g = np.load(os.path.join(ROOT, "tests", "golden", "ref_gpu_vectors.npz"))
        sc = dict(pos=g["trace_pos"], size=g["trace_size"], normal=g["trace_normal"], gpos=g["trace_gpos"],
                  gsize=g["trace_gsize"], inter=g["trace_inter"], rpos=g["trace_rpos"], rsize=g["trace_rsize"],
                  rnorm=g["trace_rnorm"], face=0, ginfo=16, pixel=float(g["trace_pl"]), sun=g["trace_sun"],
                  dni=1000.0, csr=0.1, sigma=0.002,
                  desc="the 9-heliostat scene of the reference's own GPU pin (2x2 m mirrors, 8x8 m receiver at 128x128)")
    else:
        w = W.mid()
        pos, size = w.pos, w.size
        hd = 0.5 * np.linalg.norm(size[:, [0, 2]], axis=1) + 1.0
        lo = np.array([(pos[:, 0] - hd).min(), (pos[:, 1] - hd).min(), (pos[:, 2] - hd).min()], np.float32)
        hi = np.array([(pos[:, 0] + hd).max(), (pos[:, 1] + hd).max(), (pos[:, 2] + hd).max()], np.float32)
        inter = np.full(3, 25.0, np.float32)
        sc = dict(pos=pos, size=size, normal=aimed_normals(pos, w.aim, np.asarray(w.sun.dir[:], np.float32)),
                  gpos=lo, gsize=(hi - lo).astype(np.float32), inter=inter, rpos=np.array(w.receiver.pos[:], np.float32),
                  rsize=np.array(w.receiver.size[:], np.float32), rnorm=np.array(w.receiver.normal[:], np.float32),
                  face=0, ginfo=21, pixel=10.0 / 11.0, sun=np.asarray(w.sun.dir[:], np.float32), dni=1000.0,
                  csr=float(w.sun.csr), sigma=float(w.sigma),
                  desc="the mid field (1000 heliostats 10x10 m, aim offsets, 25 m cells), 11x11 grid micro-points "
                       "per heliostat x 2048 rays, receiver 12x12 m at 21 px/m = 252x252 (the reference's integer "
                       "pixels per metre)")
    return sc


def ref_cuda_checks(sc):
    """CPU checks on the exact inputs: every registration cube of
    CGridHelioMatch (half-side sqrt(|size|)/2, grid.cpp:49-59) and every
    micro-point (on the mirror, within its half-diagonal of the centre) lies
    inside the grid, so boxIntersect and NotCollision index in range."""
    pos, size, gpos, gsize, inter = (np.asarray(sc[k], np.float64) for k in ("pos", "size", "gpos", "gsize", "inter"))
    dims = np.ceil(gsize / inter).astype(int)
    rad = np.sqrt(np.linalg.norm(size, axis=1)) / 2
    lo = ((pos - rad[:, None]) - gpos) / inter
    hi = ((pos + rad[:, None]) - gpos) / inter
    if lo.min() < 0 or np.any(hi.astype(int) > dims - 1):
        return "a registration cube leaves the grid"
    hd = 0.5 * np.linalg.norm(size, axis=1)
    if np.any(pos - hd[:, None] < gpos) or np.any(pos + hd[:, None] > gpos + gsize):
        return "a micro-point may lie outside the grid"
    return None


def ref_cuda_child(name, reps):
    """Run in a child process (the reference exits the process on any CUDA
    error, utils.h:13-22): the reference's pass over one sun position on the
    given scene, `reps` times; prints one JSON line."""
    import torch  # noqa: F401  (CUDA context set-up on the same device as the parent)
    sc = ref_cuda_scene(name)
    why = ref_cuda_checks(sc)
    if why:
        print(json.dumps({"scene": name, "skipped": why}))
        return
    L = C.CDLL(REF_LIB)
    fp = C.POINTER(C.c_float)
    P = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(fp)  # noqa: E731
    keep = {k: np.ascontiguousarray(sc[k], np.float32) for k in ("pos", "size", "normal", "gpos", "gsize", "inter",
                                                                  "rpos", "rsize", "rnorm", "sun")}
    n = keep["pos"].shape[0]
    res = np.zeros(2, np.int32)
    rays = C.c_longlong()
    pass_ms = np.zeros(reps, np.float64)
    trace_ms = np.zeros(reps, np.float32)
    spill = C.c_int()
    L.ref_run_field.restype = C.c_int
    rc = L.ref_run_field(n, *(P(keep[k]) for k in ("pos", "size", "normal", "gpos", "gsize", "inter", "rpos", "rsize",
                                                 "rnorm")), sc["face"], sc["ginfo"], C.c_float(sc["pixel"]),
                         P(keep["sun"]), C.c_float(sc["dni"]), C.c_float(sc["csr"]), C.c_float(sc["sigma"]), 128, 2048,
                         C.c_ulonglong(2018), reps, None, res.ctypes.data_as(C.POINTER(C.c_int)), C.byref(rays),
                         pass_ms.ctypes.data_as(C.POINTER(C.c_double)), trace_ms.ctypes.data_as(fp), C.byref(spill))
    if rc != 0:
        print(json.dumps({"scene": name, "skipped": "reference pass returned %d" % rc}))
        return
    best = int(np.argmin(pass_ms[1:])) + 1 if reps > 1 else 0
    print(json.dumps({"scene": name, "desc": sc["desc"], "heliostats": n, "rays": int(rays.value),
                      "res": [int(res[0]), int(res[1])], "passes": reps, "pass_ms": float(np.median(pass_ms[1:] if reps > 1 else pass_ms)),
                      "map_tracing_ms": float(np.median(trace_ms[1:] if reps > 1 else trace_ms)),
                      "rays_per_s": float(rays.value / (np.median(pass_ms[1:] if reps > 1 else pass_ms) * 1e-3)),
                      "map_tracing_rays_per_s": float(rays.value / (np.median(trace_ms[1:] if reps > 1 else trace_ms) * 1e-3)),
                      "wrote_past_image": bool(spill.value), "best_pass": best}))


def reference_cuda_section(local, reps=3):
    """The reference's own CUDA build (oracle/_ref/libref.so, compiled from
    its sources by oracle/ref.mk) on its per-heliostat structure: per
    heliostat a cuRAND sun table, micro-points, vertices, groups and one
    map_tracing launch followed by a device synchronisation (Gtest.cu:21-35,
    recthelio_tracing.cpp:46-80, ray_tracing.cu:12-27).  A baseline, not the
    measured product; each scene runs in a child process."""
    if not os.path.exists(REF_LIB):
        return {"unavailable": "oracle/_ref/libref.so is not built (the reference sources were absent at build time)"}
    out = {}
    env = dict(os.environ)
    visible = env.get("CUDA_VISIBLE_DEVICES")
    env["CUDA_VISIBLE_DEVICES"] = visible.split(",")[local] if visible else str(local)
    for name in ("nine", "mid"):
        try:
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-cuda-child", name,
                                "--ref-cuda-reps", str(reps)], capture_output=True, text=True, timeout=900, env=env)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            out[name] = json.loads(lines[-1]) if r.returncode == 0 and lines else \
                {"skipped": "child exited %d: %s" % (r.returncode, (r.stderr or r.stdout)[-300:])}
        except subprocess.TimeoutExpired:
            out[name] = {"skipped": "child timed out"}
    return out


def b200_arm(a, rank, world, local):
    import torch
    from onemirror_b200 import capi, workloads as W
    from onemirror_b200 import dist as D

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
    if a.sun_elev is not None:  # the oracle sample follows the same sun
        w.sun = W.make_sun(a.sun_elev, 180.0, w.sun.dni, w.sun.csr)

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

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    run = FieldRun(w, rank, world, dev, flush, sun_elev=a.sun_elev, variant=a.variant)
    sc, p, rays = run.sc, run.p, run.rays
    for k in range(a.warmup):
        run.step(k, D.shard_item(rank, 1000 + k))
    r, _ = run.step(a.warmup, D.shard_item(rank, 5000), want_stats=True)
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
    # the trace kernel's own events stay in the timed steps (its time is the
    # roofline's denominator); the setup is timed on a few steps after them
    step_ms, kern_ms, _ = run.timed(a.steps, a.warmup + 1, capi.TIMING_TRACE)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.stop((t_begin, time.time()))
    _, _, setup_ms = run.timed(5, a.warmup + 1 + a.steps, capi.TIMING_SETUP | capi.TIMING_TRACE)
    total_ms = float(sum(step_ms))
    if world > 1:
        total_ms = D.max_over_ranks(total_ms, dev)
    value = rays * world * a.steps / (total_ms * 1e-3)

    e2e = run.e2e(a.e2e_steps) if a.e2e_steps > 0 else None

    batch = adj = refcuda = None
    fields = {}
    default_run = rank == 0 and world == 1 and a.workload == "mid" and not a.rays
    if default_run:
        if not a.no_batch:
            batch = batch_section()
        if not a.no_adjoint:
            adj = adjoint_section()
        if not a.no_fields:
            fields["small"] = field_block("small", rank, world, dev, flush, steps=100, e2e_steps=20)
            fields["large"] = field_block("large", rank, world, dev, flush, steps=10, e2e_steps=3)
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
    if default_run and not a.no_ref_cuda:
        refcuda = reference_cuda_section(local)
        if "mid" in refcuda and "rays_per_s" in refcuda["mid"]:
            refcuda["value_over_reference_mid"] = value / refcuda["mid"]["rays_per_s"]
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
            "traffic_source": "committed ncu summary profiles/trace_kernel_%s.md (dram bytes of one launch)" % a.workload,
            "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
            "hbm_peak_source": "measured copy" if "hbm_gbs" in peaks else "fallback (6.65 TB/s, earlier copy on B200)"}
    if traffic is not None:
        roof["hbm_achieved_gbs"] = traffic / kern_s / 1e9
        roof["hbm_frac"] = roof["hbm_achieved_gbs"] / roof["hbm_peak_gbs"]
    per_step = {"zero_geometry": 1, "aim": 1, "candidates": 1, "grid_scan": 1, "grid_fill": 1, "grid_cells": 1,
                "point_masks": 1, "zero_maps": 1, "trace": 1, "finalize": 1, "smooth": 1}
    if sc.grid_info().cells > 65536:  # the cell-count scan over tiles: three launches
        per_step["grid_scan"] = 3
    if w.grid.fine_div > 1:
        per_step["grid_coarse"] = 1
    launches = sum(per_step.values())
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": bench_config(w, world),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "flux_rmse": accuracy,
            "gpu_launches": launches * a.steps,
            "launches_per_step": per_step,
            "setup_ms": statistics.mean(setup_ms) if setup_ms else None,
            "setup_ms_note": "aim, candidates and grid build, timed on 5 steps after the timed region",
            "clocks": clocks,
            "fields": fields or None,
            "reference_cuda": refcuda,
            "batched": batch,
            "adjoint": adj,
            "stats": {"shadowed": gst.shadowed / gst.rays, "blocked": gst.blocked / gst.rays,
                      "hit": gst.hit / gst.rays, "intercept_ratio": gst.intercept_ratio}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    run.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    rank, world, local = dist_env()
    if a.ref_cuda_child:
        ref_cuda_child(a.ref_cuda_child, a.ref_cuda_reps)
        return
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return
    b200_arm(a, rank, world, local)


if __name__ == "__main__":
    main()
