"""Edge cases of the CUDA path against the FP64 oracle (same bar as
test_gpu_parity): one heliostat, rays-per-point that is not a power of two,
regular grid points through the full trace, given normals / tilts /
per-heliostat slope errors, a sun below the horizon, zero DNI, accumulation,
one scene across suns and point sets, traces past 2^32 rays, and the
arguments that must be rejected."""
import ctypes as C

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from onemirror_b200.scene import SolarScene  # noqa: E402
from test_gpu_parity import check_pair  # noqa: E402


def trace_pair(w, sc, sun, params):
    """GPU records and maps plus the oracle's on the same points and Philox stream."""
    g = sc.trace(sun, params, records=True)
    torch.cuda.synchronize()
    gi = sc.grid_info()
    ref = O.Scene(sc.pos, sc.size, sc.slope_sigma if sc.slope_sigma is not None else sc.sigma, w.receiver,
                  w.grid.cell[0], w.grid.margin, list(sun.dir), quirks=params.quirks, aim=sc.aim, normal=sc.normal,
                  tilt=sc.tilt, grid_csr=sc.read_grid(), grid_bounds=(list(gi.origin), list(gi.cell), list(gi.dims)))
    xz, helio = sc.read_points()
    weight = np.asarray(sc.size[:, 0] * sc.size[:, 2], np.float64) / np.bincount(helio, minlength=sc.n)
    rays = int(g["stats"].rays)
    cfg = ref.cfg(sun.csr, params.seed, rays, params.rays_per_point, xz, helio, weight, quirks=params.quirks,
                  item=params.item)
    return g, ref.trace_philox(cfg)


def test_single_heliostat_spot_fits_the_receiver():
    pos = np.array([[0.0, 1.5, -40.0]], np.float32)
    size = np.array([[2.0, 0.05, 2.0]], np.float32)
    rec = W.flat_receiver(20.0, 6.0, 6.0, 96, 96)
    w = W.Workload("one", pos, size, 0.002, rec, W.grid(5.0), W.make_sun(50.0, 180.0), W.params(64 * 256, 256, 0.2))
    sc = SolarScene.from_workload(w)
    g, o = trace_pair(w, sc, w.sun, w.params)
    check_pair(w, g, o)
    st = g["stats"]
    assert st.shadowed == 0 and st.blocked == 0 and st.hit == st.rays and st.offmap == 0
    assert abs(st.intercept_ratio - 1.0) < 1e-3  # every ray lands (reflectivity cancels in the ratio)
    sc.close()


def test_rays_per_point_not_a_power_of_two():
    w = W.small()
    sc = SolarScene.from_workload(w)
    p = W.params(w.n * 16 * 100, 100, 0.3, seed=17)
    g, o = trace_pair(w, sc, w.sun, p)
    check_pair(w, g, o)
    sc.close()


def test_regular_grid_points_through_the_full_trace():
    w = W.small()
    sc = SolarScene.from_workload(w)
    p = W.params(0, 64, 0.25, seed=19, mode=capi.POINTS_GRID)
    g, o = trace_pair(w, sc, w.sun, p)
    assert g["stats"].rays == w.n * 8 * 8 * 64  # 2 x 2 m mirrors, 0.25 m cells
    check_pair(w, g, o)
    sc.close()


def test_given_normals_tilts_and_per_heliostat_slope_errors():
    w = W.small()
    rng = np.random.default_rng(5)
    ref = O.Scene(w.pos, w.size, w.sigma, w.receiver, w.grid.cell[0], w.grid.margin, list(w.sun.dir))
    normal = ref.normal + rng.normal(0, 0.01, ref.normal.shape)
    normal = (normal / np.linalg.norm(normal, axis=1, keepdims=True)).astype(np.float32)
    slope = rng.uniform(0.001, 0.004, w.n).astype(np.float32)
    sc = SolarScene(w.pos, w.size, w.receiver, w.grid, sigma=w.sigma, normal=normal, slope_sigma=slope)
    g, o = trace_pair(w, sc, w.sun, w.params)
    check_pair(w, g, o)
    sc.close()
    tilt = rng.normal(0, 0.004, (w.n, 2)).astype(np.float32)
    sc = SolarScene(w.pos, w.size, w.receiver, w.grid, sigma=w.sigma, tilt=tilt)
    g, o = trace_pair(w, sc, w.sun, W.params(int(w.params.rays), 256, 0.3, seed=23))
    check_pair(w, g, o)
    sc.close()


def test_sun_below_the_horizon():
    """An incident direction pointing up: the mirrors face away from the
    receiver; whatever the geometry gives, both sides give the same."""
    w = W.small()
    sc = SolarScene.from_workload(w)
    sun = W.make_sun(-5.0, 180.0)
    g, o = trace_pair(w, sc, sun, W.params(int(w.params.rays), 256, 0.3, seed=29))
    check_pair(w, g, o)
    sc.close()


def test_zero_dni_and_accumulation():
    w = W.small()
    sc = SolarScene.from_workload(w)
    ref = sc.trace(w.sun, w.params)
    counts, flux = ref["counts"].clone(), ref["flux"].clone()
    dark = W.make_sun(45.0, 180.0, 0.0, 0.1)
    g = sc.trace(dark, w.params)
    assert torch.equal(g["counts"], counts) and float(g["flux"].abs().max()) == 0.0
    assert g["stats"].total_power == 0.0
    out = sc._outputs(0, False)
    sc.trace(w.sun, w.params, stats=False, outputs=out)
    p = W.params(int(w.params.rays), 256, 0.3)
    p.accumulate = 1
    sc.trace(w.sun, p, stats=False, outputs=out)
    assert torch.equal(out[1]["counts"], 2 * counts)
    assert torch.allclose(out[1]["flux"], 2 * flux, rtol=1e-6, atol=1e-3)
    sc.close()


def test_one_scene_across_suns_and_point_sets_equals_fresh_scenes():
    """A scene keeps its per-sun passes (aiming, occluder candidates, the
    points' candidate masks and world coordinates) and its points between
    traces, and rebuilds them when the sun or the point set changes: one
    scene traced under sun A, sun B, a second point set, and sun A again
    gives, ray for ray, what a fresh scene gives for each trace."""
    w = W.small()
    sun_b = W.make_sun(25.0, 120.0)
    p_other = W.params(int(w.params.rays), 128, 0.2)  # 32 points per mirror
    steps = [(w.sun, w.params), (sun_b, w.params), (w.sun, p_other), (w.sun, w.params)]
    sc = SolarScene.from_workload(w)
    for sun, params in steps:
        h = sc.trace(sun, params)  # the production kernel meets the change first
        counts = h["counts"].clone()
        g = sc.trace(sun, params, records=True)
        fresh = SolarScene.from_workload(w)
        f = fresh.trace(sun, params, records=True)
        torch.cuda.synchronize()
        assert torch.equal(g["flags"], f["flags"]) and torch.equal(g["pixel"], f["pixel"])
        assert torch.equal(counts, f["counts"]) and torch.equal(g["counts"], f["counts"])
        assert (g["stats"].hit, g["stats"].shadowed, g["stats"].blocked) == (f["stats"].hit, f["stats"].shadowed,
                                                                             f["stats"].blocked)
        fresh.close()
    sc.close()


def test_traces_past_2_to_the_32_rays():
    """2^32 + 2^24 rays (2^20 + 4096 points x 4096 on the mid field): ray ids
    pass 32 bits, so the trace runs as two launches whose threads carry the
    low word of their ray id and whose Philox counters carry the high word.
    The count map sums to the hits; the records of a ray range straddling
    2^32 equal the FP64 oracle's for the same 64-bit ray ids; the limits that
    remain are refused before anything is allocated: 2^32 rays or more with a
    rays-per-point that is not a power of two, and 2^31 points."""
    from test_gpu_parity import AGREE, compare_records
    w = W.mid()
    total = (1 << 32) + (1 << 24)
    w.params = W.params(total, 4096, 0.18)
    sc = SolarScene.from_workload(w)
    g = sc.trace(w.sun, w.params)
    st = g["stats"]
    assert st.rays == total
    assert g["counts"].sum().item() == st.hit - st.offmap
    assert 0.5 < st.hit / st.rays < 0.8
    # a range across 2^32: records indexed by ray id, so the output pointers
    # are given as if the buffers started at ray 0 (only [begin, end) is written)
    begin, n = (1 << 32) - 8192, 16384
    flags = torch.zeros(n, dtype=torch.uint8, device="cuda")
    pixel = torch.zeros(n, dtype=torch.int32, device="cuda")
    o = capi.Outputs()
    o.d_ray_flags = flags.data_ptr() - begin
    o.d_ray_pixel = pixel.data_ptr() - 4 * begin
    p = W.params(total, 4096, 0.18)
    p.ray_begin, p.ray_end = begin, begin + n
    capi.check(capi.lib().qmcrt_trace(sc.h, C.byref(w.sun), C.byref(p), C.byref(o), None,
                                      C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    gi = sc.grid_info()
    ref = O.Scene(w.pos, w.size, w.sigma, w.receiver, w.grid.cell[0], w.grid.margin, list(w.sun.dir), aim=w.aim,
                  grid_csr=sc.read_grid(), grid_bounds=(list(gi.origin), list(gi.cell), list(gi.dims)))
    sc.sample_points_count = total // 4096
    xz, helio = sc.read_points()
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    cfg = ref.cfg(w.sun.csr, p.seed, total, 4096, xz, helio, weight, ray_begin=begin, ray_end=begin + n)
    orc = ref.trace_philox(cfg, maps=False)
    frac, nbad = compare_records(flags.cpu().numpy(), pixel.cpu().numpy(), orc["flags"], orc["pixel"],
                                 w.receiver.res_x)
    assert frac >= AGREE, (frac, nbad)
    assert (flags.cpu().numpy() & capi.RAY_HIT).any()
    for bad in (W.params(3000 * 1431656, 3000, 0.18), W.params((1 << 31) * 256, 256, 0.18)):
        with pytest.raises(capi.QmcrtError) as e:
            sc.trace(w.sun, bad)
        assert e.value.status == capi.ERR_INVALID_ARGUMENT
    sc.close()


def test_rejected_fields_and_grids():
    w = W.small()
    with pytest.raises(capi.QmcrtError):  # empty field
        SolarScene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), w.receiver, w.grid)
    g = W.grid(10.0)
    g.explicit_bounds = 1
    g.origin[:] = [-20.0, -1.0, -20.0]   # a box that misses most of the field
    g.extent[:] = [40.0, 20.0, 40.0]
    with pytest.raises(capi.QmcrtError) as e:
        SolarScene(w.pos, w.size, w.receiver, g)
    assert e.value.status == capi.ERR_INVALID_ARGUMENT and "outside the explicit grid" in str(e.value)
    bad = W.grid(0.0)
    with pytest.raises(capi.QmcrtError):
        SolarScene(w.pos, w.size, w.receiver, bad)


def test_faceted_paraboloid_heliostat():
    """The reference's own kind of scene (scene_file_proc.cpp:288-341, 422-444):
    one heliostat of 3 x 3 canted facets on a paraboloid, 100 m south of a
    1.4 x 1.4 m receiver facing +z; each facet is a rectangle with its given
    normal."""
    sun = W.make_sun(50.0, 180.0)
    sd = np.array(sun.dir[:], np.float64)
    centre = np.array([0.0, 4.0, 100.0])
    aim = np.array([0.0, 13.0, 0.0])
    to_rec = (aim - centre) / np.linalg.norm(aim - centre)
    n = to_rec - sd / np.linalg.norm(sd)
    n /= np.linalg.norm(n)
    pos, size, nrm = W.paraboloid_facets(20.0, 20.0, n, centre)
    rec = W.flat_receiver(13.0, 1.4, 1.4, 140, 140, normal=(0.0, 0.0, 1.0))
    w = W.Workload("facets", pos, size, 0.001, rec, W.grid(1.0), sun, W.params(9 * 64 * 256, 256, 0.03, seed=31))
    sc = SolarScene(pos, size, rec, w.grid, sigma=w.sigma, normal=nrm)
    g, o = trace_pair(w, sc, sun, w.params)
    check_pair(w, g, o)
    assert g["stats"].intercept_ratio > 0.5
    sc.close()


def test_fp64_reciprocals_within_bound():
    """The tracer's own double reciprocal and reciprocal square root (the
    hardware approximation plus one Newton-Raphson step) against exact
    values: relative error below 3e-12 (one step squares the approximation's
    ~2^-20) over the receiver determinants' and the near-unit squared
    lengths' ranges (and well beyond)."""
    import ctypes as C
    rng = np.random.default_rng(5)
    mag = 10.0 ** rng.uniform(-6, 6, 200000)
    x = np.concatenate([mag, -mag, 1.0 + rng.uniform(-1e-5, 1e-5, 100000), [1.0, 2.0, 0.5, 1e-300 * 1e290]])
    d = torch.as_tensor(x, device="cuda")
    rcp = torch.empty_like(d)
    capi.check(capi.lib().qmcrt_fp64_recip_probe(C.c_void_p(d.data_ptr()), d.numel(), C.c_void_p(rcp.data_ptr()),
                                                 None, None))
    pos = x > 0
    dp = torch.as_tensor(x[pos], device="cuda")
    rsq = torch.empty_like(dp)
    capi.check(capi.lib().qmcrt_fp64_recip_probe(C.c_void_p(dp.data_ptr()), dp.numel(), None,
                                                 C.c_void_p(rsq.data_ptr()), None))
    r = rcp.cpu().numpy()
    q = rsq.cpu().numpy()
    assert np.max(np.abs(r * x - 1.0)) < 3e-12
    assert np.max(np.abs(q * np.sqrt(x[pos]) - 1.0)) < 3e-12


@pytest.mark.parametrize("csr", [0.05, 0.2])
def test_buie_bucket_lookup_equals_max_less_index(csr):
    """The tracer's Buie inverse CDF (2048 uniform buckets, one interval
    record each, the record of the next bucket past a boundary) against the
    reference's search, max_less_index (scene_instance_process.cu:98-113),
    and linear interpolation (:115-137) in float32: uniforms at random, at
    every interval boundary and bucket edge (mapped back through the
    kernel's float multiply) and their neighbours a few ulps away.  The
    interval must be the reference's for every value of the core; the angle
    is then the same float computation (one fused multiply-add), so equal to
    the expected value within one ulp (a float64 stand-in for the fused
    operation can round once more)."""
    x = np.zeros(1025, np.float32)
    y = np.zeros(1025, np.float32)
    sl = np.zeros(1024, np.float32)
    p = np.zeros(6, np.float32)
    capi.check(capi.lib().qmcrt_buie_table(C.c_float(csr), capi.as_fp(x), capi.as_fp(y), capi.as_fp(sl), capi.as_fp(p)))
    core, total = np.float32(p[2]), np.float32(p[3])
    inv = np.float32(2048) / core
    rng = np.random.default_rng(3)
    marks = np.concatenate([y[1:1024], np.arange(1, 2048, dtype=np.float32) / inv]).astype(np.float32)
    u0 = (marks / total).astype(np.float32)
    up, down = [u0], [u0]
    for _ in range(3):  # 1 to 3 ulps either side
        up.append(np.nextafter(up[-1], np.float32(1)))
        down.append(np.nextafter(down[-1], np.float32(0)))
    u = np.concatenate([rng.random(1 << 20, dtype=np.float32)] + up + down[1:]).astype(np.float32)
    u = u[(u >= 0) & (u < 1)]
    du = torch.as_tensor(u, device="cuda")
    th = torch.empty_like(du)
    capi.check(capi.lib().qmcrt_buie_sample_probe(C.c_float(csr), C.c_void_p(du.data_ptr()), du.numel(),
                                                  C.c_void_p(th.data_ptr()), None))
    g = th.cpu().numpy()
    uu = (u * total).astype(np.float32)
    core_ = uu < core
    uu, g = uu[core_], g[core_]
    assert uu.size > (1 << 19)
    idx = np.minimum(np.searchsorted(y, uu, side="right") - 1, 1023)  # largest i <= 1023 with y[i] <= uu
    d = (uu - y[idx]).astype(np.float32)
    want = (d.astype(np.float64) * sl[idx].astype(np.float64) + x[idx].astype(np.float64)).astype(np.float32)
    ulp = np.spacing(np.abs(want))
    assert np.all(np.abs(g - want) <= ulp), np.max(np.abs(g - want) / ulp)
    assert np.mean(g == want) > 0.999


def test_ray_range_traces_the_same_rays():
    """qmcrt_trace_params.ray_begin/ray_end: one heliostat's rays (one range,
    as the reference launches them) give the whole trace's flags and pixels
    for those rays, count maps that add up to the whole trace's, and
    statistics of the range alone."""
    w = W.small()
    sc = SolarScene.from_workload(w)
    p = w.params
    g = sc.trace(w.sun, p, records=True)
    f_all, px_all = g["flags"].cpu().numpy(), g["pixel"].cpu().numpy()
    c_all = g["counts"].cpu().numpy().astype(np.int64)
    _, helio = sc.read_points()
    bounds = np.concatenate([[0], np.cumsum(np.bincount(helio, minlength=w.n))]) * p.rays_per_point
    total = np.zeros_like(c_all)
    for h in (0, 1, w.n // 2, w.n - 1):
        p.ray_begin, p.ray_end = int(bounds[h]), int(bounds[h + 1])
        r = sc.trace(w.sun, p, records=True)
        b, e = p.ray_begin, p.ray_end
        assert np.array_equal(r["flags"].cpu().numpy()[b:e], f_all[b:e])
        assert np.array_equal(r["pixel"].cpu().numpy()[b:e], px_all[b:e])
        assert r["stats"].rays == e - b
        pix = px_all[b:e]
        want = np.bincount(pix[pix >= 0], minlength=c_all.size).reshape(c_all.shape)
        assert np.array_equal(r["counts"].cpu().numpy().astype(np.int64), want)
    # every heliostat's range, accumulated, is the whole trace
    p.accumulate = 1
    outs = sc._outputs(int(p.rays), False)
    for h in range(w.n):
        p.ray_begin, p.ray_end = int(bounds[h]), int(bounds[h + 1])
        sc.trace(w.sun, p, stats=False, outputs=outs)
    total = outs[1]["counts"].cpu().numpy().astype(np.int64)
    assert np.array_equal(total, c_all)
    p.accumulate = 0
    for bad in ((5, 5), (10, int(p.rays) + 1)):
        p.ray_begin, p.ray_end = bad
        with pytest.raises(capi.QmcrtError):
            sc.trace(w.sun, p)
    p.ray_begin = p.ray_end = 0
    sc.close()



def test_stage_timing_is_opt_in_and_leaves_the_maps_unchanged():
    """qmcrt_scene_set_timing: no stage is timed by default (qmcrt_scene_timing
    refuses), each enabled stage reports a duration and the others -1, and
    the timing events change none of the trace's results."""
    w = W.small()
    sc = SolarScene.from_workload(w)
    plain = sc.trace(w.sun, w.params)["counts"].cpu().numpy()
    with pytest.raises(capi.QmcrtError):
        sc.timing()
    sc.set_timing(capi.TIMING_TRACE)
    g = sc.trace(W.make_sun(44.0, 180.0), w.params)  # a new sun: the setup runs, untimed
    t = sc.timing()
    assert t.trace_kernel_ms > 0 and t.setup_ms == -1.0 and t.finalize_ms == -1.0
    sc.set_timing(capi.TIMING_ALL)
    g = sc.trace(w.sun, w.params)
    t = sc.timing()
    assert t.setup_ms > 0 and t.trace_kernel_ms > 0 and t.finalize_ms > 0
    assert np.array_equal(g["counts"].cpu().numpy(), plain)
    sc.set_timing(capi.TIMING_FINALIZE)
    sc.trace(w.sun, w.params)  # cached geometry: no setup
    t = sc.timing()
    assert t.finalize_ms > 0 and t.trace_kernel_ms == -1.0 and t.setup_ms == -1.0
    with pytest.raises(capi.QmcrtError):
        sc.set_timing(8)
    sc.set_timing(0)
    sc.trace(w.sun, w.params)
    with pytest.raises(capi.QmcrtError):
        sc.timing()
    sc.close()
