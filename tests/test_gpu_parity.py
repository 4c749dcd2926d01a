"""CUDA path against the FP64 oracle, through the C-ABI.

Bar (per ray, on identical sample streams): shadow/block/hit flags and pixel
indices agree on >= 99.99% of rays, and every pixel disagreement is between
adjacent pixels (a hit on a pixel edge).  Integer count maps agree exactly
wherever the per-ray records agree; the float energy/flux maps agree to the
relative tolerances written in each test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from onemirror_b200.scene import SolarScene, image_smooth  # noqa: E402

AGREE = 0.9999


def oracle_scene(w, sc, sun, quirks=0, use_gpu_grid=True):
    gi = sc.grid_info()
    csr = sc.read_grid() if use_gpu_grid else None
    return O.Scene(w.pos, w.size, w.sigma, w.receiver, w.grid.cell[0], w.grid.margin, list(sun.dir), quirks=quirks,
                   aim=w.aim, grid_csr=csr, grid_bounds=(list(gi.origin), list(gi.cell), list(gi.dims)))


def compare_records(gf, gp, of, op, res_x, wrap=False):
    """Fraction of rays with equal flags and pixels, and the count of the
    others.  wrap: the columns close on themselves (cylinder receiver)."""
    gf, gp, of, op = (np.asarray(a) for a in (gf, gp, of, op))
    same = (gf == of) & (gp == op)
    frac = same.mean()
    bad = np.nonzero(gp != op)[0]
    both = bad[(gp[bad] >= 0) & (op[bad] >= 0)]
    # pixel disagreements on rays both sides trace to the receiver must be
    # neighbouring pixels: the hit lies on a pixel edge
    dr = np.abs(gp[both] // res_x - op[both] // res_x)
    dc = np.abs(gp[both] % res_x - op[both] % res_x)
    if wrap:
        dc = np.minimum(dc, res_x - dc)
    assert np.all((dr <= 1) & (dc <= 1)), "non-adjacent pixel disagreement"
    return frac, int((~same).sum())


@pytest.fixture(scope="module")
def small():
    w = W.small()
    sc = SolarScene.from_workload(w)
    yield w, sc
    sc.close()


def test_philox_kernel_equals_oracle():
    n = 4096
    out = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    ctr = (C.c_uint32 * 4)(7, 0xFFFFFFF0, 3, 0x51A7)
    key = (C.c_uint32 * 2)(0xDEADBEEF, 12345)
    capi.check(capi.lib().qmcrt_philox_blocks(ctr, key, n, C.c_void_p(out.data_ptr()), None))
    g = out.cpu().numpy().view(np.uint32)
    for i in list(range(0, n, 97)) + [n - 1]:
        ref = O.philox([(7 + i) & 0xFFFFFFFF, 0xFFFFFFF0, 3, 0x51A7], [0xDEADBEEF, 12345])
        assert np.array_equal(g[i], ref)


def test_philox_matches_curand():
    """The in-kernel generator is cuRAND's Philox4_32_10 stream for the same key/counter."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "cuda"))
    import build as cb
    L = C.CDLL(cb.build())
    L.curand_ref_philox.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_int, C.c_void_p]
    n = 512
    seed = 0x0123456789ABCDEF
    for sub0, k in [(0, 0), (1 << 33, 5), (77, 1000)]:
        out = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
        assert L.curand_ref_philox(seed, sub0, k, n, out.data_ptr()) == 0
        g = out.cpu().numpy().view(np.uint32)
        for i in range(0, n, 37):
            s = sub0 + i
            ref = O.philox([k, 0, s & 0xFFFFFFFF, s >> 32], [seed & 0xFFFFFFFF, seed >> 32])
            assert np.array_equal(g[i], ref), (sub0, k, i)


def test_poisson_points_bit_exact(small):
    w, sc = small
    xz, helio = sc.points(w.params)
    oxz, oh = O.points_poisson(w.size, int(w.params.rays // w.params.rays_per_point), w.params.point_spacing,
                               w.params.seed)
    assert np.array_equal(helio, oh)
    assert xz.tobytes() == oxz.tobytes()


def test_poisson_points_bit_exact_large_mirrors():
    w = W.mid(rays=1 << 22)
    n = 40
    pos, size = w.pos[:n].copy(), w.size[:n].copy()
    sc = SolarScene(pos, size, w.receiver, w.grid, sigma=w.sigma)
    p = W.params(n * 1000 * 64, 64, 0.18, seed=99)
    xz, helio = sc.points(p)
    oxz, oh = O.points_poisson(size, n * 1000, 0.18, 99)
    assert np.array_equal(helio, oh) and xz.tobytes() == oxz.tobytes()
    sc.close()


def test_poisson_too_dense_reports_sampling_error():
    w = W.small()
    sc = SolarScene.from_workload(w)
    p = W.params(w.n * 500 * 32, 32, 0.3)  # 500 points 0.3 m apart cannot fit on 2x2 m
    with pytest.raises(capi.QmcrtError) as e:
        sc.sample_points(p)
    assert e.value.status == capi.ERR_SAMPLING
    sc.close()


def test_grid_points_match_reference_formula(small):
    w, sc = small
    p = W.params(0, 16, 0.25, mode=capi.POINTS_GRID)
    xz, helio = sc.points(p)
    oxz, oh = O.points_grid(w.size, 0.25)
    assert np.array_equal(helio, oh) and xz.tobytes() == oxz.tobytes()


@pytest.mark.parametrize("quirks", [0, capi.QUIRK_AABB_RADIUS])
def test_geometry_and_grid_equal_oracle(small, quirks):
    w, sc = small
    sc.set_sun(w.sun, quirks)
    nrm, vert = sc.read_geometry()
    ref = oracle_scene(w, sc, w.sun, quirks, use_gpu_grid=False)
    assert np.allclose(nrm, ref.normal, atol=1e-13)
    assert np.allclose(vert, ref.vert, atol=1e-10)
    start, ent = sc.read_grid()
    assert np.array_equal(start, ref.cell_start)
    assert np.array_equal(ent, ref.entries[: start[-1]])


@pytest.mark.parametrize("name", ["mid", "large"])
def test_big_field_grids_equal_oracle(name):
    """The grid CSR of the mid field (one CTA scans its cell counts) and of
    the large field's 12.5 m fine level (more than 65 536 cells: tiles of
    4096 cells, one CTA each, then the tiles' offsets) against the oracle's
    grid over the same bounds."""
    w = W.BUILDERS[name](rays=1 << 20)
    sc = SolarScene.from_workload(w)
    sc.set_sun(w.sun, 0)
    gi = sc.grid_info()
    cells = int(np.prod(list(gi.dims)))
    assert (cells > 65536) == (name == "large"), cells
    ref = oracle_scene(w, sc, w.sun, 0, use_gpu_grid=False)
    start, ent = sc.read_grid()
    assert start.size == cells + 1
    assert np.array_equal(start, ref.cell_start)
    assert np.array_equal(ent, ref.entries[: start[-1]])
    sc.close()


@pytest.mark.parametrize("name", ["small", "mid", "large"])
def test_grid_built_on_demand_after_a_candidate_trace(name):
    """A Philox trace that tests occluder candidates leaves its geometry's
    grid unbuilt unless a list overflows; reading the grid afterwards (and a
    grid-walk trace of the same sun) builds it then, through the single-CTA
    scan (small, mid) or the tiled scan (large), equal to the oracle's CSR,
    and a second demand does not build it twice."""
    w = W.small() if name == "small" else W.BUILDERS[name](rays=1 << 22)
    sc = SolarScene.from_workload(w)
    p = w.params
    cnt = sc.trace(w.sun, p, stats=True)["counts"].clone()
    ref = oracle_scene(w, sc, w.sun, 0, use_gpu_grid=False)
    for _ in range(2):
        start, ent = sc.read_grid()
        assert np.array_equal(start, ref.cell_start)
        assert np.array_equal(ent, ref.entries[: start[-1]])
    p.kernel_variant = 5  # the grid walk, same sun: the cached geometry and its grid
    g5 = sc.trace(w.sun, p, stats=True)
    assert torch.equal(g5["counts"], cnt) and g5["stats"].dda_cells > 0
    p.kernel_variant = 0
    sc.close()


def run_pair(w, sc, sun, params, quirks=0):
    params.quirks = quirks
    g = sc.trace(sun, params, records=True)
    torch.cuda.synchronize()
    ref = oracle_scene(w, sc, sun, quirks)
    xz, helio = sc.read_points()
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    cfg = ref.cfg(sun.csr, params.seed, int(params.rays), params.rays_per_point, xz, helio, weight, quirks=quirks,
                  item=params.item, atten=params.attenuation)
    o = ref.trace_philox(cfg)
    return g, o


def check_pair(w, g, o, min_events=0):
    frac, nbad = compare_records(g["flags"].cpu().numpy(), g["pixel"].cpu().numpy(), o["flags"], o["pixel"],
                                 w.receiver.res_x, wrap=w.receiver.type == capi.RECEIVER_CYLINDER)
    assert frac >= AGREE, (frac, nbad)
    st = g["stats"]
    assert st.rays == o["stats"][0]
    assert abs(int(st.shadowed) - o["stats"][1]) <= nbad and abs(int(st.blocked) - o["stats"][2]) <= nbad
    assert st.shadowed + st.blocked >= min_events
    gc = g["counts"].cpu().numpy().ravel().astype(np.int64)
    oc = o["counts"].astype(np.int64)
    assert gc.sum() == st.hit - st.offmap
    assert np.abs(gc - oc).sum() <= 2 * nbad
    if nbad == 0:
        assert np.array_equal(gc, oc)
    ge = g["energy"].cpu().numpy().ravel().astype(np.float64)
    tol = 1e-5 * ge.max() + 2.0 * nbad * (o["energy"].max() / max(oc.max(), 1))
    assert np.abs(ge - o["energy"]).max() <= tol
    return frac, nbad


def test_trace_small_records_equal_oracle(small):
    w, sc = small
    g, o = run_pair(w, sc, w.sun, w.params)
    frac, nbad = check_pair(w, g, o)
    st = g["stats"]
    # the whole-map totals
    assert abs(st.intercepted_power - (g["flux"].sum().item() * sc_pixel_area(w))) / st.intercepted_power < 1e-4
    assert 0.5 < st.intercept_ratio <= 1.0


def sc_pixel_area(w):
    return (w.receiver.size[0] / w.receiver.res_x) * (w.receiver.size[1] / w.receiver.res_y)


def test_trace_low_sun_shadow_and_block_equal_oracle(small):
    w, sc = small
    sun = W.make_sun(12.0, 200.0, 950.0, 0.1)
    p = W.params(int(w.params.rays), 256, 0.3, seed=21)
    g, o = run_pair(w, sc, sun, p)
    check_pair(w, g, o, min_events=20000)


def test_trace_reference_quirks_equal_oracle(small):
    w, sc = small
    sun = W.make_sun(14.0, 160.0, 1000.0, 0.2)
    q = capi.QUIRK_SKIP_ORIGIN_CELL | capi.QUIRK_AABB_RADIUS | capi.QUIRK_PIXEL_EDGE
    p = W.params(int(w.params.rays), 256, 0.3, seed=5)
    g, o = run_pair(w, sc, sun, p, quirks=q)
    check_pair(w, g, o)


def test_trace_tables_mode_equals_oracle(small):
    """Parity mode: explicit sun/perturbation tables, the map_tracing sampling structure."""
    w, sc = small
    sun = W.make_sun(18.0, 190.0, 1000.0, 0.1)
    T = 8192
    rng = np.random.default_rng(8)
    th = rng.random(T) * 0.009
    ph = rng.random(T) * 2 * np.pi
    sun_local = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    ts = rng.normal(0, 0.002, T)
    tp = rng.random(T) * 2 * np.pi
    turb_local = np.stack([np.sin(ts) * np.cos(tp), np.cos(ts), np.sin(ts) * np.sin(tp)], 1).astype(np.float32)
    xz, helio = O.points_grid(w.size, 0.25)
    start = rng.integers(0, T, len(helio)).astype(np.int32)
    rpp = 64
    # every reference quirk except SELF_HIT, whose outcome is FP32 rounding
    # noise of t around 0 on the ray's own mirror (test_self_hit_quirk_...)
    for quirks in (0, capi.QUIRKS_REFERENCE & ~capi.QUIRK_ZENITH_FRAME & ~capi.QUIRK_SELF_HIT):
        p = W.params(0, rpp, 0.25, seed=1, quirks=quirks)
        g = sc.trace_tables(sun, p, sun_local, turb_local, start, xz, helio)
        ref = oracle_scene(w, sc, sun, quirks)
        cfg = ref.cfg(sun.csr, 1, len(helio) * rpp, rpp, xz, helio, quirks=quirks)
        o = ref.trace_tables(cfg, sun_local, turb_local, start)
        frac, nbad = compare_records(g["flags"].cpu().numpy(), g["pixel"].cpu().numpy(), o["flags"], o["pixel"],
                                     w.receiver.res_x)
        assert frac >= AGREE, (quirks, frac, nbad)
        # flux scaling of the reference driver: DNI * S_sub * rho / N_c / S_rec (Gtest.cu:40-46)
        e = g["energy"].cpu().numpy().astype(np.float64)
        f = g["flux"].cpu().numpy().astype(np.float64)
        scale = 1000.0 * 0.25 ** 2 * 0.88 / rpp / sc_pixel_area(w)
        assert np.allclose(f, e * scale, rtol=1e-6, atol=1e-6)


def test_self_hit_quirk_only_adds_self_shadowing(small):
    """QMCRT_QUIRK_SELF_HIT drops the own-heliostat exclusion, leaving only the
    reference's t > 1e-6 test (global_function.cuh:101-102).  Rays start on
    their own mirror, so whether that mirror 'shadows' them depends on the
    rounding of t around 0: in FP32 a fraction of rays self-shadow, in the
    FP64 oracle almost none do.  The quirk can only add shadowed rays."""
    w, sc = small
    p = W.params(int(w.params.rays), 256, 0.3, seed=3)
    g0 = sc.trace(w.sun, p, records=True)
    f0 = g0["flags"].clone()
    p.quirks = capi.QUIRK_SELF_HIT
    g1 = sc.trace(w.sun, p, records=True)
    f1 = g1["flags"]
    assert torch.all((f0 & 1) <= (f1 & 1))  # shadowed stays shadowed
    diff = f0 != f1
    assert diff.float().mean().item() > 0.0
    # every changed ray ended earlier: newly shadowed, or newly blocked by its own mirror
    assert torch.all((f1[diff] == 1) | ((f1[diff] == 2) & ((f0[diff] & 1) == 0)))


@pytest.mark.parametrize("name", ["mid", "large"])
def test_big_fields_on_ray_ranges(name):
    """Mid (flat receiver) and large (cylinder) geometry: records of ray ranges spread over the field."""
    w = W.BUILDERS[name](rays=1 << 24)
    sc = SolarScene.from_workload(w)
    g = sc.trace(w.sun, w.params, records=True)
    torch.cuda.synchronize()
    ref = oracle_scene(w, sc, w.sun)
    xz, helio = sc.read_points()
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    gf = g["flags"].cpu().numpy()
    gp = g["pixel"].cpu().numpy()
    R = int(w.params.rays)
    total_bad, total = 0, 0
    for b in np.linspace(0, R - (1 << 15), 12).astype(np.int64):
        cfg = ref.cfg(w.sun.csr, w.params.seed, R, 256, xz, helio, weight, ray_begin=int(b), ray_end=int(b) + (1 << 15))
        o = ref.trace_philox(cfg, maps=False)
        frac, nbad = compare_records(gf[b:b + (1 << 15)], gp[b:b + (1 << 15)], o["flags"], o["pixel"],
                                     w.receiver.res_x, wrap=w.receiver.type == capi.RECEIVER_CYLINDER)
        total_bad += nbad
        total += 1 << 15
    assert 1 - total_bad / total >= AGREE, (total_bad, total)
    st = g["stats"]
    assert g["counts"].sum().item() == st.hit - st.offmap
    sc.close()


def test_cylinder_columns_agree_across_resolutions():
    """The cylinder's column rule from 512 to 65 536 columns.  The column
    edges of a map with 2r columns include every edge of the map with r
    columns, bit for bit (the angles 2 pi k / r are formed as (2 pi k) / r,
    and doubling k and r scales numerator and denominator by a power of two),
    so each hit's column at r is its column at 2r halved.  512 and 32 768
    columns take the polynomial column estimate, 65 536 the atan2f one; the
    edge tests must settle both on the same column for every ray."""
    cols, flags0 = {}, None
    for res in (512, 1024, 32768, 65536):
        w = W.large(rays=1 << 22)
        w.receiver.res_x, w.receiver.res_y = res, 16
        sc = SolarScene.from_workload(w)
        g = sc.trace(w.sun, w.params, records=True)
        f, p = g["flags"].cpu().numpy(), g["pixel"].cpu().numpy()
        sc.close()
        if flags0 is None:
            flags0 = f
        assert np.array_equal(f, flags0)
        cols[res] = np.where(p >= 0, p % res, -1)
    hit = cols[512] >= 0
    assert hit.mean() > 0.5
    for r in (512, 32768):
        assert np.array_equal(cols[r][hit], cols[2 * r][hit] // 2), r
    assert np.array_equal(cols[512][hit], cols[32768][hit] // 64)
    assert np.all(cols[65536][~hit] == -1)


def test_two_level_grid_equals_its_fine_level():
    """Large field on its 50 m / 12.5 m two-level grid: the coarse level only
    steps through coarse cells whose heights the ray cannot meet, so flags,
    pixels, maps and even the counts of tested cells and rectangles equal a
    walk of the fine level alone (kernel_variant 4); the fine grid is the one
    a single-level 12.5 m scene builds."""
    w = W.large(rays=1 << 22)
    sc = SolarScene.from_workload(w)
    gi = sc.grid_info()
    assert gi.fine_div == 4 and list(gi.cell) == [12.5, 12.5, 12.5]
    assert all(d % 4 == 0 for d in gi.dims)
    w.params.kernel_variant = 5  # walk the grid (not the candidate lists)
    g2 = sc.trace(w.sun, w.params, records=True)
    f2, p2, c2 = g2["flags"].clone(), g2["pixel"].clone(), g2["counts"].clone()
    w.params.kernel_variant = 4
    g1 = sc.trace(w.sun, w.params, records=True)
    assert torch.equal(f2, g1["flags"]) and torch.equal(p2, g1["pixel"]) and torch.equal(c2, g1["counts"])
    s1, s2 = g1["stats"], g2["stats"]
    assert (s1.rect_tests, s1.dda_cells) == (s2.rect_tests, s2.dda_cells)
    # production kernels (no records, no statistics; separately compiled, so
    # the compiler's FMA contraction may differ and a ray on a rectangle edge
    # may flip): the same maps up to a few such rays
    w.params.kernel_variant = 5
    m2 = sc.trace(w.sun, w.params, stats=False)["counts"].clone()
    w.params.kernel_variant = 4
    m1 = sc.trace(w.sun, w.params, stats=False)["counts"]
    edge = 2 * max(1, int(1e-5 * c2.sum().item()))
    assert (m2 - c2).abs().sum().item() <= edge and (m1 - c2).abs().sum().item() <= edge
    # a single-level scene with the fine cell size builds the same grid
    w1 = W.large(rays=1 << 22)
    w1.grid = W.grid(12.5)
    sc1 = SolarScene.from_workload(w1)
    gi1 = sc1.grid_info()
    if list(gi1.dims) == list(gi.dims):
        a, b = sc.read_grid(), sc1.read_grid()
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    sc1.close()
    sc.close()


@pytest.mark.parametrize("name", ["small", "large"])
def test_attenuation_equals_oracle(name):
    """eta(d) of the mirror-to-receiver leg (QMCRT_ATTEN_POLY_EXP): records and
    maps against the oracle; the large field's slant ranges pass 1000 m, so
    both branches of the formula run.  Attenuation scales energies only: the
    count map is the plain trace's."""
    w = W.small() if name == "small" else W.large(rays=1 << 22)
    sc = SolarScene.from_workload(w)
    p = w.params
    p.attenuation = capi.ATTEN_POLY_EXP
    g, o = run_pair(w, sc, w.sun, p)
    check_pair(w, g, o)
    p.attenuation = capi.ATTEN_NONE
    g0 = sc.trace(w.sun, p, records=True)
    assert torch.equal(g0["counts"], g["counts"])
    r = (g["energy"].double().sum() / g0["energy"].double().sum()).item()
    assert (0.9 if name == "small" else 0.8) < r < 0.99, r
    sc.close()


@pytest.mark.parametrize("name", ["small", "mid", "large"])
def test_lean_builds_equal_the_general_build(name):
    """The production launch picks a build compiled for its receiver type and,
    in the common case, a lean one (power-of-two rays per point, point masks,
    no attenuation, no pixel-edge quirk: none of them tested per ray); kernel_variant 3 runs the general build,
    which reads the receiver type and tests every case per ray.  (Per-ray
    records and statistics take the general build too, so the production
    launch is compared through its maps.)  The count maps are bit-identical
    and the energy maps equal to the order of their float additions (flat
    receivers on the small and mid fields, the cylinder on the large field)."""
    w = W.small() if name == "small" else W.BUILDERS[name](rays=1 << 22)
    sc = SolarScene.from_workload(w)
    p = w.params
    g = sc.trace(w.sun, p, records=False, stats=False)
    cnt, en = g["counts"].clone(), g["energy"].clone()
    p.kernel_variant = 3
    g3 = sc.trace(w.sun, p, records=False, stats=False)
    p.kernel_variant = 0
    assert torch.equal(cnt, g3["counts"]) and int(cnt.sum()) > 0
    # the energy map is a sum of float atomics: equal to float reordering
    assert torch.allclose(en, g3["energy"], rtol=1e-5, atol=1e-6 * float(en.max()))
    sc.close()


@pytest.mark.parametrize("name,elev", [("small", 45.0), ("small", 12.0), ("mid", 30.0), ("mid", 8.0), ("large", 20.0)])
def test_candidate_lists_equal_the_grid_walk(name, elev):
    """Philox rays test only their heliostat's occluder candidates (the
    heliostats a cone bounding the sampler's directions can reach); every
    flag, pixel and count equals the grid walk's (kernel_variant 5), and only
    rays of overflowing lists walk cells."""
    w = W.small() if name == "small" else W.BUILDERS[name](rays=1 << 22)
    sun = W.make_sun(elev, 200.0, 1000.0, w.sun.csr)
    sc = SolarScene.from_workload(w)
    p = w.params
    g = sc.trace(sun, p, records=True)
    f, px, cnt = g["flags"].clone(), g["pixel"].clone(), g["counts"].clone()
    p.kernel_variant = 5
    g5 = sc.trace(sun, p, records=True)
    assert torch.equal(f, g5["flags"]) and torch.equal(px, g5["pixel"]) and torch.equal(cnt, g5["counts"])
    assert g["stats"].dda_cells < g5["stats"].dda_cells  # only overflowing lists walk
    sc.close()


def test_overflowing_candidate_lists_walk_the_grid():
    """A row of 60 small mirrors laid along the sun's horizontal direction
    under a 1 degree sun: the first mirrors' shadow rays graze over more than
    32 others, so those lists overflow and their rays walk the grid (cells
    walked > 0); every flag, pixel and count still equals the pure walk's."""
    sun = W.make_sun(1.0, 150.0, 1000.0, 0.1)
    sd = np.array(sun.dir[:], np.float64)
    toward = -np.array([sd[0], 0.0, sd[2]])
    toward /= np.linalg.norm(toward)
    p0 = np.array([0.0, 1.5, -40.0])
    pos = np.array([p0 + 1.5 * i * toward for i in range(60)], np.float32)
    size = np.tile(np.array([[1.0, 0.05, 1.0]], np.float32), (60, 1))
    rec = W.flat_receiver(30.0, 6.0, 6.0, 64, 64)
    w = W.Workload("row", pos, size, 0.002, rec, W.grid(5.0), sun, W.params(60 * 16 * 256, 256, 0.1, seed=3))
    sc = SolarScene.from_workload(w)
    p = w.params
    g = sc.trace(sun, p, records=True)
    f, px, cnt = g["flags"].clone(), g["pixel"].clone(), g["counts"].clone()
    assert g["stats"].dda_cells > 0  # some lists overflowed
    assert g["stats"].shadowed > 0
    p.kernel_variant = 5
    g5 = sc.trace(sun, p, records=True)
    assert torch.equal(f, g5["flags"]) and torch.equal(px, g5["pixel"]) and torch.equal(cnt, g5["counts"])
    sc.close()


def candidate_field(name):
    if name == "batch4000":
        return W.batched(rays_per_item=1 << 16)[0][2]
    return W.small() if name == "small" else W.BUILDERS[name](rays=1 << 20)


@pytest.mark.parametrize("name,elev,az", [("small", 45.0, 200.0), ("small", 0.4, 90.0), ("mid", 30.0, 200.0),
                                          ("mid", 5.0, 120.0), ("mid", 0.3, 250.0), ("large", 20.0, 200.0),
                                          ("large", 6.0, 45.0), ("batch4000", 10.0, 250.0)])
def test_candidate_bucket_search_equals_every_pair(name, elev, az):
    """The candidate search visits only the centre buckets a cone can reach;
    its lists hold the same heliostats as testing every pair.  A 0.3-0.4 deg
    sun makes shadow cones that do not rise, which visit every bucket."""
    w = candidate_field(name)
    sc = SolarScene.from_workload(w)
    sc.set_sun(W.make_sun(elev, az, 1000.0, w.sun.csr))
    c, ids = sc.read_candidates()
    ce, ide = sc.read_candidates(exhaustive=True)
    assert np.array_equal(c, ce)
    assert c.sum() > 0
    kept = c <= capi.CAND_CAP  # overflowing lists store only their first records, in search order
    assert np.array_equal(np.sort(ids, axis=2)[kept], np.sort(ide, axis=2)[kept])
    # a moved field rebuilds the buckets: move half the mirrors 0.5 m (within
    # the grid's margin) and compare again
    sc.pos[0::2, 0] += 0.5
    sc.pos[1::2, 2] -= 0.5
    sc.update_field()
    sc.set_sun(W.make_sun(elev, az, 1000.0, w.sun.csr))
    c2, ids2 = sc.read_candidates()
    ce2, ide2 = sc.read_candidates(exhaustive=True)
    kept = c2 <= capi.CAND_CAP
    assert np.array_equal(c2, ce2)
    assert np.array_equal(np.sort(ids2, axis=2)[kept], np.sort(ide2, axis=2)[kept])
    sc.close()


def test_wide_slope_error_takes_every_heliostat():
    """A slope error so large (0.2 rad: the 6-sigma block cone passes 69
    degrees) that no cone bounds the block rays: every other heliostat is a
    block candidate, and a trace through the lists equals the grid walk."""
    w = W.small()
    n = 24
    sc = SolarScene(w.pos[:n].copy(), w.size[:n].copy(), w.receiver, w.grid, sigma=0.2)
    sun = W.make_sun(30.0, 200.0, 1000.0, w.sun.csr)
    sc.set_sun(sun)
    c, _ = sc.read_candidates()
    assert np.all(c[:, 1] == n - 1)
    ce, _ = sc.read_candidates(exhaustive=True)
    assert np.array_equal(c, ce)
    p = W.params(n * 16 * 256, 256, 0.3)
    g = sc.trace(sun, p, records=True)
    f, px, cnt = g["flags"].clone(), g["pixel"].clone(), g["counts"].clone()
    p.kernel_variant = 5
    g5 = sc.trace(sun, p, records=True)
    assert torch.equal(f, g5["flags"]) and torch.equal(px, g5["pixel"]) and torch.equal(cnt, g5["counts"])
    sc.close()


def test_candidates_need_a_sun():
    w = W.small()
    sc = SolarScene.from_workload(w)
    with pytest.raises(capi.QmcrtError):
        sc.read_candidates()
    sc.close()


def test_smoothing_heaps_bit_exact_with_reference_gpu_kernel():
    """QMCRT_TRIM_HEAPS against ImageSmoother::image_smooth's output on a B200."""
    from test_oracle_pins import GV
    for k in range(len(GV["smooth_params"])):
        r, ratio = GV["smooth_params"][k]
        d = torch.as_tensor(GV["smooth_in_%d" % k], device="cuda")
        out = image_smooth(d, int(r), float(ratio), capi.TRIM_HEAPS)
        assert out.cpu().numpy().tobytes() == GV["smooth_out_%d" % k].tobytes(), k


def test_trace_tables_image_matches_reference_map_tracing():
    """Table mode with the reference's quirks against the receiver image the
    reference's own map_tracing produced on a B200 for the same 9-heliostat
    scene, grid and tables (same bar as the oracle's pin)."""
    from test_oracle_pins import GV, TRACE_QUIRKS, assert_trace_image_matches
    res_x, res_y = (int(v) for v in GV["trace_res"])
    rec = W.flat_receiver(0.0, 1.0, 1.0, res_x, res_y, normal=tuple(float(v) for v in GV["trace_rnorm"]))
    rec.pos[:] = [float(v) for v in GV["trace_rpos"]]
    rec.size[:] = [float(v) for v in GV["trace_rsize"]]
    grid = W.grid(float(GV["trace_inter"][0]))
    grid.explicit_bounds = 1
    grid.origin[:] = [float(v) for v in GV["trace_gpos"]]
    grid.extent[:] = [float(v) for v in GV["trace_gsize"]]
    sc = SolarScene(GV["trace_pos"], GV["trace_size"], rec, grid, sigma=0.0, normal=GV["trace_normal"])
    sun = W.make_sun(45.0, 180.0, 1000.0, 0.1)
    sun.dir[:] = [float(v) for v in GV["trace_sun"]]
    lights = int(GV["trace_lights"])
    pl = float(GV["trace_pl"])
    xz, helio = sc.points(W.params(0, lights, pl, mode=capi.POINTS_GRID))
    p = W.params(0, lights, pl, quirks=TRACE_QUIRKS)
    g = sc.trace_tables(sun, p, GV["trace_sun_local"], GV["trace_turb_local"], GV["trace_start"], xz, helio)
    assert_trace_image_matches(g["energy"].cpu().numpy(), GV["trace_image"], len(helio) * lights)
    sc.close()


def test_grid_fine_div_must_be_a_power_of_two():
    w = W.small()
    w.grid = W.grid(10.0, fine_div=3)
    with pytest.raises(capi.QmcrtError):
        SolarScene.from_workload(w)


def test_smoothing_u32_sorted_bit_exact():
    rng = np.random.default_rng(4)
    # radii 1-3 take the register sorting network, the others the general path;
    # maps narrower than the window, and counts up to the uint32 maximum (the
    # network pads clipped windows with that value)
    for (h, w_), r, ratio in [((128, 128), 2, 0.2), ((67, 201), 3, 0.1), ((1, 1), 2, 0.2), ((5, 300), 7, 0.45),
                              ((64, 64), 0, 0.2), ((40, 33), 2, 0.0), ((50, 77), 1, 0.3), ((3, 2), 3, 0.2),
                              ((256, 256), 1, 0.0), ((9, 40), 2, 0.49), ((33, 31), 3, 0.45), ((20, 20), 4, 0.2)]:
        img = rng.integers(0, 5000, (h, w_)).astype(np.uint32)
        img[rng.random(img.shape) < 0.3] = 0
        img[rng.random(img.shape) < 0.05] = 0xFFFFFFFF
        img[rng.random(img.shape) < 0.05] = 0xFFFFFFF0
        d = torch.as_tensor(img.view(np.int32), device="cuda")
        out = image_smooth(d, r, ratio, capi.TRIM_SORTED).cpu().numpy()
        ref = O.smooth_u32(img, r, ratio, 0)
        assert out.tobytes() == ref.tobytes(), (h, w_, r, ratio)


def test_smoothing_heaps_bit_exact_float_and_counts():
    rng = np.random.default_rng(5)
    imgf = (rng.random((96, 130)) * 100).astype(np.float32)
    imgf[rng.random(imgf.shape) < 0.4] = 0
    for r, ratio in [(2, 0.2), (5, 0.02), (1, 0.3)]:
        out = image_smooth(torch.as_tensor(imgf, device="cuda"), r, ratio, capi.TRIM_HEAPS).cpu().numpy()
        assert out.tobytes() == O.smooth_f32(imgf, r, ratio, 1).tobytes()
    imgu = rng.integers(0, 1000, (50, 70)).astype(np.uint32)
    out = image_smooth(torch.as_tensor(imgu.view(np.int32), device="cuda"), 2, 0.2, capi.TRIM_HEAPS).cpu().numpy()
    assert out.tobytes() == O.smooth_u32(imgu, 2, 0.2, 1).tobytes()
    # float maps, sorted definition: FP32 sums against the FP64 oracle (radii
    # 1-3 on the register sorting network, 5 on the general path)
    for r in (1, 2, 3, 5):
        out = image_smooth(torch.as_tensor(imgf, device="cuda"), r, 0.2, capi.TRIM_SORTED).cpu().numpy()
        assert np.allclose(out, O.smooth_f32(imgf, r, 0.2, 0), rtol=1e-5, atol=1e-5), r


def test_smoothing_of_traced_counts_bit_exact(small):
    w, sc = small
    g = sc.trace(w.sun, w.params)
    out = image_smooth(g["counts"], w.smooth_radius, w.smooth_ratio, capi.TRIM_SORTED).cpu().numpy()
    ref = O.smooth_u32(g["counts"].cpu().numpy().view(np.uint32), w.smooth_radius, w.smooth_ratio, 0)
    assert out.tobytes() == ref.tobytes()


def test_smoothing_argument_errors():
    d = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    with pytest.raises(capi.QmcrtError):
        capi.check(capi.lib().qmcrt_smooth_trimmed_f32(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), 8, 8, 2,
                                                       C.c_float(0.2), 0, None))
    with pytest.raises(capi.QmcrtError):
        image_smooth(d, 9, 0.2)
    with pytest.raises(capi.QmcrtError):
        image_smooth(d, 2, 0.6)


def test_full_size_properties_mid():
    """2^28 rays: count-map sum equals hits, reruns reproduce counts exactly, disjoint items differ."""
    w = W.mid()
    sc = SolarScene.from_workload(w)
    a = sc.trace(w.sun, w.params)
    ca = a["counts"].clone()
    b = sc.trace(w.sun, w.params)
    st = a["stats"]
    assert st.rays == 1 << 28
    assert ca.sum().item() == st.hit - st.offmap
    assert torch.equal(ca, b["counts"])
    assert torch.allclose(a["energy"], b["energy"], rtol=1e-4, atol=1e-3)
    w.params.item = 1
    c = sc.trace(w.sun, w.params)
    assert not torch.equal(ca, c["counts"])
    rel = abs(c["stats"].intercepted_power - st.intercepted_power) / st.intercepted_power
    assert rel < 1e-3  # two independent 2^28-ray estimates of the same power
    sc.close()


def test_host_entry_point_matches_device_path(small):
    w, sc = small
    counts, flux, st = sc.trace_host(w.sun, w.params)
    g = sc.trace(w.sun, w.params)
    assert np.array_equal(counts.view(np.int32), g["counts"].cpu().numpy())
    assert np.allclose(flux, g["flux"].cpu().numpy(), rtol=1e-4, atol=1e-2)


def test_trace_argument_errors(small):
    w, sc = small
    p = W.params(1001, 256, 0.3)
    with pytest.raises(capi.QmcrtError) as e:
        sc.trace(w.sun, p)
    assert e.value.status == capi.ERR_INVALID_ARGUMENT
    bad = W.make_sun(45, 180)
    bad.csr = 0.0
    with pytest.raises(capi.QmcrtError):
        sc.trace(bad, w.params)
    p = W.params(int(w.params.rays), 256, 0.3)
    p.quirks = 1 << 20
    with pytest.raises(capi.QmcrtError):
        sc.trace(w.sun, p)
    for field, value in (("attenuation", 7), ("kernel_variant", 9)):
        p = W.params(int(w.params.rays), 256, 0.3)
        setattr(p, field, value)
        with pytest.raises(capi.QmcrtError) as e:
            sc.trace(w.sun, p)
        assert e.value.status == capi.ERR_INVALID_ARGUMENT
    # the scene still works after rejected calls
    g = sc.trace(w.sun, w.params)
    assert g["stats"].rays == w.params.rays
