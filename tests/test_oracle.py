"""The FP64 oracle against analytic known answers and independent restatements.

The reference has no tests or golden vectors, so the oracle is pinned by
(a) analytic cases with known answers, (b) brute-force traversal, (c) small
pure-Python restatements, and (d) the reference's own host-callable code
compiled in oracle/_ref (tests/test_oracle_pins.py).
"""
import ctypes as C
import heapq

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W
from oracle import oracle as O


def flat_recv(pos, size, res, normal=(0.0, 0.0, -1.0)):
    r = capi.Receiver()
    r.type = 0
    r.pos[:] = list(pos)
    r.size[:] = list(size)
    r.normal[:] = list(normal)
    r.face = 0
    r.res_x, r.res_y = res
    return r


def test_philox_counter_and_key_sensitivity():
    a = O.philox([1, 2, 3, 4], [5, 6])
    assert not np.array_equal(a, O.philox([1, 2, 3, 5], [5, 6]))
    assert not np.array_equal(a, O.philox([1, 2, 3, 4], [5, 7]))
    assert np.array_equal(a, O.philox([1, 2, 3, 4], [5, 6]))
    # bits look uniform over many counters
    bits = np.array([O.philox([i, 0, 0, 0], [9, 9]) for i in range(4000)]).ravel()
    assert abs(np.unpackbits(bits.view(np.uint8)).mean() - 0.5) < 0.01


def test_buie_inverse_cdf_monotone_and_bounded():
    x, y, s, p = O.buie_table(0.1)
    L = O.lib()
    us = np.linspace(1e-7, 1 - 1e-7, 20001)
    th = np.array([L.orc_buie_sample(u, O._p(x, O.fp), O._p(y, O.fp), O._p(s, O.fp), O._p(p, O.fp)) for u in us])
    assert np.all(np.diff(th) >= -1e-12)
    assert th[0] >= 0 and th[-1] <= 9.3 + 1e-4
    # the core/aureole boundary sits at 4.65 mrad with the reference's mass split
    frac_core = float(p[2] / p[3])
    assert abs(np.mean(th < 4.65) - frac_core) < 2e-3


def test_buie_sample_density_matches_the_tabulated_profile():
    # density of theta is the trapezoid-interpolated core profile (no sin
    # theta Jacobian, scene_instance_process.cu:56-60) scaled by 1/A
    x, y, s, p = O.buie_table(0.1)
    L = O.lib()
    rng = np.random.default_rng(1)
    u = rng.random(200000)
    th = np.array([L.orc_buie_sample(v, O._p(x, O.fp), O._p(y, O.fp), O._p(s, O.fp), O._p(p, O.fp)) for v in u])
    hist, edges = np.histogram(th, bins=31, range=(0.0, 4.65))
    mid = 0.5 * (edges[1:] + edges[:-1])
    prof = np.cos(0.326 * mid) / np.cos(0.308 * mid)
    expect = prof / p[3] * (edges[1] - edges[0]) * len(u)
    assert np.max(np.abs(hist - expect) / np.sqrt(expect)) < 5


@pytest.mark.parametrize("csr", [0.05, 0.1, 0.2])
def test_buie_cdf_equals_the_integrated_profile(csr):
    """The table's cumulative values are the integral of the core profile
    cos(0.326 t)/cos(0.308 t) (t in mrad, no sin t Jacobian) from 0 to each
    node (1024 trapezoids to 4.65 mrad: exact to the trapezoid error), the
    aureole mass is the integral of e^k t^gamma from 4.65 to 9.3 mrad, and
    the analytic aureole inverse lands where the integrated CDF reaches u."""
    from scipy.integrate import quad
    x, y, s, p = O.buie_table(csr)
    k, gamma, core, total = (float(v) for v in p[:4])
    prof = lambda t: np.cos(0.326 * t) / np.cos(0.308 * t)
    for i in (1, 100, 512, 900, 1024):
        exact = quad(prof, 0.0, float(x[i]), epsabs=1e-13)[0]
        assert abs(float(y[i]) - exact) <= 1e-4 * exact, (i, y[i], exact)
    aur = lambda t: np.exp(k) * t ** gamma
    assert abs((total - core) - quad(aur, 4.65, 9.3, epsabs=1e-13)[0]) <= 1e-4 * (total - core)
    L = O.lib()
    for frac in (0.2, 0.5, 0.9):
        u = (core + frac * (total - core)) / total
        th = L.orc_buie_sample(u, O._p(x, O.fp), O._p(y, O.fp), O._p(s, O.fp), O._p(p, O.fp))
        reached = core + quad(aur, 4.65, th, epsabs=1e-13)[0]
        assert abs(reached - u * total) <= 1e-4 * total, (frac, th)


def test_local2world_frame():
    L = O.lib()
    rng = np.random.default_rng(3)
    for _ in range(50):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        cols = []
        for e in np.eye(3):
            o = (C.c_double * 3)()
            L.orc_local2world((C.c_double * 3)(*e), (C.c_double * 3)(*n), 0, o)
            cols.append(np.array(o[:]))
        M = np.array(cols)
        assert np.allclose(M @ M.T, np.eye(3), atol=1e-12)
        assert np.allclose(cols[1], n, atol=1e-12)  # local y -> n
        assert abs(cols[0][1]) < 1e-12  # u is horizontal
    # zenith: identity for +y; -y flips unless the reference quirk is on
    o = (C.c_double * 3)()
    L.orc_local2world((C.c_double * 3)(0.1, 0.9, 0.2), (C.c_double * 3)(0, -1, 0), 0, o)
    assert np.allclose(o[:], [0.1, -0.9, -0.2])
    L.orc_local2world((C.c_double * 3)(0.1, 0.9, 0.2), (C.c_double * 3)(0, -1, 0), capi.QUIRK_ZENITH_FRAME, o)
    assert np.allclose(o[:], [0.1, 0.9, 0.2])


def test_parallelogram_known_answers():
    L = O.lib()
    A, B, Cc = (C.c_double * 3)(0, 0, 0), (C.c_double * 3)(0, 0, 2), (C.c_double * 3)(2, 0, 0)
    t, u, v = C.c_double(), C.c_double(), C.c_double()

    def hit(o, d):
        return L.orc_ray_parallelogram((C.c_double * 3)(*o), (C.c_double * 3)(*d), A, B, Cc, C.byref(t), C.byref(u),
                                       C.byref(v))

    assert hit((0.5, 3, 1.5), (0, -1, 0)) and abs(t.value - 3) < 1e-12
    assert abs(u.value - 0.75) < 1e-12 and abs(v.value - 0.25) < 1e-12  # u along B-A, v along C-A
    assert not hit((2.5, 3, 1.0), (0, -1, 0))  # outside
    assert not hit((0.5, 3, 1.0), (0, 1, 0))   # behind (t < 0)
    assert not hit((0.5, 3, 1.0), (1, 0, 0))   # parallel
    assert hit((2.0, 1, 2.0), (0, -1, 0))      # corner is inside (closed interval)


def dense_scene(quirks=0, elev=15.0):
    w = W.small()
    sun = W.make_sun(elev, 180.0)
    sc = O.Scene(w.pos, w.size, w.sigma, w.receiver, 10.0, 1.0, list(sun.dir), quirks=quirks)
    return w, sc


def test_dda_equals_brute_force_in_corrected_mode():
    w, sc = dense_scene(0, elev=12.0)
    rng = np.random.default_rng(5)
    hits = 0
    for k in range(3000):
        h = int(rng.integers(0, w.n))
        v = sc.vert[h].reshape(3, 3)
        a, b = rng.random(2)
        o = v[0] + a * (v[1] - v[0]) + b * (v[2] - v[0])
        d = rng.normal(size=3)
        d[1] = abs(d[1]) * 0.3
        d /= np.linalg.norm(d)
        r1 = sc.dda(o, d, h)
        r2 = sc.dda(o, d, h, brute=True)
        assert r1 == r2
        hits += r1
    assert hits > 100  # the case exercises occluders


def test_skip_origin_cell_quirk_misses_same_cell_occluders():
    w, sc0 = dense_scene(0, elev=12.0)
    _, sc1 = dense_scene(capi.QUIRK_SKIP_ORIGIN_CELL, elev=12.0)
    rng = np.random.default_rng(6)
    diff = 0
    for k in range(3000):
        h = int(rng.integers(0, w.n))
        v = sc0.vert[h].reshape(3, 3)
        o = v[0] + 0.5 * (v[1] - v[0]) + 0.5 * (v[2] - v[0])
        d = rng.normal(size=3)
        d[1] = abs(d[1]) * 0.3
        d /= np.linalg.norm(d)
        a, b = sc0.dda(o, d, h), sc1.dda(o, d, h)
        assert b <= a  # skipping cells can only lose hits
        diff += a != b
    assert diff > 0


def single_heliostat_case(sigma=0.0):
    # one 2x2 m heliostat 50 m north of a 5x5 m receiver, aimed at its centre
    pos = np.array([[0.0, 2.0, -50.0]], np.float32)
    size = np.array([[2.0, 0.05, 2.0]], np.float32)
    rec = flat_recv((0.0, 20.0, 0.0), (5.0, 5.0, 0.0), (64, 64))
    sun = W.make_sun(40.0, 180.0)
    sc = O.Scene(pos, size, sigma, rec, 10.0, 1.0, list(sun.dir))
    xz, helio = O.points_poisson(size, 16, 0.3, 11)
    return sc, sun, xz, helio


def test_single_heliostat_intercept_is_one():
    sc, sun, xz, helio = single_heliostat_case()
    cfg = sc.cfg(0.1, 3, 16 * 512, 512, xz, helio, weight=[4.0 / 16])
    r = sc.trace_philox(cfg)
    st = r["stats"]
    assert st[0] == 16 * 512 and st[3] == st[0] and st[1] == 0 and st[2] == 0
    # with sigma = 0 every ray carries |n . s| * A / P: intercept ratio 1
    n = sc.normal[0]
    s = np.array(sun.dir[:], np.float64)
    s /= np.linalg.norm(s)
    expect = abs(n @ s) * 4.0 * 512
    assert abs(r["energy"].sum() - expect) / expect < 1e-12
    # the spot is centred on the receiver
    c = r["counts"].reshape(64, 64)
    ys, xs = np.nonzero(c)
    assert abs(np.average(ys, weights=c[ys, xs]) - 31.5) < 2 and abs(np.average(xs, weights=c[ys, xs]) - 31.5) < 2


def test_face_to_face_shadow_known_answer():
    # heliostat A in the full shadow of a larger heliostat B placed between A
    # and the sun (the geometry of userData/face2face_shadow.scn)
    el = 30.0
    sun = W.make_sun(el, 180.0)
    towards_sun = -np.array(sun.dir[:], np.float64)
    towards_sun /= np.linalg.norm(towards_sun)
    pa = np.array([0.0, 2.0, -60.0])
    pb = pa + 23.0 * towards_sun
    pos = np.array([pa, pb], np.float32)
    size = np.array([[2.0, 0.05, 2.0], [3.0, 0.05, 3.0]], np.float32)
    normal = np.array([towards_sun, towards_sun], np.float32)
    rec = flat_recv((0.0, 80.0, 0.0), (5.0, 5.0, 0.0), (32, 32))
    sc = O.Scene(pos, size, 0.0, rec, 10.0, 1.0, list(sun.dir), normal=normal)
    xz, helio = O.points_poisson(size, 32, 0.2, 5)
    cfg = sc.cfg(0.1, 9, 32 * 64, 64, xz, helio)
    r = sc.trace_philox(cfg)
    f = r["flags"].reshape(32, 64)
    assert np.all(f[helio == 0] & 1)       # every ray of A is shadowed
    assert not np.any(f[helio == 1] & 1)   # nothing shadows B


def test_points_poisson_spacing_count_and_determinism():
    size = np.array([[2.0, 0.05, 2.0], [10.0, 0.1, 10.0], [3.0, 0.1, 1.0]], np.float32)
    xz, helio = O.points_poisson(size, 3 * 100, 0.12, 42)
    for h in range(3):
        p = xz[helio == h].astype(np.float64)
        assert len(p) == 100
        assert np.all(np.abs(p[:, 0]) <= size[h, 0] / 2) and np.all(np.abs(p[:, 1]) <= size[h, 2] / 2)
        d = np.sqrt(((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)) + np.eye(len(p)) * 1e9
        assert d.min() >= 0.12 - 2 ** -15
    xz2, _ = O.points_poisson(size, 3 * 100, 0.12, 42)
    assert np.array_equal(xz, xz2)
    with pytest.raises(RuntimeError):
        O.points_poisson(size[:1], 1000, 0.3, 1)  # cannot fit 1000 points 0.3 m apart on 4 m^2


def test_points_poisson_equals_a_plain_python_restatement():
    size = np.array([[1.0, 0.05, 0.7]], np.float32)
    xz, _ = O.points_poisson(size, 20, 0.1, 77)
    # sequential dart throwing with the same Philox candidates, O(n^2) checks
    Rq = int(0.1 * 65536)
    key = [(77 ^ 0x5A17C0DE) & 0xFFFFFFFF, (0 ^ 0x0B5E55ED) & 0xFFFFFFFF]
    W_, H_ = int(1.0 * 65536), int(np.float32(0.7) * 65536.0)
    pts = []
    c = 0
    while len(pts) < 20:
        w = O.philox([0, c & 0xFFFFFFFF, c >> 32, 0x9015], key)
        c += 1
        ix, iz = (int(w[0]) * W_) >> 32, (int(w[1]) * H_) >> 32
        if all((ix - a) ** 2 + (iz - b) ** 2 >= Rq * Rq for a, b in pts):
            pts.append((ix, iz))
    ref = np.array([[np.float32(a / 65536.0) - np.float32(0.5), np.float32(b / 65536.0) - np.float32(0.35)]
                    for a, b in pts], np.float32)
    assert np.array_equal(xz, ref)


def _heap_replica(vals, k):
    """heap.cuh semantics in plain Python (float32 sums), for tiny windows."""
    f = np.float32
    mx, mn = [], []  # python heaps: mx stores negatives
    value = f(0)
    for v in vals:
        v = f(v)
        value = f(value + v)
        if len(mx) < k:
            heapq.heappush(mx, -v)
            heapq.heappush(mn, v)
        elif mx and v < -mx[0]:
            heapq.heapreplace(mx, -v)
        elif mn and v > mn[0]:
            heapq.heapreplace(mn, v)
    return sorted(-x for x in mx), sorted(mn), value


def test_trimmed_mean_sorted_u32_matches_numpy():
    rng = np.random.default_rng(0)
    img = rng.integers(0, 50, (9, 13)).astype(np.uint32)
    img[4, 6] = 100000
    for r, ratio in [(2, 0.2), (1, 0.1), (3, 0.05), (0, 0.2)]:
        out = O.smooth_u32(img, r, ratio, 0)
        for y in range(9):
            for x in range(13):
                win = np.sort(img[max(y - r, 0):y + r + 1, max(x - r, 0):x + r + 1].ravel())
                k = int(np.float32(win.size) * np.float32(ratio))
                ref = np.float32(np.float32(win[k:win.size - k].sum()) / np.float32(win.size - 2 * k))
                assert out[y, x] == ref


def test_trimmed_mean_heaps_keep_the_reference_else_if_chain():
    # the window [1,2,3,4,5 | 4 | 0 ...]: the 4 goes to the max-heap only, so
    # the min-heap keeps the early 1 (heap.cuh:45-53); sorted trimming differs
    img = np.zeros((5, 5), np.float32)
    img[0, :] = [1, 2, 3, 4, 5]
    img[1, 0] = 4
    heaps = O.smooth_f32(img, 2, 0.2, 1)
    srt = O.smooth_f32(img, 2, 0.2, 0)
    assert heaps[2, 2] != srt[2, 2]
    lo, hi, value = _heap_replica(img.ravel(), 5)
    ref = np.float32(np.float32(np.float32(value - np.float32(sum(lo))) - np.float32(sum(hi))) / np.float32(15))
    assert heaps[2, 2] == ref


def test_trimmed_mean_heaps_equals_python_replica_on_random_maps():
    rng = np.random.default_rng(2)
    img = (rng.random((7, 11)) * 10).astype(np.float32)
    img[rng.random(img.shape) < 0.3] = 0
    out = O.smooth_f32(img, 2, 0.2, 1)
    for y in range(7):
        for x in range(11):
            win = img[max(y - 2, 0):y + 3, max(x - 2, 0):x + 3].ravel()
            k = int(np.float32(win.size) * np.float32(0.2))
            lo, hi, value = _heap_replica(win, k)
            s_lo = np.float32(0)
            for v in lo:
                s_lo = np.float32(s_lo + v)
            s_hi = np.float32(0)
            for v in hi:
                s_hi = np.float32(s_hi + v)
            # heap.sum() adds in array order; on these values the order does not change the float sum
            ref = np.float32(np.float32(np.float32(value - s_lo) - s_hi) / np.float32(win.size - 2 * k))
            assert abs(out[y, x] - ref) <= 1e-6 * max(1.0, abs(ref))


def test_grid_conservative_covers_every_rectangle():
    w, sc = dense_scene(0)
    cs, ent = sc.cell_start, sc.entries
    gd = list(sc.s.gdims)
    gp, gc = np.array(sc.s.gpos[:]), np.array(sc.s.gcell[:])
    for h in range(w.n):
        v = sc.vert[h].reshape(3, 3)
        for a in np.linspace(0, 1, 5):
            for b in np.linspace(0, 1, 5):
                p = v[0] + a * (v[1] - v[0]) + b * (v[2] - v[0])
                idx = np.clip(np.floor((p - gp) / gc).astype(int), 0, np.array(gd) - 1)
                c = (idx[0] * gd[1] + idx[1]) * gd[2] + idx[2]
                assert h in ent[cs[c]:cs[c + 1]]


def test_mid_field_hits_rarely_share_a_pixel_within_a_warp():
    """Why the tracer deposits with plain reductions and no warp aggregation:
    a warp's 32 rays start from one sample point (256 consecutive rays per
    point) and spread over metres at the receiver, so few of its hits land on
    a pixel that another lane of the same warp also hits.  Mid field (1000
    heliostats, 256 x 256 pixels of 4.7 cm), oracle records of 2^20 rays
    (32 768 warps) in 8 ranges spread over 2^22 rays: 0.28 % of hits share
    a pixel, so aggregating them would save 0.14 % of the reductions; bar
    1 %."""
    w = W.mid(rays=1 << 22)
    sc = O.Scene(w.pos, w.size, w.sigma, w.receiver, w.grid.cell[0], w.grid.margin, list(w.sun.dir), aim=w.aim)
    R, rpp = int(w.params.rays), int(w.params.rays_per_point)
    xz, helio = O.points_poisson(w.size, R // rpp, w.params.point_spacing, w.params.seed)
    weight = np.asarray(w.size[:, 0] * w.size[:, 2], np.float64) / np.bincount(helio, minlength=w.n)
    shared = hits = saved = 0
    for b in np.linspace(0, R - (1 << 17), 8).astype(np.int64) // 32 * 32:
        cfg = sc.cfg(w.sun.csr, w.params.seed, R, rpp, xz, helio, weight, ray_begin=int(b), ray_end=int(b) + (1 << 17))
        pix = np.asarray(sc.trace_philox(cfg, maps=False)["pixel"]).reshape(-1, 32)
        for lanes in pix:
            hit = lanes[lanes >= 0]
            _, inv, cnt = np.unique(hit, return_inverse=True, return_counts=True)
            shared += int((cnt[inv] > 1).sum())
            saved += hit.size - cnt.size
            hits += hit.size
    assert hits > (1 << 19)
    frac = shared / hits
    print("mid field: hits sharing a pixel with another lane of their warp %.4f %%, atomics aggregation would save %.4f %%"
          % (100 * frac, 100 * saved / hits))
    assert frac < 0.01, frac
