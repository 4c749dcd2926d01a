"""Generates tests/golden/ref_gpu_vectors.npz from the REFERENCE's own CUDA
code (oracle/_ref/libref.so, built by oracle/ref.mk from the reference
sources; oracle/ref_harness.cu drives it).  Needs a GPU:

    make -C oracle -f ref.mk && make -C oracle && python tests/golden/gen_ref_gpu_vectors.py [out.npz]

Three pins, all on seeded inputs:
  smooth_*  ImageSmoother::image_smooth (image_smooth.cu:60-115) on float maps;
  grid_*    RectGrid::CGridHelioMatch (grid.cpp:25-83) on the 100-heliostat field;
  trace_*   map_tracing through ray_tracing (rectgrid_raytracing.cu:155-196,
            ray_tracing.cu:3-32), one launch per heliostat as
            recthelio_ray_tracing does, on a 9-heliostat scene with explicit
            sun-shape and perturbation tables; the raw receiver image.

Every input is checked on the CPU before the reference runs, against the
out-of-range accesses that reading the reference shows:
  - trimmed_mean reads one heap slot past its share of shared memory when a
    window trims nothing (k = 0): every window here trims at least one value;
  - boxIntersect indexes a host vector with the truncated cell of each
    registration cube: every cube lies inside the grid;
  - NotCollision indexes the grid with the origin's cell: every sample point
    lies inside the grid;
  - receiver_drawing writes row u*res_y without clamping (u = 1 is one row
    past the image): an oracle trace of the same tables first shows that every
    ray that reaches the receiver plane lands at least 2 pixels inside the
    edges, far beyond the FP32/FP64 difference.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from onemirror_b200 import capi  # noqa: E402  (constants only)
from oracle import oracle as O  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libref.so")
fp = C.POINTER(C.c_float)
ip = C.POINTER(C.c_int)
i64p = C.POINTER(C.c_longlong)


def P(a, t=fp):
    return a.ctypes.data_as(t)


class Rec:
    """Receiver description in the oracle's attribute layout."""

    def __init__(self, pos, size, normal, face, res_x, res_y):
        self.type = 0
        self.pos, self.size, self.normal = list(pos), list(size), list(normal)
        self.face, self.res_x, self.res_y = face, res_x, res_y


def smoothing(L, rng, out):
    L.ref_image_smooth.argtypes = [fp, C.c_int, C.c_int, C.c_int, C.c_float, fp]
    cases = []
    for k, (w, h, r, ratio) in enumerate([(37, 29, 2, 0.2), (64, 48, 3, 0.1), (33, 40, 2, 0.3)]):
        img = rng.poisson(6.0, (h, w)).astype(np.float32)
        img[rng.random((h, w)) < 0.2] = 0
        if k == 1:
            img = (img * rng.uniform(0.5, 2.0, (h, w))).astype(np.float32)  # non-integer values
        # every window keeps k = int(cnt*ratio) >= 1 (corner windows are the
        # smallest) and needs k+1 <= heap slots (the interior window's)
        heap = int(np.float32((2 * r + 1) ** 2) * np.float32(ratio) + np.float32(1))
        for cnt in {(r + 1) ** 2, (r + 1) * (2 * r + 1), (2 * r + 1) ** 2}:
            kk = int(np.float32(cnt) * np.float32(ratio))
            assert 1 <= kk and kk + 1 <= heap and cnt - 2 * kk > 0, (cnt, kk, heap)
        res = np.zeros_like(img)
        assert L.ref_image_smooth(P(img), w, h, r, C.c_float(ratio), P(res)) == 0
        out["smooth_in_%d" % k], out["smooth_out_%d" % k] = img, res
        cases.append((r, ratio))
    out["smooth_params"] = np.array(cases, np.float32)


def aimed_normals(pos, target, sun):
    """Unit bisectors of the reversed sun direction and the direction to `target` (float32)."""
    to_t = target[None, :] - pos
    to_t /= np.linalg.norm(to_t, axis=1, keepdims=True)
    n = to_t - sun[None, :] / np.linalg.norm(sun)
    return (n / np.linalg.norm(n, axis=1, keepdims=True)).astype(np.float32)


def grid_match(L, out):
    L.ref_grid_match.argtypes = [C.c_int, fp, fp, fp, fp, fp, fp, ip, ip, ip, C.c_int]
    L.ref_grid_match.restype = C.c_int
    rng = np.random.default_rng(20261204)
    n = 100
    pos = np.stack([rng.uniform(-60, 60, n), rng.uniform(1.2, 2.0, n), rng.uniform(-160, -40, n)], 1).astype(np.float32)
    size = np.stack([rng.uniform(1.5, 10, n), np.full(n, 0.1), rng.uniform(1.5, 10, n)], 1).astype(np.float32)
    sun = np.array([0.0, -0.7, 0.7], np.float32)
    normal = aimed_normals(pos, np.array([0, 80, 0], np.float32), sun)
    inter = np.array([10.0, 10.0, 10.0], np.float32)
    gpos = np.array([-80.0, -10.0, -180.0], np.float32)
    gsize = np.array([160.0, 30.0, 160.0], np.float32)
    dims = np.ceil(gsize / inter).astype(int)
    rad = np.sqrt(np.linalg.norm(size, axis=1)) / 2
    lo = ((pos - rad[:, None]) - gpos) / inter
    hi = ((pos + rad[:, None]) - gpos) / inter
    assert lo.min() >= 0 and np.all(hi.astype(int) <= dims - 1)
    dims_out = np.zeros(3, np.int32)
    cap = 1 << 16
    start = np.zeros(int(np.prod(dims)) + 1, np.int32)
    ent = np.zeros(cap, np.int32)
    nm = L.ref_grid_match(n, P(pos), P(size), P(normal), P(gpos), P(gsize), P(inter), P(dims_out, ip), P(start, ip),
                          P(ent, ip), cap)
    assert nm > 0
    out.update(grid_pos=pos, grid_size=size, grid_normal=normal, grid_gpos=gpos, grid_gsize=gsize, grid_inter=inter,
               grid_dims=dims_out, grid_start=start, grid_entries=ent[:nm])


def trace(L, out):
    L.ref_trace_tables.argtypes = [C.c_int, fp, fp, fp, fp, fp, fp, fp, fp, fp, C.c_int, C.c_int, C.c_float, fp,
                                   C.c_int, C.c_int, fp, fp, ip, C.c_longlong, fp, ip, i64p, fp]
    L.ref_trace_tables.restype = C.c_int
    L.ref_receiver_vertices.argtypes = [fp, fp, fp, C.c_int, C.c_int, fp, ip]
    rng = np.random.default_rng(20261205)
    # nine 2x2 m mirrors north of a 10 m tower (the reference's 9-facet
    # arrangement), close to the world origin
    xs, zs = np.meshgrid([-4.0, 0.0, 4.0], [-9.0, -12.0, -15.0])
    n = 9
    pos = np.stack([xs.ravel() + rng.uniform(-0.3, 0.3, n), np.full(n, 1.5), zs.ravel()], 1).astype(np.float32)
    size = np.tile(np.array([[2.0, 0.1, 2.0]], np.float32), (n, 1))
    sun = np.array([0.25, -0.8, 0.55], np.float32)
    sun /= np.linalg.norm(sun)
    rpos = np.array([0.0, 10.0, 0.0], np.float32)
    rsize = np.array([8.0, 8.0, 0.5], np.float32)
    rnorm = np.array([0.0, 0.0, -1.0], np.float32)
    face, ginfo, pl = 0, 16, 0.05
    normal = aimed_normals(pos, rpos, sun)
    gpos = np.array([-8.0, -1.0, -19.0], np.float32)
    gsize = np.array([16.0, 8.0, 16.0], np.float32)
    inter = np.array([2.5, 2.5, 2.5], np.float32)
    dims = np.ceil(gsize / inter).astype(int)
    # RectangleReceiver::Cset_resolution (receiver.cpp:41-45): size * geometry_info
    res_x, res_y = int(np.float32(rsize[0]) * np.float32(ginfo)), int(np.float32(rsize[1]) * np.float32(ginfo))
    v4 = np.zeros(12, np.float32)
    res = np.zeros(2, np.int32)
    L.ref_receiver_vertices(P(rpos), P(rsize), P(rnorm), face, ginfo, P(v4), P(res, ip))
    assert (int(res[0]), int(res[1])) == (res_x, res_y), res
    groups, lights = 64, 64
    T = groups * lights
    th = np.sqrt(rng.random(T)) * 0.0046
    ph = rng.random(T) * 2 * np.pi
    sun_local = np.stack([np.sin(th) * np.cos(ph), np.cos(th), np.sin(th) * np.sin(ph)], 1).astype(np.float32)
    ts = np.abs(rng.normal(0, 0.002, T))
    tp = rng.random(T) * 2 * np.pi
    turb_local = np.stack([np.sin(ts) * np.cos(tp), np.cos(ts), np.sin(ts) * np.sin(tp)], 1).astype(np.float32)
    xz, helio = O.points_grid(size, pl)
    start = rng.integers(0, T, len(helio)).astype(np.int32)
    # CPU checks before the reference runs: sample points inside the grid,
    # registration cubes inside the grid, and every ray that reaches the
    # receiver plane lands >= 2 pixels inside its edges
    rad = np.sqrt(np.linalg.norm(size, axis=1)) / 2
    assert ((pos - rad[:, None]) - gpos).min() >= 0 and np.all((((pos + rad[:, None]) - gpos) / inter).astype(int) <= dims - 1)
    assert np.all(np.abs(pos[:, [0, 2]] - (gpos + gsize / 2)[[0, 2]]) + 1.5 < gsize[[0, 2]] / 2)
    rec = Rec(rpos, rsize, rnorm, face, res_x, res_y)
    q = capi.QUIRK_SKIP_ORIGIN_CELL | capi.QUIRK_AABB_RADIUS | capi.QUIRK_PREV_PERTURB | capi.QUIRK_PIXEL_EDGE
    osc = O.Scene(pos, size, 0.0, rec, float(inter[0]), 0.0, list(sun), quirks=q, normal=normal,
                  grid_bounds=(list(gpos), list(inter), list(dims)))
    cfg = osc.cfg(0.1, 1, len(helio) * lights, lights, xz, helio, quirks=q)
    o = osc.trace_tables(cfg, sun_local, turb_local, start)
    fl, px = o["flags"], o["pixel"]
    reached = (fl & 3) == 0
    assert np.all(fl[reached] & 4), "a ray that passed both traversals missed the receiver"
    assert not np.any(fl & 8)
    rows, cols = px[reached] // res_x, px[reached] % res_x
    assert rows.min() >= 2 and rows.max() <= res_y - 3 and cols.min() >= 2 and cols.max() <= res_x - 3
    image = np.zeros(res_x * res_y, np.float32)
    npts = C.c_longlong()
    ms = C.c_float()
    rc = L.ref_trace_tables(n, P(pos), P(size), P(normal), P(gpos), P(gsize), P(inter), P(rpos), P(rsize), P(rnorm),
                            face, ginfo, pl, P(sun), groups, lights, P(sun_local), P(turb_local), P(start, ip),
                            len(helio), P(image), P(res, ip), C.byref(npts), C.byref(ms))
    assert rc == 0 and npts.value == len(helio), (rc, npts.value, len(helio))
    rays = len(helio) * lights
    print("reference map_tracing: %d rays in %.3f ms (%.3g rays/s), oracle hit %.4f, shadowed %.4f, blocked %.4f"
          % (rays, ms.value, rays / (ms.value * 1e-3), (fl & 4).mean() / 4, (fl & 1).mean(), (fl & 2).mean() / 2))
    out.update(trace_pos=pos, trace_size=size, trace_normal=normal, trace_sun=sun, trace_rpos=rpos, trace_rsize=rsize,
               trace_rnorm=rnorm, trace_res=np.array([res_x, res_y], np.int32), trace_gpos=gpos, trace_gsize=gsize,
               trace_inter=inter, trace_pl=np.float32(pl), trace_lights=np.int32(lights),
               trace_sun_local=sun_local, trace_turb_local=turb_local, trace_start=start,
               trace_image=image.reshape(res_y, res_x), trace_ref_ms=np.float32(ms.value))


def main():
    dst = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gpu_vectors.npz")
    L = C.CDLL(LIB)
    out = {}
    smoothing(L, np.random.default_rng(20261206), out)
    grid_match(L, out)
    trace(L, out)
    np.savez_compressed(dst, **out)
    print("wrote", len(out), "arrays to", dst)


if __name__ == "__main__":
    main()
