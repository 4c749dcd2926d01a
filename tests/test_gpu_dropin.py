"""The drop-in replacement of the reference's results_with_given_normal
(Gtest.cu:10-63), compiled against the reference's own headers.

tests/dropin/results_with_given_normal.cu is the C++ a maintainer of the
reference puts in place of its per-heliostat loop; oracle/ref.mk compiles it
with the reference's headers and links it with the reference's classes
(libref.so) and this library (libqmcrt.so) into oracle/_ref/libdropin.so.  A
harness builds a real SolarScene from arrays with the reference's classes.
These tests run it on the 9-heliostat scene of the reference's own GPU pin
and check that it gives what the Python binding of the same C-ABI gives for
the same inputs and seed: identical integer counts and count smoothing,
flux maps to float-atomic ordering, and the reference's two result files.
"""
import ctypes as C
import os

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from onemirror_b200.scene import SolarScene, write_intercept_ratio  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libdropin.so")
LIGHTS = 256
SEED = 2018  # the seed results_with_given_normal passes
fp = C.POINTER(C.c_float)


@pytest.fixture(scope="module")
def scene():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libdropin.so is not built (needs the reference sources at build time)")
    capi.lib()
    L = C.CDLL(LIB)
    g = np.load(os.path.join(ROOT, "tests", "golden", "ref_gpu_vectors.npz"))
    s = {k: np.ascontiguousarray(g["trace_" + k], np.float32) for k in
         ("pos", "size", "normal", "gpos", "gsize", "inter", "rpos", "rsize", "rnorm", "sun")}
    s["pixel"], s["ginfo"], s["sigma"], s["csr"], s["dni"] = 0.05, 16, 0.002, 0.1, 1000.0
    # the harness runs RectGrid::CGridHelioMatch: every registration cube
    # (half-side sqrt(|size|)/2, grid.cpp:49-59) must lie inside the grid
    dims = np.ceil(s["gsize"] / s["inter"]).astype(int)
    rad = np.sqrt(np.linalg.norm(s["size"], axis=1)) / 2
    assert ((s["pos"] - rad[:, None]) - s["gpos"]).min() >= 0
    assert np.all((((s["pos"] + rad[:, None]) - s["gpos"]) / s["inter"]).astype(int) <= dims - 1)
    return L, s


def args(s):
    P = lambda k: s[k].ctypes.data_as(fp)  # noqa: E731
    return [len(s["pos"]), P("pos"), P("size"), P("normal"), P("gpos"), P("gsize"), P("inter"), P("rpos"), P("rsize"),
            P("rnorm"), 0, s["ginfo"], C.c_float(s["pixel"]), P("sun"), C.c_float(s["dni"]), C.c_float(s["csr"]),
            C.c_float(s["sigma"]), LIGHTS]


def dropin(L, s, radius, ratio, method, source):
    res = int(s["rsize"][0] * s["ginfo"]) * int(s["rsize"][1] * s["ginfo"])
    counts = np.zeros(res, np.uint32)
    flux = np.zeros(res, np.float32)
    sm = np.zeros(res, np.float32)
    ro = np.zeros(2, np.int32)
    st = np.zeros(4, np.float64)
    nrm = np.zeros_like(s["normal"])
    sun = np.zeros(3, np.float32)
    rc = L.dropin_results(*args(s), C.c_ulonglong(SEED), radius, C.c_float(ratio), method, source,
                          counts.ctypes.data_as(C.POINTER(C.c_uint32)), flux.ctypes.data_as(fp), sm.ctypes.data_as(fp),
                          ro.ctypes.data_as(C.POINTER(C.c_int)), st.ctypes.data_as(C.POINTER(C.c_double)),
                          nrm.ctypes.data_as(fp), sun.ctypes.data_as(fp))
    assert rc == 0
    # the reference's objects hold the inputs re-normalised in float
    assert np.allclose(nrm, s["normal"], atol=1e-6) and np.allclose(sun, s["sun"], atol=1e-6)
    shape = (int(ro[1]), int(ro[0]))
    return counts.reshape(shape), flux.reshape(shape), sm.reshape(shape), st, nrm, sun


def python_side(s, radius, ratio, method, source, normal=None, sun_dir=None):
    """The same scene through the Python binding of the C-ABI (with the
    normals and sun direction the drop-in passed on, when given)."""
    rec = capi.Receiver()
    rec.type = capi.RECEIVER_FLAT
    rec.pos[:], rec.size[:], rec.normal[:] = list(s["rpos"]), list(s["rsize"]), list(s["rnorm"])
    rec.face = 0
    rec.res_x, rec.res_y = int(s["rsize"][0] * s["ginfo"]), int(s["rsize"][1] * s["ginfo"])
    gp = capi.GridParams()
    gp.cell[:], gp.origin[:], gp.extent[:] = list(s["inter"]), list(s["gpos"]), list(s["gsize"])
    gp.explicit_bounds, gp.fine_div = 1, 1
    sc = SolarScene(s["pos"], s["size"], rec, gp, sigma=s["sigma"], normal=s["normal"] if normal is None else normal)
    sun = capi.Sun()
    sun.dir[:] = list(s["sun"] if sun_dir is None else sun_dir)
    sun.dni, sun.csr = s["dni"], s["csr"]
    p = W.params(0, LIGHTS, s["pixel"], seed=SEED, mode=capi.POINTS_GRID)
    out = sc.results_host(sun, p, radius, ratio, method, source, stats=True)
    sc.close()
    return out


def test_dropin_equals_the_binding_on_counts_and_count_smoothing(scene):
    L, s = scene
    counts, flux, sm, st, nrm, sun = dropin(L, s, 2, 0.2, capi.TRIM_SORTED, capi.SMOOTH_COUNTS)
    py = python_side(s, 2, 0.2, capi.TRIM_SORTED, capi.SMOOTH_COUNTS, nrm, sun)
    assert counts.sum() > 0 and np.array_equal(counts, py["counts"])
    assert sm.tobytes() == py["smoothed"].tobytes()
    assert np.allclose(flux, py["flux"], rtol=0, atol=1e-5 * flux.max())
    assert st[0] == py["stats"].rays and st[1] == py["stats"].hit
    assert abs(st[3] - py["stats"].intercept_ratio) < 1e-6


def test_dropin_smooths_the_energy_image_as_the_reference_does(scene):
    L, s = scene
    counts, flux, sm, _, nrm, sun = dropin(L, s, 5, 0.02, capi.TRIM_HEAPS, capi.SMOOTH_ENERGY)
    py = python_side(s, 5, 0.02, capi.TRIM_HEAPS, capi.SMOOTH_ENERGY, nrm, sun)
    assert np.array_equal(counts, py["counts"])
    assert np.allclose(sm, py["smoothed"], rtol=0, atol=1e-5 * sm.max())
    # a smoothed flux map: same total scale as the flux, spread out
    assert sm.max() < flux.max() and abs(sm.sum() / flux.sum() - 1) < 0.05


def test_results_with_given_normal_writes_the_reference_result_files(scene, tmp_path):
    L, s = scene
    ns, sm = tmp_path / "nonsmooth.txt", tmp_path / "smooth.txt"
    assert L.dropin_results_with_given_normal(*args(s), str(ns).encode(), str(sm).encode()) == 0
    _, _, _, _, nrm, sun_used = dropin(L, s, 5, 0.02, capi.TRIM_HEAPS, capi.SMOOTH_ENERGY)
    py = python_side(s, 5, 0.02, capi.TRIM_HEAPS, capi.SMOOTH_ENERGY, nrm, sun_used)
    # total energy as Gtest.cu:29,39-44: sum |n . sun| DNI w h, times rho / S_rec
    sun = s["sun"] / np.linalg.norm(s["sun"])
    total = np.float32(0)
    for n, size in zip(s["normal"], s["size"]):
        total += np.float32(abs(np.float32(np.dot(n, sun)) * np.float32(s["dni"]) * size[0] * size[2]))
    total *= np.float32(0.88) / np.float32((1.0 / s["ginfo"]) ** 2)
    for path, m in ((ns, py["flux"]), (sm, py["smoothed"])):
        got = float(path.read_text().split()[0])
        want = write_intercept_ratio(None, m, float(total))
        assert 0 < got < 1 and abs(got - want) <= 2e-5 * want, (path.name, got, want)
