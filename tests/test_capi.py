"""C-ABI library: loads, exports every declared symbol, host-only helpers.

No GPU is touched here; the host helpers (sun direction, Buie table, layout
generator, .scn parser) are pure host code inside libqmcrt.so.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from onemirror_b200 import capi, workloads as W
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qmcrt.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qmcrt_\w+)\s*\(", txt)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["qmcrt_scene_create", "qmcrt_scene_destroy", "qmcrt_trace", "qmcrt_trace_tables",
                 "qmcrt_smooth_trimmed_u32", "qmcrt_smooth_trimmed_f32", "qmcrt_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_functions()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (qmcrt_\w+)", out))
    assert set(names) <= exported
    # the Python binding covers the same set
    assert set(names) == set(capi.PROTOTYPES)


def test_argument_errors_need_no_gpu():
    """Entry points refuse NULL and out-of-range arguments with a status and a
    message before touching the device (these run on a machine without one)."""
    L = capi.lib()
    assert L.qmcrt_tape_energy(None, None, None) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_adjoint_loss(None, None, None, None, None, None) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_adjoint_replay(None, None, None, None, None) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_adjoint_backward(None, None, None, None) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_buie_sample_probe(C.c_float(0.1), None, 16, None, None) == capi.ERR_INVALID_ARGUMENT
    dummy = C.c_void_p(16)  # never dereferenced: the csr check comes first
    assert L.qmcrt_buie_sample_probe(C.c_float(1.5), dummy, 16, dummy, None) == capi.ERR_INVALID_ARGUMENT
    assert b"csr" in L.qmcrt_last_error()
    assert L.qmcrt_buie_sample_probe(C.c_float(0.1), dummy, 0, dummy, None) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_scene_set_timing(None, capi.TIMING_TRACE) == capi.ERR_INVALID_ARGUMENT
    assert L.qmcrt_scene_timing(None, None) == capi.ERR_INVALID_ARGUMENT


def test_version_and_status_strings():
    L = capi.lib()
    assert b"sm_100a" in L.qmcrt_version()
    assert L.qmcrt_status_string(capi.ERR_INVALID_ARGUMENT) == b"invalid argument"


def test_sun_direction_matches_reference_convention():
    # main.cpp:71-73: (-sin z sin a, -cos z, sin z cos a), z = zenith
    for el, az in [(45, 180), (30, 90), (20, 0), (89, 270)]:
        d = np.array(__import__("onemirror_b200.workloads", fromlist=["x"]).sun_dir(el, az))
        z, a = np.radians(90 - el), np.radians(az)
        ref = np.array([-np.sin(z) * np.sin(a), -np.cos(z), np.sin(z) * np.cos(a)])
        assert np.allclose(d, ref, atol=1e-7)
    d = (C.c_float * 3)()
    assert capi.lib().qmcrt_sun_direction(C.c_float(120.0), C.c_float(0.0), d) == capi.ERR_INVALID_ARGUMENT
    assert b"elevation" in capi.lib().qmcrt_last_error()


@pytest.mark.parametrize("csr", [0.05, 0.1, 0.2, 0.3])
def test_buie_table_is_the_oracles_bit_for_bit(csr):
    x = np.zeros(1025, np.float32)
    y = np.zeros(1025, np.float32)
    s = np.zeros(1024, np.float32)
    p = np.zeros(6, np.float32)
    capi.check(capi.lib().qmcrt_buie_table(C.c_float(csr), capi.as_fp(x), capi.as_fp(y), capi.as_fp(s), capi.as_fp(p)))
    ox, oy, os_, op = O.buie_table(csr)
    assert x.tobytes() == ox.tobytes() and y.tobytes() == oy.tobytes()
    assert s.tobytes() == os_.tobytes() and p.tobytes() == op.tobytes()
    assert np.all(np.diff(y) > 0) and np.all(s > 0)
    assert abs(x[-1] - 4.65) < 1e-4 and p[3] > p[2] > 0


@pytest.mark.parametrize("csr", [0.01, 0.1, 0.5, 0.9])
def test_buie_buckets_hold_one_interval_boundary_at_most(csr):
    """The tracer looks the Buie inverse CDF up through 2048 uniform buckets
    of [0, core): record b is the interval of the bucket's smallest value, and
    record b + 1 the next one, which is right as long as no bucket holds two
    interval boundaries.  A boundary y_k lies in bucket int(y_k * 2048 / core)
    (the kernel's float multiply).  The library refuses to build a table that
    breaks this; the core table does not depend on csr."""
    x = np.zeros(1025, np.float32)
    y = np.zeros(1025, np.float32)
    s = np.zeros(1024, np.float32)
    p = np.zeros(6, np.float32)
    capi.check(capi.lib().qmcrt_buie_table(C.c_float(csr), capi.as_fp(x), capi.as_fp(y), capi.as_fp(s), capi.as_fp(p)))
    inv = np.float32(2048) / p[2]
    buckets = (y[1:1024] * inv).astype(np.float32).astype(np.int64)
    assert len(np.unique(buckets)) == len(buckets)
    # the narrowest interval is the last one, 0.88 buckets wide
    assert np.diff(y.astype(np.float64)).min() * inv > 0.8


def test_buie_rejects_bad_csr():
    a = np.zeros(1025, np.float32)
    b = np.zeros(1024, np.float32)
    p = np.zeros(6, np.float32)
    assert capi.lib().qmcrt_buie_table(C.c_float(0.0), capi.as_fp(a), capi.as_fp(a), capi.as_fp(b),
                                       capi.as_fp(p)) == capi.ERR_INVALID_ARGUMENT


def test_layout_radial_staggered_properties():
    from onemirror_b200 import workloads as W
    for n, w, rmin, rmax, span in [(100, 2.0, 40.0, 200.0, 120.0), (1000, 10.0, 100.0, 600.0, 120.0),
                                   (3000, 11.0, 120.0, 1300.0, 360.0)]:
        pos = W.layout(n, w, w, rmin, rmax, az_span=span)
        assert pos.shape == (n, 3) and np.all(np.isfinite(pos))
        r = np.hypot(pos[:, 0], pos[:, 2])
        assert r.min() >= rmin - 1e-3 and r.max() <= rmax + 1e-3
        # no two mirrors closer than their diagonal (no overlap at any orientation)
        from scipy.spatial import cKDTree
        d, _ = cKDTree(pos[:, [0, 2]]).query(pos[:, [0, 2]], k=2)
        assert d[:, 1].min() >= np.sqrt(2) * w
        if span < 360:  # north field: z < 0 (z is south)
            assert np.all(pos[:, 2] < 0)
        again = W.layout(n, w, w, rmin, rmax, az_span=span)
        assert np.array_equal(pos, again)


def test_layout_rejects_impossible_fields():
    p = capi.LayoutParams()
    p.n, p.helio_w, p.helio_h, p.r_min, p.r_max, p.az_span_deg = 10000, 10.0, 10.0, 100.0, 110.0, 30.0
    got = C.c_int32()
    assert capi.lib().qmcrt_layout_radial_staggered(C.byref(p), None, 0, C.byref(got)) == capi.ERR_INVALID_ARGUMENT


def _parse(path):
    L = capi.lib()
    rv, gp, n = capi.Receiver(), capi.GridParams(), C.c_int32()
    capi.check(L.qmcrt_scn_parse(path.encode(), C.byref(rv), C.byref(gp), None, None, 0, C.byref(n)))
    pos = np.zeros((n.value, 3), np.float32)
    size = np.zeros((n.value, 3), np.float32)
    capi.check(L.qmcrt_scn_parse(path.encode(), C.byref(rv), C.byref(gp), capi.as_fp(pos), capi.as_fp(size),
                                 n.value, C.byref(n)))
    return rv, gp, pos, size


def test_scn_parser_reads_the_reference_format():
    rv, gp, pos, size = _parse(os.path.join(ROOT, "tests", "golden", "tiny_field.scn"))
    assert pos.shape == (4, 3)
    assert np.allclose(pos[3], [6.0, 1.5, -20.0]) and np.allclose(size[3], [3.0, 0.1, 1.5])
    assert rv.type == 0 and list(rv.pos) == [0.0, 20.0, 0.0] and rv.face == 0
    assert (rv.res_x, rv.res_y) == (300, 250)  # size * 1/0.01 m
    assert gp.explicit_bounds == 1 and list(gp.cell) == [5.0, 5.0, 5.0]
    assert list(gp.origin) == [-20.0, -1.0, -40.0]


def test_scn_parser_reference_sample_if_present():
    path = os.path.join(os.environ.get("QMCRT_REFERENCE_ROOT", "/root/reference"), "Hu_smooth", "userData",
                        "face2face_shadow.scn")
    if not os.path.exists(path):
        pytest.skip("reference tree not mounted")
    rv, gp, pos, size = _parse(path)
    assert pos.shape[0] == 1 and size[0, 1] > 0
    assert gp.cell[0] > 0 and rv.size[0] > 0


def test_scn_parser_errors(tmp_path):
    L = capi.lib()
    n = C.c_int32()
    assert L.qmcrt_scn_parse(b"/nonexistent.scn", None, None, None, None, 0, C.byref(n)) == capi.ERR_INVALID_ARGUMENT
    bad = tmp_path / "bad.scn"
    bad.write_text("Recv 0\npos 0 1 2\nend\nGrid 0\ninter 1 1 1\nn 2\nend\ngap 0 0\nmatrix 1 1\nhelio 0 0 0\n1 0.1 1\n")
    assert L.qmcrt_scn_parse(str(bad).encode(), None, None, None, None, 0, C.byref(n)) == capi.ERR_INVALID_ARGUMENT
    assert b"declares 2" in L.qmcrt_last_error()


def _reference_facets(a, b, n, centre):
    """The 3 x 3 facet layout of SceneFileProc::SceneFileRead
    (scene_file_proc.cpp:288-341) restated in float64: centres on the local
    lattice +-(sqrt(2)/3 + 0.1), heights x^2/a^2 + z^2/b^2, the frame
    mirrorToGround with e1 = (n.z, 0, -n.x) / sqrt(n.x^2 + n.y^2) (sign by
    n.z), n, e1 x n, and normals (-2x/a^2, 1, -2z/b^2) through the same frame."""
    d = np.sqrt(2.0) / 3 + 0.1
    cx = np.array([-d, 0, d] * 3)
    cz = np.repeat([-d, 0.0, d], 3)
    cy = cx * cx / a / a + cz * cz / b / b
    t = np.sqrt(n[0] ** 2 + n[1] ** 2)
    if n[2] > 0:
        e1 = np.array([n[2] / t, 0, -n[0] / t])
    elif n[2] < 0:
        e1 = np.array([-n[2] / t, 0, n[0] / t])
    else:
        e1 = np.array([0.0, 0, 1])
    M = np.stack([e1, n, np.cross(e1, n)], 1)
    pos = (M @ np.stack([cx, cy, cz])).T + centre
    nrm = (M @ np.stack([-2 * cx / a / a, np.ones(9), -2 * cz / b / b])).T
    return pos, nrm / np.linalg.norm(nrm, axis=1, keepdims=True)


def test_paraboloid_facets_reproduce_the_reference_layout():
    n = np.array([0.3, 0.9, -0.2])
    n /= np.linalg.norm(n)
    centre = np.array([1.0, 2.0, 100.0])
    pos, size, nrm = W.paraboloid_facets(8.0, 8.0, n, centre, reference_frame=True)
    rp, rn = _reference_facets(8.0, 8.0, n.astype(np.float32).astype(np.float64), centre)
    assert np.allclose(pos, rp, atol=2e-5) and np.allclose(nrm, rn, atol=1e-6)
    assert np.allclose(size, [[np.sqrt(2) / 3, 0.1, np.sqrt(2) / 3]] * 9, atol=1e-7)


def test_paraboloid_facets_corrected_frame_geometry():
    n = np.array([0.3, 0.9, -0.2])
    n /= np.linalg.norm(n)
    centre = np.array([1.0, 2.0, 100.0])
    pos, size, nrm = W.paraboloid_facets(6.0, 9.0, n, centre, rows=3, cols=5, facet=0.5, gap=0.05)
    e1 = np.array([-n[2], 0, n[0]]) / np.hypot(n[0], n[2])  # n.z < 0 branch
    e2 = np.cross(e1, n)
    rel = pos.astype(np.float64) - centre
    x, y, z = rel @ e1, rel @ n, rel @ e2
    assert np.allclose(y, x * x / 36 + z * z / 81, atol=2e-5)
    assert np.allclose(np.unique(np.round(x, 4)), (np.arange(5) - 2) * 0.55, atol=1e-4)
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1, atol=1e-6)
    g = np.stack([-2 * x / 36, np.ones_like(x), -2 * z / 81], 1)
    gw = g[:, :1] * e1 + g[:, 1:2] * n + g[:, 2:] * e2
    assert np.allclose(nrm, gw / np.linalg.norm(gw, axis=1, keepdims=True), atol=1e-6)
    with pytest.raises(capi.QmcrtError):
        W.paraboloid_facets(0.0, 8.0, n, centre)
