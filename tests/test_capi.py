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

from onemirror_b200 import capi
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
    path = "/root/reference/Hu_smooth/userData/face2face_shadow.scn"
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
