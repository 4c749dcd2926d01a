"""The ctypes binding (onemirror_b200/capi.py) against the C header.

Every `typedef struct qmcrt_* {...}` of include/qmcrt.h must have a ctypes
twin with the same members in the same order, and a C compiler must place
them where ctypes does: a small C program built here with gcc prints
sizeof and offsetof of every member, compared with ctypes.sizeof and the
fields' offsets.  A drift would otherwise pass arguments silently shifted.
"""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from onemirror_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "qmcrt.h")

# C struct -> ctypes class
TWINS = {
    "qmcrt_field": capi.Field, "qmcrt_receiver": capi.Receiver, "qmcrt_grid_params": capi.GridParams,
    "qmcrt_sun": capi.Sun, "qmcrt_trace_params": capi.TraceParams, "qmcrt_outputs": capi.Outputs,
    "qmcrt_trace_stats": capi.TraceStats, "qmcrt_table_inputs": capi.TableInputs, "qmcrt_grid_info": capi.GridInfo,
    "qmcrt_layout_params": capi.LayoutParams, "qmcrt_facet_params": capi.FacetParams,
    "qmcrt_batch_item": capi.BatchItem, "qmcrt_batch_tuning": capi.BatchTuning, "qmcrt_timing": capi.Timing,
    "qmcrt_smooth_params": capi.SmoothParams,
}


def header_structs():
    """{name: [member names in order]} of every typedef'd struct in the header."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for name, body, alias in re.findall(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        assert name == alias
        members = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "float helio_w, helio_h" / "const float* pos" / "float pos[3]" / "qmcrt_sun sun"
            head, *rest = [p.strip() for p in decl.split(",")]
            first = re.sub(r"\[.*?\]", "", head).replace("*", " ").split()[-1]
            members.append(first)
            members += [re.sub(r"\[.*?\]", "", r).replace("*", " ").split()[-1] for r in rest]
        out[name] = members
    return out


def test_every_header_struct_has_a_ctypes_twin_with_the_same_members():
    structs = header_structs()
    assert set(structs) == set(TWINS), set(structs) ^ set(TWINS)
    for name, members in structs.items():
        assert [f[0] for f in TWINS[name]._fields_] == members, name


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_sizes_and_offsets_equal_the_c_compilers(tmp_path):
    structs = header_structs()
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "qmcrt.h"', "int main(void) {"]
    for name, members in structs.items():
        lines.append('  printf("%s sizeof %%zu\\n", sizeof(%s));' % (name, name))
        for m in members:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (name, m, name, m))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        struct, member, value = ln.split()
        got[(struct, member)] = int(value)
    for name, members in structs.items():
        cls = TWINS[name]
        assert got[(name, "sizeof")] == C.sizeof(cls), name
        for m in members:
            assert got[(name, m)] == getattr(cls, m).offset, (name, m)


def test_every_declared_function_has_a_prototype():
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    declared = set(re.findall(r"\b(qmcrt_\w+)\s*\(", text))
    assert declared == set(capi.PROTOTYPES), declared ^ set(capi.PROTOTYPES)


def header_enum_values():
    """{name: value} of every QMCRT_* enumerator of the header (values are
    integer literals, shifts and ors)."""
    text = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    out = {}
    for body in re.findall(r"enum(?:\s+\w+)?\s*\{(.*?)\}", text, flags=re.S):
        for item in body.split(","):
            m = re.match(r"\s*(QMCRT_\w+)\s*=\s*([0-9xXa-fA-Fu<>| ()]+?)\s*$", item)
            if m:
                expr = re.sub(r"(?<=[0-9a-fA-F])[uU]\b", "", m.group(2))
                assert re.fullmatch(r"[0-9xXa-fA-F<>| ()]+", expr), expr
                out[m.group(1)] = eval(expr)  # noqa: S307  (checked above: literals, shifts and ors only)
    return out


def test_header_constants_equal_the_bindings():
    """The binding's constants (QUIRK_*, TIMING_*, TRIM_*, ...) carry the
    header's values, so a caller through ctypes passes the same bits as one
    compiled against include/qmcrt.h."""
    values = header_enum_values()
    assert values["QMCRT_TIMING_ALL"] == values["QMCRT_TIMING_TRACE"] | values["QMCRT_TIMING_SETUP"] | \
        values["QMCRT_TIMING_FINALIZE"]
    checked = 0
    for name, v in values.items():
        short = name[len("QMCRT_"):]
        if hasattr(capi, short):
            assert getattr(capi, short) == v, name
            checked += 1
    for short in ("TIMING_TRACE", "TIMING_SETUP", "TIMING_FINALIZE", "TIMING_ALL", "TRIM_SORTED", "SMOOTH_COUNTS",
                  "QUIRK_PIXEL_EDGE", "QUIRKS_REFERENCE"):
        assert hasattr(capi, short) and "QMCRT_" + short in values, short
    assert checked >= 20, checked
