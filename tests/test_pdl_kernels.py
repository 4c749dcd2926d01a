"""Every kernel the library launches with programmatic dependent launch opens
with pdl_wait(): under programmatic stream serialization a kernel may start
while the one before it in the stream is still running, so it must not touch
memory before griddepcontrol.wait (a source check, no GPU needed)."""
import glob
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "onemirror_b200", "csrc")


def sources():
    out = {}
    for p in glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")):
        out[p] = open(p).read()
    return out


def launched_with_pdl(srcs):
    names = set()
    for s in srcs.values():
        for m in re.finditer(r"launch_pdl\(\s*[^,]+,\s*([A-Za-z_]\w*)", s):
            if m.group(1) != "k":
                names.add(m.group(1))
        # launch_trace instantiates trace_kernel and passes it as `k`
        if re.search(r"auto k = trace_kernel<", s) and "launch_pdl(true, k," in s:
            names.add("trace_kernel")
    return names


def test_pdl_kernels_wait_before_touching_memory():
    srcs = sources()
    names = launched_with_pdl(srcs)
    assert {"aim_kernel", "cand_kernel", "point_mask_kernel", "trace_kernel", "finalize_kernel",
            "smooth_sorted_kernel"} <= names, names
    for name in names:
        bodies = []
        for s in srcs.values():
            for m in re.finditer(r"__global__[^;{]*?\b" + name + r"\s*\(", s):
                j = s.find("{", m.end())
                bodies.append(s[j + 1:j + 200])
        assert bodies, name
        for b in bodies:
            first = b.strip().split(";")[0].strip()
            assert first == "pdl_wait()", (name, first)
