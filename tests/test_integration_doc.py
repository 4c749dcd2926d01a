"""INTEGRATION.md's drop-in code is the compiled file, not a copy that can drift."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_the_documented_dropin_is_the_compiled_file():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", doc, flags=re.S)
    src = open(os.path.join(ROOT, "tests", "dropin", "results_with_given_normal.cu")).read()
    assert src in blocks


def test_every_declared_function_is_named_in_the_integration_guide():
    header = open(os.path.join(ROOT, "include", "qmcrt.h")).read()
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    declared = set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(qmcrt_\w+)\(", header, flags=re.M))
    assert len(declared) > 40
    missing = sorted(f for f in declared if f not in doc)
    assert not missing, missing
