"""INTEGRATION.md's drop-in code is the compiled file, not a copy that can drift."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_the_documented_dropin_is_the_compiled_file():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", doc, flags=re.S)
    src = open(os.path.join(ROOT, "tests", "dropin", "results_with_given_normal.cu")).read()
    assert src in blocks
