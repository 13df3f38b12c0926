"""The reference-side binding shown in INTEGRATION.md (the C++ file a maintainer adds in place of
the reference's GPU translation unit) compiles against the reference's own headers and this
library's C header, with warnings as errors for the binding itself."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = "/root/reference"


def test_reference_binding_compiles(tmp_path):
    if not os.path.isdir(os.path.join(REFERENCE, "source", "dock", "include")):
        pytest.skip("reference tree not present")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"## 2\. Reference-side binding.*?```cpp\n(.*?)```", text, re.S)
    assert m, "binding snippet not found"
    src = tmp_path / "cal_gso_tasks_b200.cc"
    src.write_text(m.group(1))
    inc = []
    for d in ("source/dock/include", "source/prep/include", "source/json/include"):
        inc += ["-isystem", os.path.join(REFERENCE, d)]  # the reference's headers: their warnings are not ours
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror"] + inc +
                       ["-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
