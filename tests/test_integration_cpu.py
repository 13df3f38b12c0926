"""The reference-side bindings shown in the integration guide (the C++ files a maintainer adds: one in
place of the reference's GPU translation unit, one in place of its swarm placement and ANM setup
calls) compile against the reference's own headers and this library's C header, with warnings as
errors for the bindings themselves."""
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
    section = re.search(r"## 2\. Reference-side binding(.*?)\n## 3\.", text, re.S)
    assert section, "binding section not found"
    blocks = re.findall(r"```cpp\n(.*?)```", section.group(1), re.S)
    assert len(blocks) == 2, "the hot-path binding and the setup binding"
    inc = []
    for d in ("source/dock/include", "source/prep/include", "source/json/include"):
        inc += ["-isystem", os.path.join(REFERENCE, d)]  # the reference's headers: their warnings are not ours
    for k, code in enumerate(blocks):
        src = tmp_path / f"binding_{k}.cc"
        src.write_text(code)
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror"] + inc +
                           ["-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True,
                           timeout=120)
        assert r.returncode == 0, f"block {k}: " + r.stderr[-3000:]
