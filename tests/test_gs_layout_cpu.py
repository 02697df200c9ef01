"""The gather-scatter warp layout on the CPU: tests/native/gs_layout_check.cpp
is compiled against the library's headers and libnekob200.so, builds the
layout with the library's own gs_relayout on box meshes (masked, periodic,
scaled) and checks it and the kernel's lane arithmetic against the
sequential item-form sums, bit for bit."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_gs_warp_layout_bit_exact(tmp_path):
    import neko_b200
    neko_b200.load()  # the library exists (build() ran)
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    lib = os.path.join(ROOT, "neko_b200")
    exe = str(tmp_path / "gs_layout_check")
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(lib, "csrc"),
           "-I/usr/local/cuda/include", os.path.join(HERE, "native", "gs_layout_check.cpp"),
           "-L", lib, "-lnekob200", f"-Wl,-rpath,{lib}", "-L/usr/local/cuda/lib64", "-lcudart",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("bit-identical") == 7, r.stdout
