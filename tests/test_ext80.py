"""The device's x87 extended-precision model (csu_b200/csrc/cuda/ext80.cuh) against this x86-64 host's
long double: +, *, /, conversions and the reference's least-squares gradient formula, bit for bit."""
import os
import platform
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(platform.machine() != "x86_64", reason="needs x87 long double")
def test_ext80_matches_x87(tmp_path):
    exe = str(tmp_path / "ext80_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "native", "ext80_check.cpp")],
                   check=True)
    r = subprocess.run([exe, "400000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "add=0 mul=0 div=0 cvt=0 grad=0" in r.stdout
