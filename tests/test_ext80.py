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


@pytest.mark.skipif(platform.machine() != "x86_64", reason="needs x87 long double")
def test_x87_quotient_of_doubles(tmp_path):
    """lsqdd.cuh x87_div_d, the SST LU-SGS diagonal's `long double` quotient stored to double, equals the
    host's x87 on random, exact and near-midpoint quotients -- where a plain double division differs
    (double rounding) in a few hundred cases."""
    exe = str(tmp_path / "x87div_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", exe,
                    os.path.join(ROOT, "tests", "native", "x87div_check.cpp")], check=True)
    r = subprocess.run([exe, "200000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(kv.split("=") for kv in r.stdout.split() if "=" in kv)
    assert f["mismatches"] == "0", r.stdout
    assert int(f["naive_differs"]) > 0, r.stdout  # the cases exercise the double rounding
    assert int(f["decided"]) > 0.999 * int(f["tried"]), r.stdout


@pytest.mark.skipif(platform.machine() != "x86_64", reason="needs x87 long double")
def test_certified_double_double_matches_x87(tmp_path):
    """lsqdd.cuh: the FP64 emulation of single x87 operations (accumulation step, product, sum) equals the
    host's x87 results on random, tie-prone, power-of-two and cancelling operands, and every gradient
    component the certified and exact-numerator solves return equals the x87 formula (random cells plus
    near-cancelling, one-directional, near-uniform and uniform fields); over 99 % of components decide."""
    exe = str(tmp_path / "lsqdd_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", exe,
                    os.path.join(ROOT, "tests", "native", "lsqdd_check.cpp")], check=True)
    r = subprocess.run([exe, "1000000"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    f = dict(kv.split("=") for kv in r.stdout.replace("|", " ").split() if "=" in kv)
    assert f["op_mismatches"] == "0" and f["mismatches"] == "0" and f["sum_mismatches"] == "0", r.stdout
    assert float(f["certified"]) + float(f["exact_numerator"]) > 0.99, r.stdout
