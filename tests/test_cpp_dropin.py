"""The C++ drop-in headers (grid-calculus_b200/include/gridcalc) compile
against the C ABI with g++ (CPU), and the reference-style test program built
from them passes on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp")
LIBDIR = os.path.join(ROOT, "grid-calculus_b200", "lib")


def _compile(out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", SRC, "-o", out,
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "grid-calculus_b200", "include"),
           "-L", LIBDIR, "-lgridcalc_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr


def test_dropin_compiles(tmp_path):
    _compile(str(tmp_path / "dropin_test"))


@pytest.mark.gpu
def test_dropin_runs_reference_style_checks(tmp_path):
    exe = str(tmp_path / "dropin_test")
    _compile(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 13 and "FAIL" not in r.stdout, r.stdout
