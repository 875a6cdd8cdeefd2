"""The C-ABI library loads on a machine without a GPU and exports every entry
point that include/gridcalc_b200.h declares; a plain C program uses the
entry points that need no device (no compute calls here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gridcalc_b200.h")
LIB = os.path.join(ROOT, "grid-calculus_b200", "lib", "libgridcalc_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"GC_API\s+[\w\s\*]+?\b(gc_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "gc_laplacian" in syms and "gc_ch_integrate" in syms and "gc_integrate" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_status_strings_without_gpu():
    lib = ctypes.CDLL(LIB)
    lib.gc_version.restype = ctypes.c_char_p
    lib.gc_status_string.restype = ctypes.c_char_p
    assert lib.gc_version().decode().startswith("0.15.1")
    assert lib.gc_status_string(2) == b"GC_ERR_AXIS_EXTENT"


def test_python_mirror_imports():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "grid-calculus_b200"))
    import gridcalc_b200 as gc
    g = gc.Grid(4, 5, 6, 0.5, 1.0, 2.0)
    assert g.shape == (6, 5, 4) and g.size == 120 and g.cell_volume == 1.0
    try:
        gc.Grid(0, 1, 1)
    except ValueError as e:
        assert "extents" in str(e)
    else:
        raise AssertionError("Grid(0, 1, 1) accepted")


def test_python_mirror_constants_match_the_header():
    """The Python mirror's enum-like constants are the header's values."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "grid-calculus_b200"))
    import gridcalc_b200 as gc
    text = open(HEADER).read()
    assert int(re.search(r"#define GC_BATCH_FUSED (\d+)", text).group(1)) == gc.ChBatch.FUSED
    opts = dict(re.findall(r"(GC_OPT_\w+) = (\d+)", text))
    assert int(opts["GC_OPT_CLUSTER_STEPPING"]) == gc.OPT_CLUSTER_STEPPING
    assert int(opts["GC_OPT_FUSED_STEP"]) == gc.OPT_FUSED_STEP


def test_c_program_uses_the_abi_without_gpu(tmp_path):
    """tests/c/abi_c_test.c: the header compiles as strict C99 and a C
    program linked against the library runs the device-free entry points."""
    import subprocess
    libdir = os.path.dirname(LIB)
    exe = str(tmp_path / "abi_c_test")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", os.path.join(ROOT, "tests", "c", "abi_c_test.c"),
           "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lgridcalc_b200", f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "FAIL" not in r.stdout, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 9, r.stdout
