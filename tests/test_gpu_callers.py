"""The reference's own C callers against this library (the drop-in boundary, tested from C rather than through ctypes).

oracle/Makefile (target `callers`, run by __graft_entry__.build() where the reference sources exist) compiles FPLUS's
examples/solve.c unchanged, and its tests/c/test_fplus.c with the partial-pivoting cases selected (oracle/ref_callers.c),
against include/fplus.h, linked with fplus_b200/libfplus.so.  The binaries travel with the repository under
oracle/_ref/callers/.  A layout change of fplus_options or fplus_factors, a missing symbol or a different error code
shows up here as a compile, link or check failure.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

CALLERS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "callers")


def _run(name):
    path = os.path.join(CALLERS, name)
    if not os.path.exists(path):
        pytest.skip(f"{path} was not built (the reference sources were absent at build time)")
    return subprocess.run([path], capture_output=True, text=True, timeout=300)


def test_reference_example_solve():
    """examples/solve.c: a 3 x 3 complex system and its conjugate transpose both solve to (1, 1, 1)."""
    r = _run("example_solve")
    assert r.returncode == 0, r.stdout + r.stderr
    import re
    lines = [l for l in r.stdout.splitlines() if "=" in l]
    assert len(lines) == 2, r.stdout
    for l in lines:
        # the example prints each component as re+imi with three decimals (a rounding-level negative imaginary part
        # prints as -0.000)
        parts = re.findall(r"([+-]?\d+\.\d+)([+-]\d+\.\d+)i", l.split("=")[-1])
        assert len(parts) == 3, l
        for re_, im_ in parts:
            assert abs(float(re_) - 1.0) < 1e-3 and abs(float(im_)) < 1e-3, l


def test_reference_c_test_partial_pivoting():
    """tests/c/test_fplus.c, partial pivoting: analyze / factor / solve round trips with dense lines and 12-decade row
    scaling (backward error < 1e-12 in every direction), the Ruiz range guard, and the input validation codes."""
    r = _run("test_fplus_pp")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
    assert "passed" in r.stdout
