"""The library driven from plain C (tests/abi_harness.c, which sees only include/h2g.h): set-up
from host arrays in the reference's layout, calRHS! with isothermal faces, PBiCGSTAB! with the
RB-GS smoother; the harness checks convergence, the mirror symmetry of the field and that the
heated block stays above its 300 K faces."""
import subprocess

import pytest

from test_abi import _build_c_caller

pytestmark = pytest.mark.gpu


def test_c_caller_solves(tmp_path):
    from h2_b200 import build
    build.build()
    exe = _build_c_caller(tmp_path)
    r = subprocess.run([exe, "solve"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("solve ok")
