"""The C-ABI library without a GPU: it loads, exports every symbol include/h2g.h declares,
and rejects bad arguments on the host before any launch.  The Python host interface raises the
reference's errors (unknown smoother, unknown par) and fails loudly without the library."""
import ctypes as C
import os

import numpy as np
import pytest

import h2_b200
from h2_b200 import _lib as L


@pytest.fixture(scope="module")
def lib():
    from h2_b200 import build
    build.build()
    return L.load()


def test_exports_every_declared_symbol(lib):
    names = L.header_functions()
    assert len(names) >= 24
    raw = C.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert set(names) == set(L._SIGS), set(names) ^ set(L._SIGS)


def test_status_strings(lib):
    assert lib.h2g_status_string(L.H2G_OK) == b"ok"
    assert lib.h2g_status_string(L.H2G_BREAKDOWN) == b"breakdown"
    assert b"sm_100a" in lib.h2g_version()


def test_bad_arguments_rejected_on_host(lib):
    h = C.c_void_p()
    assert lib.h2g_create(1, 5, 5, 0, C.byref(h)) == L.H2G_BAD_ARG
    assert lib.h2g_create(5, 5, 5, 7, C.byref(h)) == L.H2G_BAD_ARG
    assert lib.h2g_create(5, 5, 5, 0, None) == L.H2G_BAD_ARG
    res = L.Result()
    assert lib.h2g_pbicgstab(None, 1e-6, 10, 1, 0, None, C.byref(res)) == L.H2G_BAD_ARG
    assert lib.h2g_cg(None, 1e-6, 10, 1, 0, None, C.byref(res)) == L.H2G_BAD_ARG
    assert b"null" in lib.h2g_last_error()
    assert lib.h2g_destroy(None) == L.H2G_OK
    # the entry points added beside the reference's path check their handle and sizes first
    J = C.c_double()
    bcs = (L.Bc * 6)()
    assert lib.h2g_sor(None, 1.5, 1e-6, 10, 0, None, C.byref(res)) == L.H2G_BAD_ARG
    assert lib.h2g_calrhs(None, bcs, 1) == L.H2G_BAD_ARG
    assert lib.h2g_transient(None, bcs, 3, 0, 1e-6, 10, 1, 0, None, C.byref(res)) == L.H2G_BAD_ARG
    assert lib.h2g_adjoint(None, None, 8.0, 1e-6, 10, 1, C.byref(J), None, None, None, None) == L.H2G_BAD_ARG
    assert lib.h2g_adjoint_transient(None, bcs, 3, None, 8.0, 1e-6, 10, 1, 2, C.byref(J), None, None,
                                     None) == L.H2G_BAD_ARG
    assert lib.h2g_autotune(None, None, None, None, None) == L.H2G_BAD_ARG
    assert lib.h2g_set_tuning(None, 4, 2) == L.H2G_BAD_ARG
    hs = (C.c_void_p * 1)()
    assert lib.h2g_batch_solve(0, hs, 0, 1e-6, 10, 1, 1, (L.Result * 1)()) == L.H2G_BAD_ARG
    assert lib.h2g_batch_solve(1, hs, 0, 1e-6, 10, 1, 1, (L.Result * 1)()) == L.H2G_BAD_ARG  # null handle
    assert lib.h2g_batch_solve(1, hs, 7, 1e-6, 10, 1, 1, (L.Result * 1)()) == L.H2G_BAD_ARG
    assert lib.h2g_calcrk_noalloc(2, 5, 5, None, None, None, None, None, None, None, None, 1.0, 1.0, 1.0, None, 1,
                                  None, None, None) == L.H2G_BAD_ARG


def test_smoother_selector_errors():
    assert h2_b200.smoother_selector("gs") == L.H2G_SMOOTHER_GS
    assert h2_b200.smoother_selector(":none") == L.H2G_SMOOTHER_NONE
    with pytest.raises(ValueError, match="Unsupported smoother"):
        h2_b200.smoother_selector("jacobi")


def test_par_must_be_gpu():
    wk = h2_b200.WorkBuffers.allocate(6, 6, 6)
    with pytest.raises(ValueError, match="parallel mode"):
        h2_b200.PBiCGSTAB(wk, (1e-5, 1e-5, 1.0), 1.0, np.zeros(6), np.zeros(6), np.zeros(6), par="thread")


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(h2_b200.H2GLibraryError):
        L.load(str(tmp_path / "libh2g.so"))


def test_workbuffers_layout():
    wk = h2_b200.WorkBuffers.allocate(7, 6, 5)
    assert wk.theta.flags.f_contiguous and wk.theta.shape == (7, 6, 5)
    assert wk.mask.min() == 1.0 and wk.lam.min() == 1.0 and wk.cp.min() == 1.0 and wk.rho.max() == 0.0


def test_header_is_plain_c():
    """include/h2g.h is a C header (plain pointers and sizes, no C++ or torch types): it compiles
    as C99, so cgo, ccall, JNI or ctypes bindings can use it as it is."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    hdr = os.path.join(os.path.dirname(L.LIB_PATH), "..", "include", "h2g.h")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", hdr], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr


def _build_c_caller(tmp_path):
    """Compiles tests/abi_harness.c, a plain-C caller that sees only include/h2g.h, and links it
    against the in-tree libh2g.so the way a foreign-language binding loads it."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(L.LIB_PATH)
    exe = str(tmp_path / "abi_harness")
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-O1", "-I", os.path.join(root, "include"),
                        os.path.join(root, "tests", "abi_harness.c"), "-L", libdir, "-lh2g",
                        "-Wl,-rpath," + libdir, "-lm", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_host_checks(lib, tmp_path):
    import subprocess
    exe = _build_c_caller(tmp_path)
    r = subprocess.run([exe, "host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("host checks ok")


def test_history_buffer_checked_on_host(lib):
    """The library writes up to maxItr residuals into the caller's history buffer: a shorter or
    non-Float64 buffer is refused before any call reaches the device."""
    wk = h2_b200.WorkBuffers.allocate(6, 6, 6)
    z6, hc = np.linspace(0.0, 1e-3, 6), np.zeros(6)
    for bad, err in ((np.zeros(9), ValueError), (np.zeros(10, dtype=np.float32), TypeError)):
        with pytest.raises(err):
            h2_b200.PBiCGSTAB(wk, (1e-5, 1e-5, 1.0), 1.0, z6, np.full(6, 2e-4), hc, maxItr=10, hist=bad)
        with pytest.raises(err):
            h2_b200.solveSOR(wk.theta, wk.lam, wk.b, wk.mask, wk.rho, wk.cp, (1e-5, 1e-5, 1.0), 1.0, 1.5, z6,
                             np.full(6, 2e-4), hc, None, 1e-6, maxItr=10, hist=bad)
