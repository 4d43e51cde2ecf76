"""Python mirror of the reference's solver interface, running on the B200 library.

The functions keep the names, argument meaning and error behaviour of the Julia module
NonUniform (src/NonUniform.jl) and of WorkBuffers (src/common.jl:49-89); only
``par="gpu"`` exists here, and it runs the sm_100a kernels of libh2g.so through the C ABI.

Arrays are numpy float64 arrays of shape (MX, MY, MZ) = (NX+2, NY+2, NZ+2) in Fortran order,
the memory layout of the reference's Array{Float64,3}.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

_SMOOTHERS = {"none": L.H2G_SMOOTHER_NONE, "gs": L.H2G_SMOOTHER_GS}
_PRECISION = {"fp64": L.H2G_FP64, "mixed": L.H2G_MIXED, "mixed_ir": L.H2G_MIXED_IR}


def bc_array(bcs):
    """Six boundary conditions (type, temperature, heat_flux, htc, ambient), faces x-, x+, y-,
    y+, z-, z+ (BoundaryConditionSet, boundary_conditions.jl:24-31), as an h2g_bc[6]."""
    if len(bcs) != 6:
        raise ValueError("need 6 boundary conditions (x-, x+, y-, y+, z-, z+)")
    arr = (L.Bc * 6)()
    for f, (typ, temp, q, h, amb) in enumerate(bcs):
        arr[f] = L.Bc(int(typ), float(temp), float(q), float(h), float(amb))
    return arr


def _f64(a: np.ndarray, name: str) -> np.ndarray:
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.ndim != 3 or not a.flags.f_contiguous:
        raise TypeError(f"{name}: expected a Float64 3-D array in column-major (Fortran) order")
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _hist(hist, maxItr):
    """The residual-history buffer: the library writes up to maxItr doubles into it."""
    if hist is None:
        return None
    if not isinstance(hist, np.ndarray) or hist.dtype != np.float64 or not hist.flags.c_contiguous:
        raise TypeError("hist: expected a contiguous Float64 array")
    if hist.size < int(maxItr):
        raise ValueError(f"hist holds {hist.size} values; the solve may write maxItr = {int(maxItr)}")
    return _ptr(hist)


def smoother_selector(s) -> int:
    """smoother_selector (NonUniform.jl:36-41): :none / :gs, anything else is an ArgumentError."""
    key = s.lstrip(":") if isinstance(s, str) else s
    if key not in _SMOOTHERS:
        raise ValueError(f"Unsupported smoother: {s}. Use :none or :gs")
    return _SMOOTHERS[key]


def _check_par(par: str):
    if par != "gpu":
        raise ValueError(f"Invalid parallel mode {par!r}: this library implements par=\"gpu\" only")


@dataclass
class WorkBuffers:
    """WorkBuffers (common.jl:49-89): the 15 Float64 arrays of one grid."""
    theta: np.ndarray
    b: np.ndarray
    mask: np.ndarray
    rho: np.ndarray
    lam: np.ndarray
    cp: np.ndarray
    pcg_p: np.ndarray
    pcg_p_: np.ndarray
    pcg_r: np.ndarray
    pcg_r0: np.ndarray
    pcg_q: np.ndarray
    pcg_s: np.ndarray
    pcg_s_: np.ndarray
    pcg_t_: np.ndarray
    hsrc: np.ndarray

    @classmethod
    def allocate(cls, mx: int, my: int, mz: int) -> "WorkBuffers":
        z = lambda: np.zeros((mx, my, mz), order="F")  # noqa: E731
        o = lambda: np.ones((mx, my, mz), order="F")  # noqa: E731
        return cls(z(), z(), o(), z(), o(), o(), z(), z(), z(), z(), z(), z(), z(), z(), z())

    @property
    def shape(self):
        return self.theta.shape


class Solver:
    """A device-resident solver handle (h2g_create ... h2g_destroy) for one grid size."""

    def __init__(self, MX: int, MY: int, MZ: int, precision: str = "fp64", stream: int | None = None):
        self.lib = L.load()
        if precision not in _PRECISION:
            raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
        h = C.c_void_p()
        L.check(self.lib.h2g_create(MX, MY, MZ, _PRECISION[precision], C.byref(h)))
        self.h = h
        self.shape = (MX, MY, MZ)
        self.precision = precision
        if stream is not None:
            L.check(self.lib.h2g_set_stream(self.h, C.c_void_p(stream)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.h2g_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, a, name):
        a = _f64(a, name)
        if a.shape != self.shape:
            raise ValueError(f"{name}: shape {a.shape} != {self.shape}")
        return a

    def set_grid(self, ZC, dZ, dx, dy, dt, HC, is_steady: bool):
        ZC = np.ascontiguousarray(ZC, dtype=np.float64)
        dZ = np.ascontiguousarray(dZ, dtype=np.float64)
        HC = np.ascontiguousarray(HC, dtype=np.float64)
        if ZC.size != self.shape[2] or dZ.size < self.shape[2] - 1 or HC.size != 6:
            raise ValueError("ZC needs MZ entries, dZ at least MZ-1, HC 6")
        if dZ.size == self.shape[2] - 1:
            dZ = np.append(dZ, dZ[-1])
        L.check(self.lib.h2g_set_grid(self.h, _ptr(ZC), _ptr(dZ), float(dx), float(dy), float(dt), _ptr(HC),
                                      int(bool(is_steady))))

    def set_fields(self, lam, mask, rho=None, cp=None):
        lam = self._arr(lam, "lambda")
        mask = self._arr(mask, "mask")
        if rho is not None:
            rho = self._arr(rho, "rho")
            cp = self._arr(cp, "cp")
        L.check(self.lib.h2g_set_fields(self.h, _ptr(lam), _ptr(mask), _ptr(rho), _ptr(cp)))

    def set_rhs(self, b):
        L.check(self.lib.h2g_set_rhs(self.h, _ptr(self._arr(b, "b"))))

    def set_theta(self, theta):
        L.check(self.lib.h2g_set_theta(self.h, _ptr(self._arr(theta, "theta"))))

    def get_theta(self, out=None):
        out = np.zeros(self.shape, order="F") if out is None else self._arr(out, "theta")
        L.check(self.lib.h2g_get_theta(self.h, _ptr(out)))
        return out

    def snapshot(self, restore: bool = False):
        L.check(self.lib.h2g_theta_snapshot(self.h, 1 if restore else 0))

    def set_mixed_params(self, inner_tol: float, max_outer: int = 40):
        L.check(self.lib.h2g_set_mixed_params(self.h, float(inner_tol), int(max_outer)))

    def solve(self, method="pbicgstab", tol=1e-6, maxItr=20_000, smoother="gs", verbose=False, hist=None):
        """Returns (status, Result); the status is also Result.status.  method: "pbicgstab" or
        "cg" (solveSOR! is Solver.sor)."""
        if method not in ("pbicgstab", "cg"):
            raise ValueError(f"unknown method {method!r}: use 'pbicgstab' or 'cg' (or Solver.sor)")
        sm = smoother_selector(smoother)
        res = L.Result()
        fn = self.lib.h2g_pbicgstab if method == "pbicgstab" else self.lib.h2g_cg
        st = fn(self.h, float(tol), int(maxItr), sm, int(bool(verbose)), _hist(hist, maxItr), C.byref(res))
        L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_BREAKDOWN, L.H2G_NONFINITE))
        return st, res

    def get_rhs(self, out=None):
        out = np.zeros(self.shape, order="F") if out is None else self._arr(out, "b")
        L.check(self.lib.h2g_get_rhs(self.h, _ptr(out)))
        return out

    def set_hsrc(self, hsrc):
        L.check(self.lib.h2g_set_hsrc(self.h, _ptr(self._arr(hsrc, "hsrc"))))

    def calrhs(self, bcs, zero_b: bool = True):
        """calRHS! on the device (b of the handle; zero_b=False accumulates like the reference)."""
        L.check(self.lib.h2g_calrhs(self.h, bc_array(bcs), int(bool(zero_b))))

    def transient(self, bcs, nt: int, method="pbicgstab", tol=1e-6, maxItr=20_000, smoother="gs", verbose=False):
        """nt steps of main()'s loop on the device.  Returns (status, Result, stats) with stats
        an (nt, 5) array: theta min, max, L2 norm, iterations, final relative residual."""
        sm = smoother_selector(smoother)
        stats = np.zeros((int(nt), 5))
        res = L.Result()
        st = self.lib.h2g_transient(self.h, bc_array(bcs), int(nt), 0 if method == "pbicgstab" else 1, float(tol),
                                    int(maxItr), sm, int(bool(verbose)), _ptr(stats), C.byref(res))
        L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_BREAKDOWN, L.H2G_NONFINITE))
        return st, res, stats[: res.outer]

    def sor(self, omega=1.0, tol=1e-6, maxItr=20_000, verbose=False, hist=None):
        """solveSOR! on the handle's theta and b (FP64).  Returns (status, Result)."""
        res = L.Result()
        st = self.lib.h2g_sor(self.h, float(omega), float(tol), int(maxItr), int(bool(verbose)), _hist(hist, maxItr),
                              C.byref(res))
        L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_NONFINITE))
        return st, res

    # single kernels (host arrays in and out)
    def calc_ax(self, x):
        ax = np.zeros(self.shape, order="F")
        L.check(self.lib.h2g_calcax(self.h, _ptr(self._arr(x, "x")), _ptr(ax)))
        return ax

    def calc_rk(self):
        r = np.zeros(self.shape, order="F")
        res = C.c_double()
        L.check(self.lib.h2g_calcrk(self.h, _ptr(r), C.byref(res)))
        return r, res.value

    def rbsor_pass(self, x, b, color, omega=1.0):
        x = self._arr(x, "x")
        L.check(self.lib.h2g_rbsor_pass(self.h, _ptr(x), _ptr(self._arr(b, "b")), int(color), float(omega)))
        return x

    def preconditioner(self, bb, smoother="gs"):
        xx = np.zeros(self.shape, order="F")
        L.check(self.lib.h2g_preconditioner(self.h, _ptr(self._arr(bb, "bb")), _ptr(xx), smoother_selector(smoother)))
        return xx

    def autotune(self) -> tuple:
        """Run the launch-shape tuner now; returns the colour pass's (rows per block, planes per
        thread)."""
        return self.tuning()[:2]

    def tuning(self) -> tuple:
        """The tuner's choices (running it if needed): (rows, planes, coefficient source of the
        colour pass, of CalcAX) with the sources 0 (dd summed per cell), 1 (dd read from the
        per-cell array), 2 (stencil-class table, FP64)."""
        r, p, a, b = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        L.check(self.lib.h2g_autotune(self.h, C.byref(r), C.byref(p), C.byref(a), C.byref(b)))
        return r.value, p.value, a.value, b.value

    def set_tuning(self, rows: int, planes: int = 2):
        """Force the colour pass's shape (rows 2, 4, 8, 16; planes 1, 2); rows = 0 tunes again."""
        L.check(self.lib.h2g_set_tuning(self.h, int(rows), int(planes)))

    def set_sweep(self, fused: int, chunks: int = 1, dd_array: bool = False):
        """Force the preconditioner's sweeps 2-5: fused=1 one fused launch per sweep (with `chunks`
        z chunks and dd read or summed), 0 two colour passes per sweep, -1 let the tuner choose."""
        L.check(self.lib.h2g_set_sweep(self.h, int(fused), int(chunks), int(bool(dd_array))))

    def sweep(self) -> tuple:
        """(fused, chunks, dd read) that the next solve uses (running the tuner if needed)."""
        f, c, d = C.c_int(0), C.c_int(0), C.c_int(0)
        L.check(self.lib.h2g_get_sweep(self.h, C.byref(f), C.byref(c), C.byref(d)))
        return bool(f.value), c.value, bool(d.value)

    def set_coop(self, mode: int):
        """The PBiCGSTAB preconditioner as one cooperative launch: 1 on, 0 off, -1 default."""
        L.check(self.lib.h2g_set_coop(self.h, int(mode)))

    def coop(self) -> bool:
        """Whether the next solve runs the cooperative preconditioner."""
        on = C.c_int(0)
        L.check(self.lib.h2g_get_coop(self.h, C.byref(on)))
        return bool(on.value)

    def set_wait_limit(self, cycles: int):
        """Budget of one bounded device wait in clock cycles (0: every wait gives up at once)."""
        L.check(self.lib.h2g_set_wait_limit(self.h, int(cycles)))

    def bench_kernel(self, kind: int, reps: int) -> int:
        n = C.c_int()
        L.check(self.lib.h2g_bench_kernel(self.h, int(kind), int(reps), C.byref(n)))
        return n.value


class MultiSolver(Solver):
    """One operator, K right-hand sides (h2g_create_multi): the members of a batch that share a grid
    size.  Grid and fields as for Solver; b and theta per right-hand side; one solve runs all K
    PBiCGSTAB! iterations together, each with its lone solve's bits."""

    def __init__(self, MX: int, MY: int, MZ: int, nrhs: int, stream: int | None = None):
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.h2g_create_multi(MX, MY, MZ, int(nrhs), C.byref(h)))
        self.h = h
        self.shape = (MX, MY, MZ)
        self.precision = "fp64"
        self.nrhs = int(nrhs)
        if stream is not None:
            L.check(self.lib.h2g_set_stream(self.h, C.c_void_p(stream)))

    def _stack(self, arrays, name):
        if len(arrays) != self.nrhs:
            raise ValueError(f"{name}: {len(arrays)} arrays for {self.nrhs} right-hand sides")
        out = np.empty(self.shape + (self.nrhs,), order="F")
        for q, a in enumerate(arrays):
            out[..., q] = self._arr(a, name)
        return out

    def set_rhs_multi(self, bs):
        L.check(self.lib.h2g_set_rhs_multi(self.h, _ptr(self._stack(bs, "b"))))

    def set_theta_multi(self, thetas):
        L.check(self.lib.h2g_set_theta_multi(self.h, _ptr(self._stack(thetas, "theta"))))

    def get_theta_multi(self) -> list:
        out = np.empty(self.shape + (self.nrhs,), order="F")
        L.check(self.lib.h2g_get_theta_multi(self.h, _ptr(out)))
        return [np.asfortranarray(out[..., q]) for q in range(self.nrhs)]

    def solve_multi(self, tol=1e-6, maxItr=20_000, smoother="gs"):
        outs = (L.Result * self.nrhs)()
        st = self.lib.h2g_pbicgstab_multi(self.h, float(tol), int(maxItr), smoother_selector(smoother), outs)
        L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_BREAKDOWN, L.H2G_NONFINITE))
        return st, list(outs)


def _dh(dh):
    if len(dh) < 2:
        raise ValueError("Δh must hold (dx, dy[, dz])")
    return float(dh[0]), float(dh[1])


def _oneshot(method, wk, dh, dt, ZC, dZ, HC, tol, maxItr, smoother, par, verbose, is_steady, precision, hist):
    _check_par(par)
    sm = smoother_selector(smoother)
    if precision not in _PRECISION:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}")
    lib = L.load()
    MX, MY, MZ = wk.theta.shape
    for n in ("theta", "b", "lam", "mask", "rho", "cp"):
        a = _f64(getattr(wk, n), n)
        if a.shape != (MX, MY, MZ):
            raise ValueError(f"{n}: shape {a.shape} != {(MX, MY, MZ)}")
    dx, dy = _dh(dh)
    ZC = np.ascontiguousarray(ZC, dtype=np.float64)
    dZ = np.ascontiguousarray(dZ, dtype=np.float64)
    if dZ.size == MZ - 1:
        dZ = np.append(dZ, dZ[-1])
    HC = np.ascontiguousarray(HC, dtype=np.float64)
    if ZC.size != MZ or dZ.size != MZ or HC.size != 6:
        raise ValueError("ZC needs MZ entries, dZ MZ (or MZ-1), HC 6")
    hp = _hist(hist, maxItr)
    res = L.Result()
    fn = lib.h2g_PBiCGSTAB if method == "pbicgstab" else lib.h2g_CG
    st = fn(MX, MY, MZ, _ptr(wk.theta), _ptr(wk.b), _ptr(wk.lam), _ptr(wk.mask), _ptr(wk.rho), _ptr(wk.cp), dx, dy,
            float(dt), _ptr(ZC), _ptr(dZ), _ptr(HC), float(tol), int(maxItr), sm, int(bool(verbose)),
            int(bool(is_steady)), _PRECISION[precision], hp, C.byref(res))
    L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_BREAKDOWN, L.H2G_NONFINITE))
    return bool(res.isconverged), int(res.itr), float(res.res0)


def PBiCGSTAB(wk: WorkBuffers, dh, dt, ZC, dZ, HC, *, tol=1e-6, maxItr=20_000, smoother="none", par="gpu",
              verbose=False, is_steady=False, precision="fp64", hist=None):
    """PBiCGSTAB! (NonUniform.jl:248-350).  Updates wk.theta in place and returns
    (isconverged, itr, res0)."""
    return _oneshot("pbicgstab", wk, dh, dt, ZC, dZ, HC, tol, maxItr, smoother, par, verbose, is_steady, precision,
                    hist)


def CG(wk: WorkBuffers, dh, dt, ZC, dZ, HC, *, tol=1e-6, maxItr=20_000, smoother="none", par="gpu", verbose=False,
       is_steady=False, precision="fp64", hist=None):
    """CG! (NonUniform.jl:115-226).  Updates wk.theta in place and returns (isconverged, itr, res0)."""
    return _oneshot("cg", wk, dh, dt, ZC, dZ, HC, tol, maxItr, smoother, par, verbose, is_steady, precision, hist)


def solveSOR(theta, lam, b, mask, rho, cp, dh, dt, omega, ZC, dZ, HC, F=None, tol=1e-6, par="gpu", *,
             maxItr=20_000, is_steady=False, verbose=True, hist=None):
    """solveSOR! (NonUniform.jl:1004-1051): RB-SOR with relaxation omega until
    sqrt(sum r^2)/res0 < tol; theta is updated in place.  The reference prints
    "Initial residual", one "%10d %24.14E" line per pass and "Converged at n" to F and stdout;
    with verbose the library prints them to stdout and, when F is a writable text stream, the
    per-pass lines are written to F as well.  Returns (isconverged, itr, res0)."""
    _check_par(par)
    lib = L.load()
    MX, MY, MZ = theta.shape
    for n, a in (("theta", theta), ("lambda", lam), ("b", b), ("mask", mask), ("rho", rho), ("cp", cp)):
        a = _f64(a, n)
        if a.shape != (MX, MY, MZ):
            raise ValueError(f"{n}: shape {a.shape} != {(MX, MY, MZ)}")
    dx, dy = _dh(dh)
    ZC = np.ascontiguousarray(ZC, dtype=np.float64)
    dZ = np.ascontiguousarray(dZ, dtype=np.float64)
    if dZ.size == MZ - 1:
        dZ = np.append(dZ, dZ[-1])
    HC = np.ascontiguousarray(HC, dtype=np.float64)
    if ZC.size != MZ or dZ.size != MZ or HC.size != 6:
        raise ValueError("ZC needs MZ entries, dZ MZ (or MZ-1), HC 6")
    if F is not None and hist is None:
        hist = np.zeros(int(maxItr))
    res = L.Result()
    st = lib.h2g_SolveSOR(MX, MY, MZ, _ptr(theta), _ptr(b), _ptr(lam), _ptr(mask), _ptr(rho), _ptr(cp), dx, dy,
                          float(dt), float(omega), _ptr(ZC), _ptr(dZ), _ptr(HC), float(tol), int(maxItr),
                          int(bool(verbose)), int(bool(is_steady)), _hist(hist, maxItr), C.byref(res))
    L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_NONFINITE))
    if F is not None:
        for n in range(int(res.itr)):
            F.write("%10d %24.14E\n" % (n + 1, hist[n]))
    return bool(res.isconverged), int(res.itr), float(res.res0)


def _kernel_solver(shape, dh, dt, ZC, dZ, HC, lam, m, rho, cp, is_steady, par):
    _check_par(par)
    s = Solver(*shape)
    dx, dy = _dh(dh)
    s.set_grid(ZC, dZ, dx, dy, dt, HC, is_steady)
    s.set_fields(lam, m, None if is_steady else rho, None if is_steady else cp)
    return s


def CalcAX(ax, theta, dh, dt, lam, m, rho, cp, ZC, dZ, HC, par="gpu", *, is_steady=False):
    """CalcAX! (NonUniform.jl:454-511): ax[interior] = A theta."""
    s = _kernel_solver(theta.shape, dh, dt, ZC, dZ, HC, lam, m, rho, cp, is_steady, par)
    try:
        out = s.calc_ax(theta)
        ax[1:-1, 1:-1, 1:-1] = out[1:-1, 1:-1, 1:-1]
    finally:
        s.close()


def CalcRK(r, theta, b, lam, m, rho, cp, dh, dt, ZC, dZ, HC, par="gpu", *, is_steady=False):
    """CalcRK! (NonUniform.jl:372-434): r[interior] = b - A theta; returns ||r||_2."""
    s = _kernel_solver(theta.shape, dh, dt, ZC, dZ, HC, lam, m, rho, cp, is_steady, par)
    try:
        s.set_theta(theta)
        s.set_rhs(b)
        out, res = s.calc_rk()
        r[1:-1, 1:-1, 1:-1] = out[1:-1, 1:-1, 1:-1]
        return res
    finally:
        s.close()


def Preconditioner(xx, bb, lam, mask, rho, cp, dh, dt, smoother, ZC, dZ, HC, par="gpu", *, is_steady=False):
    """Preconditioner! (NonUniform.jl:531-559): xx = M^-1 bb with xx starting from zero."""
    sm = "gs" if smoother_selector(smoother) == L.H2G_SMOOTHER_GS else "none"
    s = _kernel_solver(bb.shape, dh, dt, ZC, dZ, HC, lam, mask, rho, cp, is_steady, par)
    try:
        xx[...] = s.preconditioner(bb, sm)
    finally:
        s.close()


def rbsor_core(theta, lam, b, m, rho, cp, dh, dt, omega, ZC, dZ, HC, color, par="gpu", *, is_steady=False):
    """rbsor_core! (NonUniform.jl:848-915): one colour pass, theta updated in place."""
    s = _kernel_solver(theta.shape, dh, dt, ZC, dZ, HC, lam, m, rho, cp, is_steady, par)
    try:
        s.rbsor_pass(theta, b, color, omega)
    finally:
        s.close()
