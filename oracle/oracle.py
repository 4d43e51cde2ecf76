"""ctypes front end of the CPU restatement in h2_oracle.c.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.

Arrays are numpy Float64 arrays of shape (MX, MY, MZ) in Fortran (column-major)
order, i.e. exactly the memory layout of the reference's ``Array{Float64,3}``.

The model builder ``build_mode3`` restates the set-up of ``q3d`` (src/heat3ds.jl:193-230):
Z grid (Zcoord.jl:133-166), geometry + properties (modelA.jl:499-556), Mode-3 boundary
conditions (heat3ds.jl:27-46, boundary_conditions.jl:94-394), heat source
(heat3ds.jl:55-64) and the right-hand side (NonUniform.jl:57-91).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libh2oracle.so")

ISOTHERMAL, HEAT_FLUX, CONVECTION = 0, 1, 2
RED_SEQ, RED_OMP, RED_NONE = 0, 1, 2
SMOOTHER = {"none": 0, "gs": 1}


class Bc(C.Structure):
    _fields_ = [("type", C.c_int), ("temperature", C.c_double), ("heat_flux", C.c_double),
                ("htc", C.c_double), ("ambient", C.c_double)]


class Grid(C.Structure):
    _fields_ = [("MX", C.c_int), ("MY", C.c_int), ("MZ", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("dt", C.c_double), ("ZC", C.POINTER(C.c_double)), ("dZ", C.POINTER(C.c_double)),
                ("HC", C.POINTER(C.c_double)), ("is_steady", C.c_int)]


_WK_NAMES = ["theta", "b", "mask", "rho", "lam", "cp", "p", "p_", "r", "r0", "q", "s", "s_", "t_", "hsrc"]


class Wk(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in _WK_NAMES]


def build(force: bool = False) -> str:
    """Compile h2_oracle.c with the committed Makefile (gcc, -ffp-contract=off)."""
    src = os.path.join(_HERE, "h2_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.h2o_pitch.restype = C.c_double
        L.h2o_fdot1.restype = C.c_double
        L.h2o_fdot2.restype = C.c_double
        L.h2o_calcrk.restype = C.c_double
        L.h2o_rbsor_core.restype = C.c_double
        L.h2o_rbsor.restype = C.c_double
        L.h2o_res_sor.restype = C.c_double
        L.h2o_calcrk.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp, dp, C.c_int]
        L.h2o_calcax.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp]
        L.h2o_rbsor_core.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp, C.c_double, C.c_int, C.c_int]
        L.h2o_rbsor.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp, C.c_double, C.c_int]
        L.h2o_preconditioner.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp, C.c_int]
        L.h2o_fdot1.argtypes = [C.POINTER(Grid), dp, C.c_int]
        L.h2o_fdot2.argtypes = [C.POINTER(Grid), dp, dp, C.c_int]
        L.h2o_bicg1.argtypes = [C.POINTER(Grid), dp, dp, dp, C.c_double, C.c_double]
        L.h2o_triad.argtypes = [C.POINTER(Grid), dp, dp, dp, C.c_double]
        L.h2o_bicg2.argtypes = [C.POINTER(Grid), dp, dp, dp, C.c_double, C.c_double]
        L.h2o_calrhs.argtypes = [C.POINTER(Grid), C.POINTER(Bc), dp, dp, dp, dp, dp]
        solver_args = [C.POINTER(Grid), C.POINTER(Wk), C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                       C.POINTER(C.c_int), C.POINTER(C.c_double), dp]
        L.h2o_pbicgstab.argtypes = solver_args
        L.h2o_cg.argtypes = solver_args
        L.h2o_solve_sor.argtypes = [C.POINTER(Grid), C.POINTER(Wk), C.c_double, C.c_double, C.c_int, C.c_int,
                                    C.c_int, C.POINTER(C.c_double), dp]
        L.h2o_res_sor.argtypes = [C.POINTER(Grid), dp, dp, dp, dp, dp, dp, C.c_double]
        L.h2o_fill_id.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, dp,
                                  C.POINTER(C.c_uint8), C.c_int]
        L.h2o_set_properties.argtypes = [C.c_size_t, C.POINTER(C.c_uint8), dp, dp, dp]
        L.h2o_apply_bc.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(Bc), dp, dp, dp, dp, dp]
        L.h2o_set_bc_coef.argtypes = [C.POINTER(Bc), dp]
        L.h2o_heat_src.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8), dp]
        L.h2o_genz.argtypes = [C.c_int, dp, dp, dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "float64 column-major expected"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _pu8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.f_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def zeros(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


# ---------------------------------------------------------------------------------------
# Boundary-condition helpers (boundary_conditions.jl:37-83)
# ---------------------------------------------------------------------------------------
def isothermal_bc(t):
    return (ISOTHERMAL, float(t), 0.0, 0.0, 0.0)


def heat_flux_bc(q):
    return (HEAT_FLUX, 0.0, float(q), 0.0, 0.0)


def adiabatic_bc():
    return (HEAT_FLUX, 0.0, 0.0, 0.0, 0.0)


def convection_bc(h, t_amb):
    return (CONVECTION, 0.0, 0.0, float(h), float(t_amb))


def mode3_bc(symmetric: bool = False):
    """set_mode3_bc_parameters (heat3ds.jl:27-46).  symmetric=True replaces the convective
    faces by adiabatic ones (the CG "no-convection-asymmetry" variant)."""
    side = adiabatic_bc() if symmetric else convection_bc(5.0, 300.0)
    top = adiabatic_bc() if symmetric else convection_bc(5.0, 300.0)
    return [side, side, side, side, isothermal_bc(300.0), top]


def bc_array(bcs):
    arr = (Bc * 6)()
    for f, (t, temp, q, h, ta) in enumerate(bcs):
        arr[f] = Bc(t, temp, q, h, ta)
    return arr


@dataclass
class Problem:
    NX: int
    NY: int
    NZ: int
    dx: float
    dy: float
    dt: float
    is_steady: bool
    Z: np.ndarray
    ZC: np.ndarray
    dZ: np.ndarray
    HC: np.ndarray
    bcs: list
    ID: np.ndarray
    wk: dict = field(default_factory=dict)

    @property
    def shape(self):
        return (self.NX + 2, self.NY + 2, self.NZ + 2)

    def grid(self) -> Grid:
        MX, MY, MZ = self.shape
        return Grid(MX, MY, MZ, self.dx, self.dy, self.dt, _p(self.ZC), _p(self.dZ), _p(self.HC),
                    int(self.is_steady))

    def wk_struct(self) -> Wk:
        return Wk(*[_p(self.wk[n]) for n in _WK_NAMES])


def genz(nz: int):
    Z = np.zeros(nz + 3)
    ZC = np.zeros(nz + 2)
    dZ = np.zeros(nz + 2)
    if lib().h2o_genz(nz, _p(Z), _p(ZC), _p(dZ)) != 0:
        raise ValueError(f"NZ must be a positive multiple of 30, got {nz}")
    return Z, ZC, dZ


def pitch(n: int) -> float:
    return lib().h2o_pitch(n)


def fill_id(NX, NY, NZ, threads: int = 0):
    Z, _, _ = genz(NZ)
    MX, MY, MZ = NX + 2, NY + 2, NZ + 2
    ID = np.zeros((MX, MY, MZ), dtype=np.uint8, order="F")
    rc = lib().h2o_fill_id(MX, MY, MZ, pitch(NX), pitch(NY), _p(Z), _pu8(ID), threads or os.cpu_count())
    if rc != 0:
        raise RuntimeError(f"h2o_fill_id failed: {rc}")
    return ID


def build_mode3(NX: int, NY: int, NZ: int = 30, *, is_steady: bool = True, dt: float = 1.0e4,
                theta_init: float = 300.0, symmetric: bool = False, ID: np.ndarray | None = None,
                hsrc: np.ndarray | None = None, threads: int = 0, calrhs: bool = True) -> Problem:
    """Set-up of q3d (heat3ds.jl:193-230 + main 113-128): returns the WorkBuffers after
    calRHS!, ready for PBiCGSTAB!/CG!."""
    L = lib()
    MX, MY, MZ = NX + 2, NY + 2, NZ + 2
    shape = (MX, MY, MZ)
    Z, ZC, dZ = genz(NZ)
    if ID is None:
        ID = fill_id(NX, NY, NZ, threads)
    wk = {n: zeros(shape) for n in _WK_NAMES}
    wk["mask"][...] = 1.0
    wk["lam"][...] = 1.0
    wk["cp"][...] = 1.0
    L.h2o_set_properties(ID.size, _pu8(ID), _p(wk["lam"]), _p(wk["rho"]), _p(wk["cp"]))
    bcs = mode3_bc(symmetric)
    bca = bc_array(bcs)
    wk["theta"][...] = theta_init
    L.h2o_apply_bc(MX, MY, MZ, bca, _p(wk["theta"]), _p(wk["lam"]), _p(wk["rho"]), _p(wk["cp"]), _p(wk["mask"]))
    HC = np.zeros(6)
    L.h2o_set_bc_coef(bca, _p(HC))
    if hsrc is None:
        L.h2o_heat_src(MX, MY, MZ, _pu8(ID), _p(wk["hsrc"]))
    else:
        wk["hsrc"][...] = hsrc
    prob = Problem(NX, NY, NZ, pitch(NX), pitch(NY), dt, is_steady, Z, ZC, dZ, HC, bcs, ID, wk)
    if calrhs:
        calRHS(prob)
    return prob


def calRHS(prob: Problem, threads: int = 1):
    L = lib()
    L.h2o_set_threads(threads)
    g = prob.grid()
    w = prob.wk
    L.h2o_calrhs(C.byref(g), bc_array(prob.bcs), _p(w["b"]), _p(w["theta"]), _p(w["rho"]), _p(w["cp"]),
                 _p(w["hsrc"]))


def calc_ax(prob: Problem, x: np.ndarray, threads: int = 1) -> np.ndarray:
    L = lib()
    L.h2o_set_threads(threads)
    ax = zeros(prob.shape)
    w = prob.wk
    g = prob.grid()
    L.h2o_calcax(C.byref(g), _p(ax), _p(x), _p(w["lam"]), _p(w["mask"]), _p(w["rho"]), _p(w["cp"]))
    return ax


def calc_rk(prob: Problem, theta=None, b=None, red_mode=RED_SEQ, threads: int = 1):
    L = lib()
    L.h2o_set_threads(threads)
    w = prob.wk
    r = zeros(prob.shape)
    g = prob.grid()
    th = w["theta"] if theta is None else theta
    bb = w["b"] if b is None else b
    res = L.h2o_calcrk(C.byref(g), _p(r), _p(th), _p(bb), _p(w["lam"]), _p(w["mask"]), _p(w["rho"]),
                       _p(w["cp"]), red_mode)
    return r, res


def rbsor_core(prob: Problem, th: np.ndarray, b: np.ndarray, color: int, omega: float = 1.0,
               red_mode=RED_SEQ, threads: int = 1) -> float:
    L = lib()
    L.h2o_set_threads(threads)
    w = prob.wk
    g = prob.grid()
    return L.h2o_rbsor_core(C.byref(g), _p(th), _p(w["lam"]), _p(b), _p(w["mask"]), _p(w["rho"]), _p(w["cp"]),
                            omega, color, red_mode)


def preconditioner(prob: Problem, bb: np.ndarray, smoother: str = "gs", threads: int = 1) -> np.ndarray:
    L = lib()
    L.h2o_set_threads(threads)
    w = prob.wk
    g = prob.grid()
    xx = zeros(prob.shape)
    L.h2o_preconditioner(C.byref(g), _p(xx), _p(bb), _p(w["lam"]), _p(w["mask"]), _p(w["rho"]), _p(w["cp"]),
                         SMOOTHER[smoother])
    return xx


def fdot2(prob: Problem, x, y, red_mode=RED_SEQ):
    g = prob.grid()
    return lib().h2o_fdot2(C.byref(g), _p(x), _p(y), red_mode)


def _solve(fn, prob, tol, maxItr, smoother, verbose, red_mode, threads):
    g = prob.grid()
    wks = prob.wk_struct()
    itr = C.c_int(0)
    res0 = C.c_double(0.0)
    hist = np.zeros(max(maxItr, 1))
    conv = fn(C.byref(g), C.byref(wks), tol, maxItr, SMOOTHER[smoother], int(verbose), red_mode,
              threads, C.byref(itr), C.byref(res0), _p(hist))
    return bool(conv), itr.value, res0.value, hist[: itr.value].copy()


def pbicgstab(prob: Problem, tol=1e-6, maxItr=20000, smoother="gs", verbose=False, red_mode=RED_SEQ,
              threads: int = 1):
    """PBiCGSTAB! (NonUniform.jl:248-350): returns (isconverged, itr, res0, hist)."""
    return _solve(lib().h2o_pbicgstab, prob, tol, maxItr, smoother, verbose, red_mode, threads)


def cg(prob: Problem, tol=1e-6, maxItr=20000, smoother="gs", verbose=False, red_mode=RED_SEQ, threads: int = 1):
    """CG! (NonUniform.jl:115-226): returns (isconverged, itr, res0, hist)."""
    return _solve(lib().h2o_cg, prob, tol, maxItr, smoother, verbose, red_mode, threads)


def solve_sor(prob: Problem, omega=1.0, tol=1e-6, maxItr=20000, red_mode=RED_SEQ, threads: int = 1):
    """solveSOR! (NonUniform.jl:1017-1051): returns (nsweeps or -maxItr, res0, hist)."""
    g = prob.grid()
    wks = prob.wk_struct()
    res0 = C.c_double(0.0)
    hist = np.zeros(max(maxItr, 1))
    n = lib().h2o_solve_sor(C.byref(g), C.byref(wks), omega, tol, maxItr, red_mode, threads, C.byref(res0),
                            _p(hist))
    return n, res0.value, hist[: abs(n)].copy()
