"""The reference's problem set-up (what q3d does before calling the solver), for benchmarks
and examples: Z grid, geometry, properties, Mode-3 boundary conditions, heat source and the
right-hand side.

* Z grid and pitch: h2g_model_zgrid / h2g_model_pitch (src/Zcoord.jl:88-166, heat3ds.jl:197-200).
  NZ = 30*m refines each of the 30 Zcase2! cells into m equal sub-cells.
* Geometry: h2g_model_fill_id, the GPU version of fillID! (src/modelA.jl:545-556).
* setProperties! (modelA.jl:499-542), apply_boundary_conditions! (boundary_conditions.jl:94-313),
  set_BC_coef (360-394) and HeatSrc! (heat3ds.jl:55-64) are table look-ups and copies, done
  here with numpy.
* calRHS! (NonUniform.jl:57-91 with RHS.jl:23-192) runs on the GPU (h2g_calrhs), in the
  reference's operation order, so b is bit-identical to the reference's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .nonuniform import WorkBuffers

ISOTHERMAL, HEAT_FLUX, CONVECTION = L.H2G_ISOTHERMAL, L.H2G_HEAT_FLUX, L.H2G_CONVECTION
Q_SRC = 1.6e11  # common.jl:16

# material table, modelA.jl:96-122: id -> (lambda, rho, C)
MATERIALS = {
    1: (386.0, 8960.0, 383.0),   # copper (TSV)
    2: (149.0, 2330.0, 720.0),   # silicon
    3: (50.0, 8500.0, 197.0),    # solder
    4: (0.4, 1850.0, 1000.0),    # FR4
    5: (222.0, 2700.0, 921.0),   # A1060 heat sink
    6: (1.5, 2590.0, 1050.0),    # resin (underfill); also every other id
    7: (149.0, 2330.0, 720.0),   # power grid (silicon)
}


def _lib():
    lib = L.load()
    lib.h2g_model_pitch.restype = C.c_double
    lib.h2g_model_pitch.argtypes = [C.c_int]
    lib.h2g_model_zgrid.restype = C.c_int
    lib.h2g_model_zgrid.argtypes = [C.c_int] + [C.POINTER(C.c_double)] * 3
    lib.h2g_model_fill_id.restype = C.c_int
    lib.h2g_model_fill_id.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8)]
    return lib


def pitch(n: int) -> float:
    return _lib().h2g_model_pitch(int(n))


def zgrid(nz: int):
    """(Z, ZC, dZ) of genZ! with NZ+3, NZ+2, NZ+2 entries."""
    Z, ZC, dZ = np.zeros(nz + 3), np.zeros(nz + 2), np.zeros(nz + 2)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    L.check(_lib().h2g_model_zgrid(int(nz), p(Z), p(ZC), p(dZ)))
    return Z, ZC, dZ


def fill_id(NX: int, NY: int, NZ: int) -> np.ndarray:
    ID = np.zeros((NX + 2, NY + 2, NZ + 2), dtype=np.uint8, order="F")
    L.check(_lib().h2g_model_fill_id(NX, NY, NZ, ID.ctypes.data_as(C.POINTER(C.c_uint8))))
    return ID


def set_properties(wk: WorkBuffers, ID: np.ndarray):
    lam = np.full(256, MATERIALS[6][0])
    rho = np.full(256, MATERIALS[6][1])
    cp = np.full(256, MATERIALS[6][2])
    for m, (l_, r_, c_) in MATERIALS.items():
        lam[m], rho[m], cp[m] = l_, r_, c_
    wk.lam[...] = lam[ID]
    wk.rho[...] = rho[ID]
    wk.cp[...] = cp[ID]


def isothermal_bc(t):
    return (ISOTHERMAL, float(t), 0.0, 0.0, 0.0)


def heat_flux_bc(q):
    return (HEAT_FLUX, 0.0, float(q), 0.0, 0.0)


def adiabatic_bc():
    return heat_flux_bc(0.0)


def convection_bc(h, t_amb):
    return (CONVECTION, 0.0, 0.0, float(h), float(t_amb))


def mode3_bc(symmetric: bool = False):
    """set_mode3_bc_parameters (heat3ds.jl:27-46); symmetric=True: adiabatic instead of convective."""
    conv = adiabatic_bc() if symmetric else convection_bc(5.0, 300.0)
    return [conv, conv, conv, conv, isothermal_bc(300.0), conv]


def _face(a, f):
    """The guard plane of face f (x-, x+, y-, y+, z-, z+) and its interior neighbour plane."""
    ax, plus = f // 2, f % 2
    sl_g = [slice(None)] * 3
    sl_i = [slice(None)] * 3
    sl_g[ax] = -1 if plus else 0
    sl_i[ax] = -2 if plus else 1
    return tuple(sl_g), tuple(sl_i)


def apply_boundary_conditions(wk: WorkBuffers, bcs):
    for f, (typ, temp, _q, _h, amb) in enumerate(bcs):
        g, i = _face(wk.theta, f)
        wk.mask[g] = 0.0
        if typ == ISOTHERMAL:
            wk.lam[g] = wk.lam[i]
            wk.rho[g] = wk.rho[i]
            wk.cp[g] = wk.cp[i]
            wk.theta[g] = temp
        elif typ == HEAT_FLUX:
            wk.lam[g] = 0.0
        else:
            wk.lam[g] = 0.0
            wk.theta[g] = amb


def set_bc_coef(bcs) -> np.ndarray:
    return np.array([h if t == CONVECTION else 0.0 for (t, _T, _q, h, _a) in bcs])


def heat_src(wk: WorkBuffers, ID: np.ndarray):
    inner = (slice(1, -1),) * 3
    hs = wk.hsrc[inner]
    hs[ID[inner] == 7] = Q_SRC


def calRHS(wk: WorkBuffers, dx: float, dy: float, dt: float, ZC: np.ndarray, dZ: np.ndarray, HC, bcs,
           is_steady: bool):
    """calRHS! (NonUniform.jl:57-91, with apply_bc2RHS! RHS.jl:23-192) on the GPU: wk.b is
    overwritten with -(a_p0*theta + hsrc*dx*dy*dz + boundary terms), computed from b = 0."""
    from .nonuniform import Solver
    s = Solver(*wk.theta.shape)
    try:
        s.set_grid(ZC, dZ, dx, dy, dt, HC, is_steady)
        s.set_fields(wk.lam, wk.mask, None if is_steady else wk.rho, None if is_steady else wk.cp)
        s.set_theta(wk.theta)
        s.set_hsrc(wk.hsrc)
        s.calrhs(bcs, zero_b=True)
        s.get_rhs(wk.b)
    finally:
        s.close()


@dataclass
class Model:
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
    wk: WorkBuffers

    @property
    def shape(self):
        return (self.NX + 2, self.NY + 2, self.NZ + 2)


def build_mode3(NX: int, NY: int | None = None, NZ: int = 30, *, is_steady: bool = True, dt: float = 1.0e4,
                theta_init: float = 300.0, symmetric: bool = False, ID: np.ndarray | None = None,
                hsrc: np.ndarray | None = None, lam_scale: np.ndarray | None = None, calrhs: bool = True) -> Model:
    """q3d's set-up (heat3ds.jl:193-230 and main 113-128) for the Mode-3 IC stack.
    lam_scale (MZ factors, optional) multiplies the conductivity of every interior cell of plane
    k before the boundary conditions copy it into isothermal guards.  calrhs=False leaves b at
    zero, for a caller that runs calRHS! on its own solver handle (Solver.calrhs)."""
    NY = NX if NY is None else NY
    Z, ZC, dZ = zgrid(NZ)
    if ID is None:
        ID = fill_id(NX, NY, NZ)
    wk = WorkBuffers.allocate(NX + 2, NY + 2, NZ + 2)
    set_properties(wk, ID)
    if lam_scale is not None:
        wk.lam[1:-1, 1:-1, 1:-1] *= np.asarray(lam_scale, dtype=np.float64)[None, None, 1:-1]
    bcs = mode3_bc(symmetric)
    wk.theta[...] = theta_init
    apply_boundary_conditions(wk, bcs)
    HC = set_bc_coef(bcs)
    if hsrc is None:
        heat_src(wk, ID)
    else:
        wk.hsrc[...] = hsrc
    dx, dy = pitch(NX), pitch(NY)
    if calrhs:
        calRHS(wk, dx, dy, dt, ZC, dZ, HC, bcs, is_steady)
    return Model(NX, NY, NZ, dx, dy, dt, is_steady, Z, ZC, dZ, HC, bcs, ID, wk)
