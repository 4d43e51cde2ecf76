"""The batched workload: many steady solves of the Mode-3 IC stack with their own heat maps on
grids of uneven size, solved concurrently (h2g_batch_solve), and sharded across ranks.

Each member i is drawn from its own generator, numpy PCG64(seed0 + i):
  * NX = NY drawn uniformly from `sizes` (120, 180, 240), NZ = 30;
  * per die (the three silicon layers, modelA.jl:64-75: z in [0.10, 0.20], [0.25, 0.35],
    [0.40, 0.50] mm), K ~ U{4..16} axis-aligned hotspot rectangles: centre uniform in the die
    footprint [0.1, 1.1]^2 mm, sides U[0.05, 0.25] mm, clipped to the footprint, spanning the
    die thickness, power density exp(ln 1e8 + N(0, 1)) W/m^3;
  * heat map: every silicon cell (ID 2 or 7, modelA.jl:96-124) of a die gets the background
    1e7 W/m^3, replaced inside hotspots by the sum of the densities of the hotspots that cover
    the cell centre.
The reference has no batched solve; this is a workload over its single-solve path
(q3d's set-up, heat3ds.jl:193-230, with HeatSrc! replaced by the heat map).
"""
from __future__ import annotations

import json
import math
from dataclasses import asdict, dataclass, field

import numpy as np

SIZES = (120, 180, 240)
NZ = 30
DIE_Z = ((0.10e-3, 0.20e-3), (0.25e-3, 0.35e-3), (0.40e-3, 0.50e-3))  # zm2-zm4, zm5-zm7, zm8-zm10
FOOTPRINT = (0.1e-3, 1.1e-3)
BACKGROUND = 1.0e7
MEDIAN_DENSITY = 1.0e8
SIGMA = 1.0
SILICON_IDS = (2, 7)


@dataclass
class Hotspot:
    die: int
    x0: float
    x1: float
    y0: float
    y1: float
    q: float


@dataclass
class Member:
    index: int
    seed: int
    nx: int
    hotspots: list = field(default_factory=list)

    @property
    def cells(self) -> int:
        return self.nx * self.nx * NZ


def draw_member(i: int, seed0: int = 1000, sizes=SIZES) -> Member:
    rng = np.random.Generator(np.random.PCG64(seed0 + i))
    nx = int(sizes[int(rng.integers(len(sizes)))])
    lo, hi = FOOTPRINT
    spots = []
    for die in range(len(DIE_Z)):
        k = int(rng.integers(4, 17))
        for _ in range(k):
            cx, cy = rng.uniform(lo, hi, size=2)
            sx, sy = rng.uniform(0.05e-3, 0.25e-3, size=2)
            q = math.exp(math.log(MEDIAN_DENSITY) + SIGMA * float(rng.standard_normal()))
            spots.append(Hotspot(die, max(cx - sx / 2, lo), min(cx + sx / 2, hi), max(cy - sy / 2, lo),
                                 min(cy + sy / 2, hi), q))
    return Member(i, seed0 + i, nx, spots)


def draw_batch(n: int = 64, seed0: int = 1000, sizes=SIZES) -> list[Member]:
    return [draw_member(i, seed0, sizes) for i in range(n)]


def to_json(members: list[Member]) -> str:
    return json.dumps([asdict(m) for m in members], indent=1)


def from_json(text: str) -> list[Member]:
    return [Member(d["index"], d["seed"], d["nx"], [Hotspot(**h) for h in d["hotspots"]]) for d in json.loads(text)]


def heat_map(m: Member, ID: np.ndarray, ZC: np.ndarray, dx: float, dy: float) -> np.ndarray:
    """hsrc (MX, MY, MZ), Fortran order, guards zero.  A hotspot spans its die's thickness, so each
    die's map is summed once in (x, y), hotspot by hotspot in draw order, and copied to the die's
    planes."""
    MX, MY, MZ = ID.shape
    xc = (np.arange(MX) - 0.5) * dx  # centre of cell i (0-based; interior i = 1..NX)
    yc = (np.arange(MY) - 0.5) * dy
    hs = np.zeros((MX, MY, MZ), order="F")
    for d, (z0, z1) in enumerate(DIE_Z):
        kin = np.flatnonzero((ZC >= z0) & (ZC <= z1))
        if kin.size == 0:
            continue
        acc = np.zeros((MX, MY))
        for h in m.hotspots:
            if h.die != d:
                continue
            ix = (xc >= h.x0) & (xc < h.x1)
            iy = (yc >= h.y0) & (yc < h.y1)
            acc[np.ix_(ix, iy)] += h.q
        plane = np.where(acc > 0.0, acc, BACKGROUND)
        sub = ID[:, :, kin]
        silicon = (sub == SILICON_IDS[0]) | (sub == SILICON_IDS[1])
        hs[:, :, kin] = np.where(silicon, plane[:, :, None], 0.0)
    hs[0, :, :] = hs[-1, :, :] = 0.0
    hs[:, 0, :] = hs[:, -1, :] = 0.0
    hs[:, :, 0] = hs[:, :, -1] = 0.0
    return hs


def shard(members: list[Member], world: int) -> list[list[int]]:
    """Greedy longest-first assignment of members to ranks by cell count (no collective in the
    data path).  Returns the member indices of every rank, each list in index order."""
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for m in sorted(members, key=lambda m: (-m.cells, m.index)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(m.index)
        load[r] += m.cells
    return [sorted(x) for x in out]


def gather_results(local: dict, dist_group=None) -> dict | None:
    """Rank 0 receives every rank's {member index: result} (torch.distributed gather of Python
    objects; any backend).  Other ranks get None.  Without an initialised process group the
    local results are returned."""
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()):
        return dict(local)
    world = td.get_world_size(dist_group)
    parts = [None] * world if td.get_rank(dist_group) == 0 else None
    td.gather_object(local, parts, dst=0, group=dist_group)
    if parts is None:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return merged


# ---- GPU side ------------------------------------------------------------------------------

class BatchSolver:
    """Device handles for a list of members (one h2g handle each, fields and right-hand side
    uploaded once) and the concurrent solve of all of them (h2g_batch_solve)."""

    def __init__(self, members: list[Member], precision: str = "fp64"):
        import ctypes as C

        from . import _lib as L
        from . import model as M
        from .nonuniform import Solver
        self.L, self.C = L, C
        self.members = list(members)
        self.solvers = []
        # the members of one grid size differ only in their heat map: the model (geometry,
        # conductivities, mask, start temperature, boundary conditions) is built once per size
        models: dict[int, object] = {}
        _, ZC, _ = M.zgrid(NZ)
        for m in self.members:
            if m.nx not in models:
                models[m.nx] = M.build_mode3(m.nx, m.nx, NZ, calrhs=False)
            model = models[m.nx]
            w = model.wk
            s = Solver(*model.shape, precision=precision)
            s.set_grid(model.ZC, model.dZ, model.dx, model.dy, model.dt, model.HC, True)
            s.set_fields(w.lam, w.mask)
            s.set_theta(w.theta)
            # calRHS! on the member's own handle: b = -(hsrc V + boundary terms), from b = 0
            s.set_hsrc(heat_map(m, model.ID, ZC, model.dx, model.dy))
            s.calrhs(model.bcs, zero_b=True)
            s.snapshot()
            self.solvers.append(s)
        self._handles = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])

    @property
    def cells(self) -> int:
        return sum(m.cells for m in self.members)

    def restore(self):
        for s in self.solvers:
            s.snapshot(restore=True)

    def solve(self, method="pbicgstab", tol=1e-8, maxItr=20_000, smoother="gs", threads=2):
        """All members at once; returns (status, list of Result)."""
        from .nonuniform import smoother_selector
        L, C = self.L, self.C
        n = len(self.solvers)
        outs = (L.Result * n)()
        mth = {"pbicgstab": 0, "cg": 1, "sor": 2}[method]
        st = L.load().h2g_batch_solve(n, self._handles, mth, float(tol), int(maxItr), smoother_selector(smoother),
                                      int(threads), outs)
        L.check(st, allowed=(L.H2G_OK, L.H2G_NOT_CONVERGED, L.H2G_BREAKDOWN, L.H2G_NONFINITE))
        return st, list(outs)

    def solve_sequential(self, method="pbicgstab", tol=1e-8, maxItr=20_000, smoother="gs"):
        """The same members one after another through the single-solve calls (method "sor":
        solveSOR! with omega = 1, as h2g_batch_solve runs it)."""
        if method == "sor":
            return [s.sor(omega=1.0, tol=tol, maxItr=maxItr)[1] for s in self.solvers]
        return [s.solve(method, tol=tol, maxItr=maxItr, smoother=smoother)[1] for s in self.solvers]

    def thetas(self) -> list:
        """theta of every member, in member order."""
        return [s.get_theta() for s in self.solvers]

    def close(self):
        for s in self.solvers:
            s.close()
        self.solvers = []


class MultiBatchSolver:
    """The batch as one multi right-hand-side solve per grid size (h2g_create_multi /
    h2g_pbicgstab_multi): the members of a size share the operator, so each size group is one
    handle with K right-hand sides, and every member's result is bit for bit its lone solve's.
    b of every member is calRHS! (GPU) of its heat map on a helper handle of its size.  The groups
    are solved one after another on the given stream."""

    def __init__(self, members: list[Member], stream: int | None = None):
        from . import model as M
        from .nonuniform import MultiSolver, Solver
        from . import _lib as L
        self.L = L
        self.members = list(members)
        self.groups = []  # (member indices in self.members, MultiSolver, theta0 list)
        _, ZC, _ = M.zgrid(NZ)
        for nx in sorted({m.nx for m in self.members}):
            idx = [q for q, m in enumerate(self.members) if m.nx == nx]
            base = M.build_mode3(nx, nx, NZ, calrhs=False)
            ID, dx = base.ID, base.dx
            w = base.wk
            helper = Solver(*base.shape, stream=stream)
            bs, th0 = [], []
            try:
                helper.set_grid(base.ZC, base.dZ, base.dx, base.dy, base.dt, base.HC, True)
                helper.set_fields(w.lam, w.mask)
                for q in idx:
                    helper.set_theta(w.theta)
                    helper.set_hsrc(heat_map(self.members[q], ID, ZC, dx, dx))
                    helper.calrhs(base.bcs, zero_b=True)
                    bs.append(helper.get_rhs())
                    th0.append(w.theta.copy(order="F"))
            finally:
                helper.close()
            ms = MultiSolver(*base.shape, len(idx), stream=stream)
            ms.set_grid(base.ZC, base.dZ, base.dx, base.dy, base.dt, base.HC, True)
            ms.set_fields(w.lam, w.mask)
            ms.set_rhs_multi(bs)
            ms.set_theta_multi(th0)
            self.groups.append((idx, ms, th0))

    @property
    def cells(self) -> int:
        return sum(m.cells for m in self.members)

    def restore(self):
        for _, ms, th0 in self.groups:
            ms.set_theta_multi(th0)

    def solve(self, tol=1e-8, maxItr=20_000, smoother="gs"):
        """All members; returns (status, list of Result in member order)."""
        L = self.L
        res = [None] * len(self.members)
        status = L.H2G_OK
        for idx, ms, _ in self.groups:
            st, outs = ms.solve_multi(tol=tol, maxItr=maxItr, smoother=smoother)
            for q, r in zip(idx, outs):
                res[q] = r
            if status == L.H2G_OK and st != L.H2G_OK:
                status = st
        return status, res

    def thetas(self) -> list:
        out = [None] * len(self.members)
        for idx, ms, _ in self.groups:
            for q, th in zip(idx, ms.get_theta_multi()):
                out[q] = th
        return out

    def close(self):
        for _, ms, _ in self.groups:
            ms.close()
        self.groups = []
