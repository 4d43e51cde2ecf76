"""Observability of a solve, in the reference's file formats.

* ConvergenceData / add_residual / export_convergence_csv: src/convergence_history.jl:17-41,
  119-144 (the CSV that `q3d` writes as convergence_<solver>_<NX>x<NY>x<NZ>[_<smoother>].csv,
  heat3ds.jl:245-255).
* parse_residuals_from_log: src/parse_log_residuals.jl:14-44.  The reference fills its
  ConvergenceData by parsing log.txt, but its solvers print the residual lines to stdout only,
  so the parse finds nothing.  The GPU path hands the device-side history to
  ConvergenceData.from_history instead.
* zline_nu / export_zline_csv: plot_line_z_nu and export_zline_csv (src/plotter.jl:13-21,
  343-416): temperatures along z through the cell that contains (xc, yc), with the nodal Z
  coordinates in mm.
* step_log_line: the per-step line that main() writes to log.txt (heat3ds.jl:149-151).
"""
from __future__ import annotations

import math
import re
import time as _time
from datetime import datetime, timezone

import numpy as np

_RESIDUAL_LINE = re.compile(r"^\s+(\d+)\s+([0-9]+\.[0-9]+E[+-]\d+)")


class ConvergenceData:
    """Iteration numbers and relative residuals of one solve (ConvergenceData)."""

    def __init__(self, solver_name: str, smoother_name: str = ""):
        self.solver_name = solver_name
        self.smoother_name = smoother_name
        self.iterations: list[int] = []
        self.residuals: list[float] = []
        self.start_time = _time.time()

    def add_residual(self, iteration: int, residual: float):
        self.iterations.append(int(iteration))
        self.residuals.append(float(residual))

    @classmethod
    def from_history(cls, solver_name: str, smoother_name: str, hist, itr: int) -> "ConvergenceData":
        """Fill from the res_hist array a solve filled (entry n-1 is iteration n)."""
        d = cls(solver_name, smoother_name)
        for n in range(int(itr)):
            d.add_residual(n + 1, float(hist[n]))
        return d


def residual_line(n: int, res: float) -> str:
    """The "%10d %24.14E" line the solvers print per iteration."""
    return "%10d %24.14E" % (n, res)


def export_convergence_csv(conv: ConvergenceData, filename: str) -> bool:
    if not conv.residuals:
        print("Warning: Convergence history data is empty")
        return False
    stamp = datetime.fromtimestamp(conv.start_time, tz=timezone.utc).strftime("%Y-%m-%d %H:%M:%S")
    with open(filename, "w") as f:
        f.write("# Convergence History Data\n")
        f.write(f"# Solver: {conv.solver_name}\n")
        if conv.smoother_name:
            f.write(f"# Smoother: {conv.smoother_name}\n")
        f.write(f"# Generated: {stamp}\n")
        f.write("Iteration,Residual\n")
        for it, r in zip(conv.iterations, conv.residuals):
            f.write("%d,%.14E\n" % (it, r))
    print(f"Convergence history CSV saved: {filename}")
    return True


def convergence_filename(solver: str, NX: int, NY: int, NZ: int, smoother: str = "") -> str:
    """Stem of the CSV name that q3d uses (heat3ds.jl:246-249)."""
    name = f"convergence_{solver}_{NX}x{NY}x{NZ}"
    return name + (f"_{smoother}" if smoother else "")


def parse_residuals_from_log(conv: ConvergenceData, filename: str = "log.txt") -> bool:
    try:
        fh = open(filename)
    except FileNotFoundError:
        print(f"Warning: Log file {filename} not found")
        return False
    count = 0
    with fh:
        for line in fh:
            m = _RESIDUAL_LINE.match(line.rstrip("\n"))
            if m:
                conv.add_residual(int(m.group(1)), float(m.group(2)))
                count += 1
    if count:
        print(f"Loaded {count} residual data points from log")
        return True
    print("Warning: No residual data found in log file")
    return False


def _chk_idx(i: int, n: int) -> int:
    return 1 if i < 1 else (n if i > n else i)


def find_i(x: float, x0: float, dx: float, nx: int) -> int:
    """1-based cell index of coordinate x: floor((x - x0)/dx + 1.5), clamped to [1, nx]."""
    return _chk_idx(int(math.floor((x - x0) / dx + 1.5)), nx)


def zline_nu(theta: np.ndarray, ox, dh, Z, xc: float, yc: float):
    """(z_mm, temperatures) along z at (xc, yc), interior planes k = 2..MZ-1 (1-based), with
    z_mm = Z[k]*1000 (Z: the node coordinates, genZ!)."""
    MX, MY, MZ = theta.shape
    i = find_i(xc, ox[0], dh[0], MX)
    j = find_i(yc, ox[1], dh[1], MY)
    ks = range(2, MZ)
    z = [Z[k - 1] * 1000 for k in ks]
    s = [float(theta[i - 1, j - 1, k - 1]) for k in ks]
    return z, s


def export_zline_csv(z, d, filename: str) -> str:
    fname = f"{filename}.csv"
    with open(fname, "w") as f:
        f.write("Z [mm], Temperature [K]\n")
        for zz, v in zip(z, d):
            f.write("%f, %f\n" % (zz, v))
    print(f"Z-line CSV saved: {fname}")
    return fname


def step_log_line(step: int, t: float, theta: np.ndarray) -> str:
    """main()'s log.txt line: step, time, min/max and L2 norm of the interior theta."""
    s = theta[1:-1, 1:-1, 1:-1]
    return "%d %f : θmin=%e  θmax=%e  L2 norm of θ=%e" % (step, t, s.min(), s.max(), float(np.sqrt((s * s).sum())))
