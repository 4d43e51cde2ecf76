"""Output formats of the reference (convergence CSV, log parsing, z-line CSV, log.txt line),
checked against the formats written out in its sources (convergence_history.jl:119-144,
parse_log_residuals.jl:14-44, plotter.jl:13-21 and 343-416, heat3ds.jl:149-151)."""
import math
import re

import numpy as np

from h2_b200 import output as O


def test_residual_line_format():
    # "%10d %24.14E", the lines PBiCGSTAB!/CG!/solveSOR! print (README.md:176-178 shows two)
    assert O.residual_line(1, 0.658308938608891) == "         1     6.58308938608891E-01"
    assert O.residual_line(208, 9.72579214884977e-05) == "       208     9.72579214884977E-05"
    assert len(O.residual_line(12345, 1.0)) == 35


def test_convergence_csv(tmp_path):
    d = O.ConvergenceData.from_history("pbicgstab", "gs", [0.658308938608891, 0.889700596995947, 1e-9], 3)
    f = tmp_path / (O.convergence_filename("pbicgstab", 240, 240, 30, "gs") + ".csv")
    assert f.name == "convergence_pbicgstab_240x240x30_gs.csv"
    assert O.export_convergence_csv(d, str(f))
    lines = f.read_text().splitlines()
    assert lines[0] == "# Convergence History Data"
    assert lines[1] == "# Solver: pbicgstab"
    assert lines[2] == "# Smoother: gs"
    assert re.fullmatch(r"# Generated: \d{4}-\d\d-\d\d \d\d:\d\d:\d\d", lines[3])
    assert lines[4] == "Iteration,Residual"
    assert lines[5:] == ["1,6.58308938608891E-01", "2,8.89700596995947E-01", "3,1.00000000000000E-09"]
    # no smoother line when the smoother is empty; nothing written for an empty history
    d2 = O.ConvergenceData.from_history("cg", "", [0.5], 1)
    O.export_convergence_csv(d2, str(tmp_path / "c.csv"))
    assert not any(ln.startswith("# Smoother") for ln in (tmp_path / "c.csv").read_text().splitlines())
    assert not O.export_convergence_csv(O.ConvergenceData("cg"), str(tmp_path / "e.csv"))
    assert not (tmp_path / "e.csv").exists()


def test_parse_log_round_trip(tmp_path):
    hist = [0.118960680068334, 3.5e-3, 9.72579214884977e-05]
    log = tmp_path / "log.txt"
    log.write_text("Initial residual = 0.002771608776496581\n"
                   + "\n".join(O.residual_line(n + 1, r) for n, r in enumerate(hist))
                   + "\nConverged at 3\n1 10000.000000 : θmin=3.006000e+02  θmax=3.494000e+02  L2 norm of θ=1.0e+00\n")
    d = O.ConvergenceData("pbicgstab", "gs")
    assert O.parse_residuals_from_log(d, str(log))
    assert d.iterations == [1, 2, 3]
    assert d.residuals == [float("%.14E" % r) for r in hist]
    # the example line of parse_log_residuals.jl:25
    d = O.ConvergenceData("pbicgstab")
    log.write_text("         1     1.18960680068334E-01\n")
    assert O.parse_residuals_from_log(d, str(log)) and d.residuals == [0.118960680068334]
    assert not O.parse_residuals_from_log(O.ConvergenceData("x"), str(tmp_path / "missing.txt"))


def test_find_i_and_zline(tmp_path):
    # find_i: floor((x - x0)/dx + 1.5), clamped to [1, nx]
    dx = 1.2e-3 / 240
    assert O.find_i(0.6e-3, 0.0, dx, 242) == math.floor(0.6e-3 / dx + 1.5) == 121
    assert O.find_i(-1.0, 0.0, dx, 242) == 1 and O.find_i(1.0, 0.0, dx, 242) == 242
    MX, MY, MZ = 8, 6, 5
    th = np.asfortranarray(np.arange(MX * MY * MZ, dtype=float).reshape((MX, MY, MZ), order="F"))
    Z = np.linspace(0.0, 0.6e-3, MZ + 1)
    z, s = O.zline_nu(th, (0.0, 0.0, 0.0), (0.2e-3, 0.2e-3, 1.0), Z, 0.5e-3, 0.3e-3)
    i, j = O.find_i(0.5e-3, 0.0, 0.2e-3, MX), O.find_i(0.3e-3, 0.0, 0.2e-3, MY)
    assert (i, j) == (4, 3)
    assert s == [th[i - 1, j - 1, k - 1] for k in range(2, MZ)]
    assert z == [Z[k - 1] * 1000 for k in range(2, MZ)]
    name = O.export_zline_csv(z, s, str(tmp_path / "temp3Z_ctr"))
    lines = open(name).read().splitlines()
    assert lines[0] == "Z [mm], Temperature [K]"
    assert lines[1] == "%f, %f" % (z[0], s[0]) and len(lines) == MZ - 1


def test_step_log_line():
    th = np.full((4, 4, 4), 300.0, order="F")
    th[1, 1, 1] = 349.4
    line = O.step_log_line(1, 1.0e4, th)
    inner = th[1:-1, 1:-1, 1:-1]
    assert line == "1 10000.000000 : θmin=3.000000e+02  θmax=3.494000e+02  L2 norm of θ=%e" % np.sqrt(
        (inner * inner).sum())
