"""h2_b200 -- B200 (sm_100a) implementation of the Heat3ds linear-solver path.

The product is the C-ABI library libh2g.so (include/h2g.h, sources in csrc/); this package
is its Python host interface, mirroring the reference's NonUniform module.
"""
from ._lib import H2GError, H2GLibraryError, load  # noqa: F401
from .nonuniform import (CG, CalcAX, CalcRK, MultiSolver, PBiCGSTAB, Preconditioner, Solver,  # noqa: F401
                         WorkBuffers, rbsor_core, smoother_selector, solveSOR)

__all__ = ["CG", "CalcAX", "CalcRK", "MultiSolver", "PBiCGSTAB", "Preconditioner", "Solver", "WorkBuffers", "rbsor_core",
           "smoother_selector", "solveSOR", "H2GError", "H2GLibraryError", "load"]
