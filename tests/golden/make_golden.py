"""Generate the golden fixtures of tests/golden/.

  python tests/golden/make_golden.py [--reference <checkout of kenoogl/H2>] [--only readme|oracle240|...]

(--reference is needed for the readme job only)

readme_240.json      the sample log of the reference README (README.md:166-183), read as text:
                     the initial residual, the relative residuals printed there, the iteration
                     of convergence and theta min/max.  Pins the oracle.
oracle_240_1e-4.json the oracle (bit-exact sequential reductions) for the README's case
                     q3d(240,240,30,"pbicgstab","gs"; epsilon=1e-4, is_steady=true): iteration
                     count, the residual history, theta statistics and theta at 4096 seeded cells.
oracle_240_1e-8.json the oracle at epsilon = 1e-8 (OpenMP reductions), same content: the FP64
                     reference for the GPU FP64 and mixed-precision solves.
oracle_240_cg_sym.json  CG + GS on the symmetric variant (convective faces replaced by adiabatic
                     ones) at epsilon = 1e-8.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SAMPLE_SEED = 20240601
NSAMPLE = 4096


def parse_readme(path: str) -> dict:
    text = open(path, encoding="utf-8").read()
    m = re.search(r"Initial residual = ([0-9.eE+-]+)", text)
    lines = re.findall(r"^\s+(\d+)\s+([0-9.]+E[+-]\d+)\s*$", text, flags=re.M)
    conv = re.search(r"Converged at (\d+)", text)
    th = re.search(r"θmin=([0-9.]+)K\s+θmax=([0-9.]+)K", text)
    eps = re.search(r"ε\s*:\s*([0-9.eE+-]+)", text)
    grid = re.search(r"Grid\s*:\s*(\d+) (\d+) (\d+)", text)
    return {
        "source": "README.md:166-183 (sample log of q3d(240,240,30,'pbicgstab','gs'; epsilon=1e-4, steady))",
        "grid": [int(g) for g in grid.groups()],
        "epsilon": float(eps.group(1)),
        "res0_repr": m.group(1),
        "residual_lines": [[int(a), b] for a, b in lines],
        "converged_at": int(conv.group(1)),
        "theta_min_K": float(th.group(1)),
        "theta_max_K": float(th.group(2)),
    }


def sample_cells(shape, n=NSAMPLE, seed=SAMPLE_SEED):
    rng = np.random.default_rng(seed)
    MX, MY, MZ = shape
    i = rng.integers(1, MX - 1, n)
    j = rng.integers(1, MY - 1, n)
    k = rng.integers(1, MZ - 1, n)
    return np.stack([i, j, k], axis=1)


def summarize(prob, conv, itr, res0, hist, extra=None):
    th = prob.wk["theta"]
    inner = th[1:-1, 1:-1, 1:-1]
    idx = sample_cells(th.shape)
    d = {
        "isconverged": conv,
        "itr": itr,
        "res0": res0,
        "hist": [float(h) for h in hist],
        "theta_min": float(inner.min()),
        "theta_max": float(inner.max()),
        "theta_l2": float(np.linalg.norm(inner)),
        "theta_sum": float(inner.sum()),
        "sample_ijk": idx.tolist(),
        "sample_theta": [float(th[a, b, c]) for a, b, c in idx],
    }
    if extra:
        d.update(extra)
    return d


def run_oracle(NX, eps, method="pbicgstab", red=O.RED_SEQ, symmetric=False):
    prob = O.build_mode3(NX, NX, 30, symmetric=symmetric, threads=os.cpu_count())
    t = time.time()
    fn = O.pbicgstab if method == "pbicgstab" else O.cg
    conv, itr, res0, hist = fn(prob, tol=eps, maxItr=20000, smoother="gs", red_mode=red, threads=os.cpu_count())
    el = time.time() - t
    print(f"{method} NX={NX} eps={eps} sym={symmetric}: conv={conv} itr={itr} res0={res0!r} t={el:.1f}s")
    return summarize(prob, conv, itr, res0, hist, {
        "NX": NX, "NY": NX, "NZ": 30, "epsilon": eps, "method": method, "smoother": "gs",
        "reduction": "sequential" if red == O.RED_SEQ else "openmp", "symmetric": symmetric,
        "oracle_seconds": el, "oracle_threads": os.cpu_count()})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="checkout of the reference (readme job)")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    if a.reference is None and (not a.only or "readme" in a.only.split(",")):
        ap.error("--reference is required for the readme job (or pick others with --only)")
    O.build()
    jobs = {
        "readme": lambda: ("readme_240.json", parse_readme(os.path.join(a.reference, "README.md"))),
        "oracle240": lambda: ("oracle_240_1e-4.json", run_oracle(240, 1e-4, red=O.RED_SEQ)),
        "oracle240_8": lambda: ("oracle_240_1e-8.json", run_oracle(240, 1e-8, red=O.RED_OMP)),
        "cgsym": lambda: ("oracle_240_cg_sym.json", run_oracle(240, 1e-8, method="cg", red=O.RED_OMP,
                                                                  symmetric=True)),
    }
    for name, job in jobs.items():
        if a.only and name not in a.only.split(","):
            continue
        fname, data = job()
        with open(os.path.join(HERE, fname), "w") as fh:
            json.dump(data, fh, indent=1)
        print("wrote", fname)


if __name__ == "__main__":
    main()
