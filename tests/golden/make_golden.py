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
oracle_480x60_1e-8.json  the oracle at 480x480x60 (each Zcase2! cell split in two), epsilon = 1e-8,
                     OpenMP reductions: the FP64 reference of the first scaling grid.
oracle_batch3.json   three members of the 64-member batched workload (seed 1000; the first member
                     of each size 120^2, 180^2, 240^2 x 30) solved by the oracle to 1e-8.
oracle_adjoint_240.json  the steady adjoint at 240x240x30: J = (sum_silicon V theta^8)^(1/8), the
                     oracle's FP64 forward and adjoint solves to 1e-10 and the numpy restatement of
                     the gradient (oracle/adjoint.py): J, per-plane sums and 4096 sampled cells of
                     dJ/dhsrc and dJ/dln(lambda).
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


def run_oracle(NX, eps, method="pbicgstab", red=O.RED_SEQ, symmetric=False, NZ=30):
    prob = O.build_mode3(NX, NX, NZ, symmetric=symmetric, threads=os.cpu_count())
    t = time.time()
    fn = O.pbicgstab if method == "pbicgstab" else O.cg
    conv, itr, res0, hist = fn(prob, tol=eps, maxItr=20000, smoother="gs", red_mode=red, threads=os.cpu_count())
    el = time.time() - t
    print(f"{method} NX={NX} eps={eps} sym={symmetric}: conv={conv} itr={itr} res0={res0!r} t={el:.1f}s")
    return summarize(prob, conv, itr, res0, hist, {
        "NX": NX, "NY": NX, "NZ": NZ, "epsilon": eps, "method": method, "smoother": "gs",
        "reduction": "sequential" if red == O.RED_SEQ else "openmp", "symmetric": symmetric,
        "oracle_seconds": el, "oracle_threads": os.cpu_count()})


def run_batch3(eps=1e-8):
    """The first member of each grid size in draw_batch(64, 1000), solved by the oracle.  The heat
    map is the workload's definition (h2_b200/batch.py: hotspot rectangles over the silicon)."""
    from h2_b200 import batch as B
    members = B.draw_batch(64, 1000)
    out = []
    for nx in B.SIZES:
        m = next(x for x in members if x.nx == nx)
        ID = O.fill_id(nx, nx, B.NZ, os.cpu_count())
        _, ZC, _ = O.genz(B.NZ)
        hs = B.heat_map(m, ID, ZC, O.pitch(nx), O.pitch(nx))
        prob = O.build_mode3(nx, nx, B.NZ, ID=ID, hsrc=hs, threads=os.cpu_count())
        t = time.time()
        conv, itr, res0, hist = O.pbicgstab(prob, tol=eps, maxItr=20000, smoother="gs", red_mode=O.RED_OMP,
                                            threads=os.cpu_count())
        print(f"batch member {m.index} ({nx}^2): conv={conv} itr={itr} t={time.time() - t:.1f}s", flush=True)
        out.append(summarize(prob, conv, itr, res0, hist, {"index": m.index, "nx": nx, "epsilon": eps}))
    return {"members": out, "seed0": 1000, "batch": 64}


def run_adjoint240(eps=1e-10, p=8.0):
    """Steady adjoint of J = (sum_silicon V theta^8)^(1/8) on the 240x240x30 model."""
    from oracle import adjoint as OA
    thr = os.cpu_count()
    fwd = O.build_mode3(240, 240, 30, threads=thr)
    w = np.where(np.isin(fwd.ID, (2, 7)), (fwd.dx * fwd.dy) * fwd.dZ[None, None, :], 0.0)
    w[0], w[-1], w[:, 0], w[:, -1], w[:, :, 0], w[:, :, -1] = 0.0, 0.0, 0.0, 0.0, 0.0, 0.0
    w = np.asfortranarray(w)
    conv_f, itr_f, _, _ = O.pbicgstab(fwd, tol=eps, maxItr=20000, smoother="gs", red_mode=O.RED_OMP, threads=thr)
    th = fwd.wk["theta"].copy(order="F")
    J = OA.objective(th, w, p)
    adj = O.build_mode3(240, 240, 30, ID=fwd.ID, threads=thr, calrhs=False)
    adj.wk["theta"][...] = 0.0
    adj.wk["b"][...] = OA.adj_rhs(th, w, p)
    conv_a, itr_a, _, _ = O.pbicgstab(adj, tol=eps, maxItr=20000, smoother="gs", red_mode=O.RED_OMP, threads=thr)
    gh, gl = OA.gradients(fwd.wk["lam"], fwd.wk["mask"], th, adj.wk["theta"], fwd.dx, fwd.dy, fwd.ZC, fwd.dZ)
    idx = sample_cells(th.shape)
    print(f"adjoint 240: J={J!r} forward {itr_f} adjoint {itr_a}", flush=True)
    return {"epsilon": eps, "p": p, "J": J, "forward_itr": itr_f, "adjoint_itr": itr_a,
            "forward_converged": conv_f, "adjoint_converged": conv_a,
            "gh_plane_sum": gh.sum(axis=(0, 1)).tolist(), "gl_plane_sum": gl.sum(axis=(0, 1)).tolist(),
            "gh_absmax": float(np.abs(gh).max()), "gl_absmax": float(np.abs(gl).max()),
            "sample_ijk": idx.tolist(), "sample_gh": [float(gh[a, b, c]) for a, b, c in idx],
            "sample_gl": [float(gl[a, b, c]) for a, b, c in idx],
            "sample_theta": [float(th[a, b, c]) for a, b, c in idx]}


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
        "oracle480": lambda: ("oracle_480x60_1e-8.json", run_oracle(480, 1e-8, red=O.RED_OMP, NZ=60)),
        "batch3": lambda: ("oracle_batch3.json", run_batch3()),
        "adjoint240": lambda: ("oracle_adjoint_240.json", run_adjoint240()),
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
