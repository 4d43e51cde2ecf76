"""Microbenchmark of one solver kernel on the Mode-3 model: the command that profilers wrap.

    python -m h2_b200.kernel_bench --kind sweep --precision fp64 --nx 240 --nz 30 --reps 5

`--kind sweep` runs one RB-GS sweep of the preconditioner (colour 0, then colour 1: two
launches of the colour-pass kernel over x, b and the key array), `--kind calcax` one CalcAX!
launch, `--kind solve` one full PBiCGSTAB+GS solve to `--tol`.  Before every timed launch the
L2 is flushed by writing 256 MiB, so the kernel reads its operands from HBM.  Prints one JSON
line: microseconds per repetition (CUDA events on the library's stream) and, for the kernels,
algorithmic GB/s (x read + written, b read and one key byte per cell for a sweep; x read, ax
written and one key byte per cell for CalcAX).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

_KINDS = {"sweep": 0, "calcax": 1}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--kind", choices=["sweep", "calcax", "solve"], default="sweep")
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_ir"], default="fp64")
    ap.add_argument("--nx", type=int, default=240)
    ap.add_argument("--nz", type=int, default=30)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--tol", type=float, default=1e-8)
    a = ap.parse_args(argv)

    import torch

    import h2_b200
    from h2_b200 import model as M

    if not torch.cuda.is_available():
        raise SystemExit("kernel_bench needs a CUDA device")
    stream = torch.cuda.Stream()
    flush = torch.empty((256 << 20) // 4, dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    m = M.build_mode3(a.nx, a.nx, a.nz)
    t_model = time.perf_counter() - t0
    w = m.wk
    s = h2_b200.Solver(*m.shape, precision=a.precision, stream=stream.cuda_stream)
    s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
    s.set_fields(w.lam, w.mask)
    s.set_rhs(w.b)
    s.set_theta(w.theta)
    s.snapshot()

    times, launches, extra = [], 0, {}
    for r in range(a.warmup + a.reps):
        if a.kind == "solve":
            s.snapshot(restore=True)
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if a.kind == "solve":
            st, res = s.solve("pbicgstab", tol=a.tol, maxItr=20000, smoother="gs")
            if st != 0:
                raise SystemExit(f"solve status {st}")
            n = res.launches
            extra = {"iterations": res.itr, "final_rel_residual": res.res}
        else:
            n = s.bench_kernel(_KINDS[a.kind], 1)
        e1.record(stream)
        e1.synchronize()
        if r >= a.warmup:
            times.append(e0.elapsed_time(e1) * 1e3)
            launches += n
    N = a.nx * a.nx * a.nz
    w_elem = 8 if (a.precision == "fp64" or (a.kind == "calcax" and a.precision == "mixed")) else 4
    rows, planes, rb_dd, ax_dd = s.tuning()
    out = {"kind": a.kind, "precision": a.precision, "grid": [a.nx, a.nx, a.nz], "reps": a.reps,
           "tuning": {"rows": rows, "planes": planes, "rb_dd": rb_dd, "ax_dd": ax_dd},
           "us_per_rep": float(np.mean(times)), "us_min": float(np.min(times)),
           "launches_per_rep": launches / a.reps, "model_build_s": t_model}
    if a.kind != "solve":
        per_cell = 3 * w_elem + 1 if a.kind == "sweep" else 2 * w_elem + 1
        out["algorithmic_bytes"] = per_cell * N
        out["gbs"] = per_cell * N / (out["us_per_rep"] * 1e-6) / 1e9
    out.update(extra)
    print(json.dumps(out), flush=True)
    s.close()


if __name__ == "__main__":
    main()
