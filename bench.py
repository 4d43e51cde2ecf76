#!/usr/bin/env python
"""Benchmark: PBiCGSTAB + RB-GS(5) time-to-eps on the Heat3ds Mode-3 IC stack, 240x240x30.

One step = one steady solve from theta = 300 K to ||r||/||r0|| <= 1e-8 on inputs resident in
HBM.  The headline `value` is the FP64 GPU solver (every kernel bit-identical per cell to the
reference's FP64 arithmetic).  The mixed variant (FP32 RB-GS preconditioner inside the FP64
PBiCGSTAB, restarted on the FP64 true residual) is timed on the same inputs and reported beside
it with its max |theta - theta_FP64|; on this operator it needs about twice the iterations, so
it is slower (the measured evidence is in the JSON line).  CG + RB-GS on the symmetric variant of
the stack (adiabatic instead of convective faces) is timed in FP64 and mixed precision too.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun, one process per GPU): every rank runs its own replica of the solve (the solve
does not shard), timing is the max over ranks.  --impl reference times the reference's CPU
algorithm (the oracle port, OpenMP on all host cores) on a bounded sample of iterations, scaled
to the iterations its FP64 solve needs.  One JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PBiCGSTAB time-to-eps (s) + stencil HBM GB/s, mixed vs FP64 GPU at 240^2x30"
L2_FLUSH_BYTES = 256 << 20


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=240)
    ap.add_argument("--nz", type=int, default=30)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--kernel-reps", type=int, default=30)
    ap.add_argument("--cpu-sample-iters", type=int, default=0, help="0 = choose ~10 s of CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=64, help="members of the batched workload (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--cg", type=int, default=1,
                    help="1 = also time CG + RB-GS on the symmetric variant (adiabatic instead of convective faces)")
    ap.add_argument("--adjoint-steps", type=int, default=200,
                    help="implicit steps of the timed transient adjoint (0 = skip the adjoint section)")
    ap.add_argument("--scaling", type=int, default=1,
                    help="1 = also measure the scaling grids (480^2x60: FP64 and mixed solves and sweep rates; "
                         "960^2x120: sweep rates)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_name(a):
    return (f"{a.nx}x{a.nx}x{a.nz} Mode-3 IC stack, steady, PBiCGSTAB + RB-GS(5 sweeps), FP64, "
            f"to ||r||/||r0|| <= {a.tol:g}")


def bench_config(a):
    """The workload of one step; identical in both arms."""
    return {"workload": workload_name(a), "grid": [a.nx, a.nx, a.nz], "tol": a.tol, "smoother": "RB-GS, 5 sweeps",
            "method": "PBiCGSTAB", "precision": "fp64"}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas)
# ----------------------------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception as e:  # pragma: no cover
            log("clock sampling unavailable:", e)
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        smax = max(num(r[2]) or 0 for r in rows)
        load = [s for s in sm if s > 0.5 * smax] or sm
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": smax, "samples": len(rows),
                "power_w_max": max(num(r[3]) or 0 for r in rows), "reasons": sorted(reasons)}


def gpu_id_for(torch, dev: int) -> str:
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        return vis.split(",")[dev] if vis else str(dev)


# ----------------------------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle port (the reference's algorithm), all host threads
# ----------------------------------------------------------------------------------------------
def fp64_reference_iterations(nx: int, nz: int, tol: float) -> int | None:
    """Iterations the reference's FP64 PBiCGSTAB needs for this workload (committed oracle run)."""
    p = os.path.join(ROOT, "tests", "golden", "oracle_240_1e-8.json")
    if nx == 240 and nz == 30 and tol == 1e-8 and os.path.exists(p):
        return int(json.load(open(p))["itr"])
    return None


class CpuBaseline:
    def __init__(self, nx, nz):
        from oracle import oracle as O  # the reference's algorithm restated in C (checker/baseline only)
        O.build()
        self.O = O
        self.cores = os.cpu_count()
        t = time.perf_counter()
        self.prob0 = O.build_mode3(nx, nx, nz, threads=self.cores)
        log(f"oracle model {nx}x{nx}x{nz}: {time.perf_counter() - t:.1f} s")

    def time_iters(self, iters: int) -> float:
        import copy
        prob = copy.deepcopy(self.prob0)
        t = time.perf_counter()
        self.O.pbicgstab(prob, tol=0.0, maxItr=iters, smoother="gs", red_mode=self.O.RED_OMP, threads=self.cores)
        return time.perf_counter() - t

    def calibrate(self, target_s=10.0) -> int:
        t1 = self.time_iters(2) / 2
        return max(3, min(200, int(target_s / max(t1, 1e-4))))


def run_reference(a, dist: Dist):
    dist.init("gloo")
    if dist.rank != 0:
        dist.close()
        return
    iters_ref = fp64_reference_iterations(a.nx, a.nz, a.tol)
    cb = CpuBaseline(a.nx, a.nz)
    per_step = a.cpu_sample_iters or max(3, cb.calibrate(target_s=2.5))
    for _ in range(a.warmup):
        cb.time_iters(per_step)
    times = [cb.time_iters(per_step) for _ in range(a.steps)]
    t_iter = float(np.mean(times)) / per_step
    if iters_ref is None:
        iters_ref = 315
    value = t_iter * iters_ref
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference Mode-3 model)",
        "config": bench_config(a),
        "parallelism": f"host threads x{cb.cores}",
        "cpu_baseline": {"value": value, "unit": "s", "cores": cb.cores, "kind": "port", "cpu_model": cpu_model(),
                         "extrapolated": True,
                         "sample": f"{per_step} PBiCGSTAB iterations per step (OpenMP reductions, "
                                   f"{cb.cores} threads); value = mean time per iteration x the {iters_ref} "
                                   f"iterations the oracle's FP64 solve needs to reach the tolerance "
                                   f"(extrapolated from the bounded sample, not a full solve)"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "seconds_per_iteration": t_iter,
    }
    print(json.dumps(line), flush=True)
    dist.close()


def cpu_baseline_leg(a, it64: int) -> dict:
    """The oracle (the reference's algorithm in C, OpenMP on all host cores) on the same workload:
    one full FP64 solve to the tolerance when it takes under ~40 s, else a bounded sample of
    iterations scaled to the GPU solve's iteration count (said so in `sample`)."""
    cb = CpuBaseline(a.nx, a.nz)
    t1 = cb.time_iters(2) / 2
    base = {"unit": "s", "cores": cb.cores, "kind": "port", "cpu_model": cpu_model()}
    if t1 * it64 <= 40.0:
        import copy
        prob = copy.deepcopy(cb.prob0)
        t = time.perf_counter()
        conv, itr, _, _ = cb.O.pbicgstab(prob, tol=a.tol, maxItr=20000, smoother="gs", red_mode=cb.O.RED_OMP,
                                         threads=cb.cores)
        tcpu = time.perf_counter() - t
        return {"value": tcpu, **base, "extrapolated": False, "iterations": itr, "converged": bool(conv),
                "sample": f"one full FP64 PBiCGSTAB+RB-GS solve of the oracle to ||r||/||r0|| <= {a.tol:g} "
                          f"({itr} iterations, OpenMP reductions, {cb.cores} threads)"}
    iters = a.cpu_sample_iters or cb.calibrate(target_s=10.0)
    tcpu = cb.time_iters(iters)
    return {"value": tcpu / iters * it64, **base, "extrapolated": True,
            "sample": f"{iters} FP64 PBiCGSTAB+RB-GS iterations of the oracle (OpenMP, {cb.cores} threads) in "
                      f"{tcpu:.2f} s, scaled to the {it64} iterations of the GPU FP64 solve"}


# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu capture each (see the
# profiles/ summaries): key (nx, nz, fused, coefficient source: 1 dd array + key word, 2 class table).
SWEEP_TRAFFIC_F64 = {(240, 30, False, 1): 37.463e6, (240, 30, False, 2): 24.584e6, (480, 60, False, 2): 222.2e6}


def kernel_rates(nx, nz, solvers, torch, stream, flush, reps):
    """Algorithmic GB/s of one RB-GS sweep (one fused launch or two colour passes, whichever the
    handle's tuner chose) and of CalcAX, per handle: warm = CUDA events around `reps` back-to-back
    launches on resident data, as inside a solve; cold = the L2 flushed (256 MiB write) before each
    single launch.  Algorithmic bytes per cell: sweep 3w + 1 (x read and written, b, one key byte),
    CalcAX 2*8 + 1 (FP64 in both handles)."""
    N = nx * nx * nz
    out = {}
    for name, s in solvers.items():
        w_elem = 8 if name == "fp64" else 4
        fused = bool(s.sweep()[0])
        source = s.tuning()[2]
        for kind, bytes_per_cell, label in ((0, 3 * w_elem + 1, "rb_sweep"), (1, 2 * 8 + 1, "calcax")):
            cold = []
            for r in range(reps + 3):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.bench_kernel(kind, 1)
                e1.record(stream)
                e1.synchronize()
                if r >= 3:
                    cold.append(e0.elapsed_time(e1) * 1e-3)
            s.bench_kernel(kind, 3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.bench_kernel(kind, reps)
            e1.record(stream)
            e1.synchronize()
            warm = e0.elapsed_time(e1) * 1e-3 / reps
            tc = float(np.mean(cold))
            nbytes = bytes_per_cell * N
            out[(name, label)] = {"seconds": warm, "gbs": nbytes / warm / 1e9, "seconds_cold": tc,
                                  "gbs_cold": nbytes / tc / 1e9, "bytes": nbytes,
                                  "launches": (1 if fused else 2) if kind == 0 else 1,
                                  "fused": fused if kind == 0 else None, "source": source}
    return out


def roofline_object(rm, peak, peak_kind, nx, nz):
    fused = bool(rm["fused"])
    src = rm.get("source", 1)
    name = ("k_rb_sweep<double>: one fused RB-GS sweep (both colours, TMA-staged z-march) of the FP64 smoother"
            if fused else "k_rb_pass<double>: one RB-GS sweep (colour 0 then colour 1) of the FP64 smoother, "
            + {0: "dd summed per cell", 1: "dd read per cell", 2: "coefficients from the stencil-class table"}[src])
    traffic = SWEEP_TRAFFIC_F64.get((nx, nz, fused, src))
    return {"bound": "hbm", "achieved": rm["gbs"], "peak": peak, "unit": "GB/s", "frac": rm["gbs"] / peak,
            "traffic": None if traffic is None else traffic * rm["launches"],
            "traffic_unit": f"DRAM bytes per sweep ({rm['launches']} launch(es)), ncu, L2 flushed",
            "kernel": name, "algorithmic_bytes": rm["bytes"], "seconds": rm["seconds"],
            "timing": "warm: CUDA events around back-to-back sweeps on resident data, as inside the solve "
                      "(at 240^2x30 the working set is L2-resident)",
            "cold": {"achieved": rm["gbs_cold"], "frac": rm["gbs_cold"] / peak, "seconds": rm["seconds_cold"],
                     "timing": "L2 flushed before each launch"},
            "peak_kind": peak_kind}


def run_scaling(a, dist, torch, stream, flush, peak):
    """The scaling grids of the workload (the reference's stack, Z cells split uniformly): at
    480x480x60 one FP64 and one mixed solve to a.tol (after one untimed solve each) and the sweep
    rates; at 960x960x120 the sweep rates.  CUDA events; L2 flushed before each solve."""
    import h2_b200
    from h2_b200 import model as M

    out = {}
    for nx, nz, solve in ((480, 60, True), (960, 120, False)):
        m = M.build_mode3(nx, nx, nz)
        w = m.wk
        solvers, entry = {}, {}
        try:
            for name in ("fp64", "mixed"):
                s = h2_b200.Solver(*m.shape, precision=name, stream=stream.cuda_stream)
                solvers[name] = s
                s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
                s.set_fields(w.lam, w.mask)
                s.set_rhs(w.b)
                s.set_theta(w.theta)
                s.snapshot()
                if solve:
                    ts, res = [], None
                    for r in range(2):
                        s.snapshot(restore=True)
                        with torch.cuda.stream(stream):
                            flush.zero_()
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        st, res = s.solve("pbicgstab", tol=a.tol, maxItr=20000, smoother="gs")
                        e1.record(stream)
                        e1.synchronize()
                        if r:
                            ts.append(e0.elapsed_time(e1) * 1e-3)
                    entry[name] = {"seconds": ts[0], "iterations": res.itr, "status": st,
                                   "final_rel_residual": res.res, "restarts": res.outer}
            if solve:
                th = {k: v.get_theta()[1:-1, 1:-1, 1:-1] for k, v in solvers.items()}
                entry["mixed"]["max_abs_dtheta_vs_fp64_K"] = float(np.abs(th["mixed"] - th["fp64"]).max())
            rates = kernel_rates(nx, nz, solvers, torch, stream, flush, 10)
            for (name, label), v in rates.items():
                v["frac_cold"] = v["gbs_cold"] / peak
                v["frac"] = v["gbs"] / peak
                entry[f"{name}_{label}"] = v
        except Exception as e:  # pragma: no cover
            log(f"scaling grid {nx}^2x{nz} failed:", e)
            entry = {"error": str(e)}
        finally:
            for s in solvers.values():
                s.close()
        out[f"{nx}x{nx}x{nz}"] = entry
    return out


# ----------------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------------
def run_ours(a, dist: Dist):
    import torch

    import h2_b200
    from h2_b200 import _lib as L
    from h2_b200 import model as M

    dist.init("nccl")
    dev = dist.local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    t = time.perf_counter()
    m = M.build_mode3(a.nx, a.nx, a.nz)
    log(f"[rank {dist.rank}] model {a.nx}x{a.nx}x{a.nz} (GPU fillID!): {time.perf_counter() - t:.2f} s")
    w = m.wk

    def make(precision):
        s = h2_b200.Solver(*m.shape, precision=precision, stream=stream.cuda_stream)
        s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
        s.set_fields(w.lam, w.mask)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        s.snapshot()
        return s

    solvers = {"fp64": make("fp64"), "mixed": make("mixed")}

    def one(s, timed: bool, tol=None):
        s.snapshot(restore=True)
        with torch.cuda.stream(stream):
            flush.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        st, res = s.solve("pbicgstab", tol=a.tol if tol is None else tol, maxItr=20000, smoother="gs")
        ev1.record(stream)
        ev1.synchronize()
        if st != 0:
            raise RuntimeError(f"solve did not converge: status {st}")
        return ev0.elapsed_time(ev1) * 1e-3, res

    results = {}
    clocks = Clocks(gpu_id_for(torch, dev))
    for name in ("fp64", "mixed"):
        s = solvers[name]
        for _ in range(a.warmup):
            one(s, False)
        torch.cuda.synchronize()
        dist.barrier()
        if name == "fp64":
            clocks.start()
        times, launches, res = [], 0, None
        for _ in range(a.steps):
            dt_, res = one(s, True)
            times.append(dt_)
            launches += res.launches
        torch.cuda.synchronize()
        dist.barrier()
        results[name] = dict(t=dist.max(float(np.mean(times))), times=times, res=res, launches=launches)
        if name == "fp64":
            clk = clocks.stop()

    th = {k: solvers[k].get_theta()[1:-1, 1:-1, 1:-1] for k in solvers}
    max_dtheta = float(np.abs(th["mixed"] - th["fp64"]).max())

    # ---- the case the reference publishes a solve time for: the same solve to eps = 1e-4
    readme = None
    if a.nx == 240 and a.nz == 30:  # the same decision on every rank
        ts_r, res_r = [], None
        for r in range(2 + a.steps):
            dt_, res_r = one(solvers["fp64"], True, tol=1e-4)
            if r >= 2:
                ts_r.append(dt_)
        readme = {"tol": 1e-4, "seconds": dist.max(float(np.mean(ts_r))), "iterations": res_r.itr,
                  "reference_published": {"seconds": 183.0, "iterations": 208, "hardware": "not stated",
                                          "source": "the reference's README.md:174-182 (Julia; compute time of this solve)"}}

    # ---- roofline of the dominant kernel: one RB-GS sweep (one fused launch, or two colour passes)
    peak, peak_kind = measured_peaks()
    roof = kernel_rates(a.nx, a.nz, solvers, torch, stream, flush, a.kernel_reps)

    # ---- end to end through the public drop-in call with pinned host buffers
    e2e, e2e_local = None, float("nan")
    try:
        shape = m.shape
        nf = int(np.prod(shape))

        def pinned():
            t_ = torch.empty(nf, dtype=torch.float64, pin_memory=True)
            return t_, np.ndarray(shape, dtype=np.float64, buffer=t_.numpy(), order="F")

        keep = []
        wk = h2_b200.WorkBuffers.allocate(*shape)
        for f in ("theta", "b", "lam", "mask", "rho", "cp"):
            t_, arr = pinned()
            keep.append(t_)
            arr[...] = getattr(w, f)
            setattr(wk, f, arr)
        theta0 = w.theta.copy(order="F")
        et = []
        for r in range(a.warmup + a.steps):
            wk.theta[...] = theta0
            t0 = time.perf_counter()
            conv, itr, res0 = h2_b200.PBiCGSTAB(wk, (m.dx, m.dy, 1.0), m.dt, m.ZC, m.dZ, m.HC, tol=a.tol,
                                                smoother="gs", par="gpu", is_steady=True, precision="fp64")
            t1 = time.perf_counter()
            if not conv:
                raise RuntimeError("e2e solve did not converge")
            if r >= a.warmup:
                et.append(t1 - t0)
        L.load().h2g_release_cached()
        e2e_local = float(np.mean(et))
        e2e = {"unit": "s", "h2d_bytes_per_step": 4 * 8 * nf + 8 * (2 * shape[2] + 6),
               "d2h_bytes_per_step": 8 * nf,
               "call": "h2g_PBiCGSTAB (one-call drop-in, host arrays in pinned memory)"}
    except Exception as e:  # pragma: no cover
        log("e2e failed:", e)
    e2e_max = dist.max(e2e_local)  # every rank takes this collective, whatever happened above
    if e2e is not None:
        e2e = {"value": e2e_max, **e2e}

    variants = run_mixed_variants(a, m, th["fp64"], max_dtheta, results, torch, stream, flush)
    cg_sym = run_cg_symmetric(a, dist, torch, stream, flush) if a.cg else None
    batch = run_batch(a, dist, torch, stream, flush) if a.batch > 0 else None
    adjoint = run_adjoint(a, dist, torch, stream) if a.adjoint_steps > 0 else None

    cpu = None
    if dist.rank == 0 and dist.world == 1 and not a.no_cpu_baseline:
        try:
            cpu = cpu_baseline_leg(a, results["fp64"]["res"].itr)
        except Exception as e:  # pragma: no cover
            log("cpu baseline failed:", e)

    rm = roof[("fp64", "rb_sweep")]
    scaling = run_scaling(a, dist, torch, stream, flush, peak) if a.scaling else None
    f64, mx = results["fp64"], results["mixed"]
    out = {
        "metric": METRIC,
        "value": f64["t"],
        "unit": "s",
        "n_gpus": dist.world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": f64["t"] * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: the reference's Mode-3 IC-stack model (GPU fillID!, heat source 1.6e11 W/m^3 "
                "on the power grids), theta_init = 300 K",
        "config": bench_config(a),
        "l2": "flushed (256 MiB write) before every timed solve; kernels timed warm (back to back, as inside "
              "the solve) and cold (L2 flushed before each launch)",
        "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
        "fp64": {"seconds": f64["t"], "iterations": f64["res"].itr, "final_rel_residual": f64["res"].res},
        "mixed": {"seconds": mx["t"], "iterations": mx["res"].itr, "restarts": mx["res"].outer,
                  "final_rel_residual": mx["res"].res, "max_abs_dtheta_vs_fp64_K": max_dtheta,
                  "precision": "FP32 RB-GS preconditioner (tables, smoother vectors); FP64 Krylov vectors, "
                               "inner products, CalcAX and solution"},
        "speedup_mixed_vs_fp64": f64["t"] / mx["t"],
        "mixed_variants": variants,
        "roofline": roofline_object(rm, peak, peak_kind, a.nx, a.nz),
        "kernels": {f"{k[0]}_{k[1]}": v for k, v in roof.items()},
        "scaling_configs": scaling,
        "readme_case": readme,
        "cg_symmetric": cg_sym,
        "batch": batch,
        "adjoint": adjoint,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": f64["launches"],
        "clocks": clk,
    }
    if dist.rank == 0:
        print(json.dumps(out), flush=True)
    for s in solvers.values():
        s.close()
    dist.close()


# Bytes per cell of one PBiCGSTAB iteration on the fused path (keys 1 byte), per precision form:
# the speed-up each form could reach at equal iterations when every kernel is memory-bound.
ITERATION_BYTES = {"fp64": 388, "mixed": 276, "mixed_ir": 200}


def run_mixed_variants(a, m, th64, max_dtheta, results, torch, stream, flush):
    """The precision forms side by side on the benchmark grid: FP64, H2G_MIXED (FP32 smoother in
    FP64 PBiCGSTAB, restarts on the FP64 true residual) and H2G_MIXED_IR (FP32 operator, smoother
    and Krylov vectors inside FP64 iterative refinement), one solve each after the timed ones (the
    IR form capped at 4000 inner iterations); time, iterations, status, max |theta - theta_FP64|
    (th64: the interior of the timed FP64 solve's field) and the byte-model ceiling at equal
    iterations."""
    import h2_b200
    out = {}
    for name, res_t in (("fp64", results["fp64"]), ("mixed", results["mixed"])):
        r = res_t["res"]
        out[name] = {"seconds": res_t["t"], "iterations": r.itr, "status": r.status, "restarts": r.outer,
                     "ceiling_at_equal_iterations": ITERATION_BYTES["fp64"] / ITERATION_BYTES[name]}
    out["mixed"]["max_abs_dtheta_vs_fp64_K"] = max_dtheta
    w = m.wk
    s = h2_b200.Solver(*m.shape, precision="mixed_ir", stream=stream.cuda_stream)
    try:
        s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
        s.set_fields(w.lam, w.mask)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, r = s.solve("pbicgstab", tol=a.tol, maxItr=4000, smoother="gs")
        e1.record(stream)
        e1.synchronize()
        entry = {"seconds": e0.elapsed_time(e1) * 1e-3, "iterations": r.itr, "status": st, "outer": r.outer,
                 "final_rel_residual": r.res, "ceiling_at_equal_iterations": ITERATION_BYTES["fp64"] / ITERATION_BYTES["mixed_ir"]}
        if st == 0:
            entry["max_abs_dtheta_vs_fp64_K"] = float(np.abs(s.get_theta()[1:-1, 1:-1, 1:-1] - th64).max())
        out["mixed_ir"] = entry
    except Exception as e:  # pragma: no cover
        out["mixed_ir"] = {"error": str(e)}
    finally:
        s.close()
    out["status_codes"] = "0 converged, 1 not converged, 2 breakdown, 3 non-finite"
    return out


def run_cg_symmetric(a, dist, torch, stream, flush):
    """CG + RB-GS(5) on the symmetric variant of the same stack: the convective faces replaced by
    adiabatic ones (heat_flux_bc(0.0)), which leaves the operator symmetric positive definite.
    FP64 and mixed precision from theta = 300 K to a.tol; CUDA events around each solve, L2
    flushed before each; max over ranks."""
    import h2_b200
    from h2_b200 import model as M

    m = M.build_mode3(a.nx, a.nx, a.nz, symmetric=True)
    w = m.wk
    out, solvers, local = {}, {}, {}
    try:
        for name in ("fp64", "mixed"):
            s = h2_b200.Solver(*m.shape, precision=name, stream=stream.cuda_stream)
            solvers[name] = s
            s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
            s.set_fields(w.lam, w.mask)
            s.set_rhs(w.b)
            s.set_theta(w.theta)
            s.snapshot()
            ts, res = [], None
            for r in range(a.warmup + a.steps):
                s.snapshot(restore=True)
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st, res = s.solve("cg", tol=a.tol, maxItr=20000, smoother="gs")
                e1.record(stream)
                e1.synchronize()
                if st != 0:
                    raise RuntimeError(f"CG ({name}) did not converge: status {st}")
                if r >= a.warmup:
                    ts.append(e0.elapsed_time(e1) * 1e-3)
            local[name] = float(np.mean(ts))
            out[name] = {"iterations": res.itr, "restarts": res.outer, "final_rel_residual": res.res}
        th = {k: v.get_theta()[1:-1, 1:-1, 1:-1] for k, v in solvers.items()}
        out["mixed"]["max_abs_dtheta_vs_fp64_K"] = float(np.abs(th["mixed"] - th["fp64"]).max())
    except Exception as e:  # pragma: no cover
        log("CG on the symmetric variant failed:", e)
        out = {"error": str(e)}
    finally:
        for s in solvers.values():
            s.close()
    # every rank takes the same collectives, whatever happened above
    for name in ("fp64", "mixed"):
        t_ = dist.max(local.get(name, float("nan")))
        if name in out:
            out[name]["seconds"] = t_
    out["workload"] = (f"{a.nx}x{a.nx}x{a.nz} Mode-3 stack with adiabatic instead of convective faces, steady, "
                       f"CG + RB-GS(5 sweeps), to ||r||/||r0|| <= {a.tol:g}")
    return out


def run_batch(a, dist, torch, stream, flush):
    """The batched workload: a.batch steady solves (seeded hotspot heat maps, grids drawn from
    120^2/180^2/240^2 x 30), sharded across ranks by cell count, each rank's members solved
    concurrently by one h2g_batch_solve.  Time = max over ranks of the CUDA-event time of the
    (synchronous) call."""
    from h2_b200 import batch as B
    members = B.draw_batch(a.batch, 1000)
    mine = [members[i] for i in B.shard(members, dist.world)[dist.rank]]
    t0 = time.perf_counter()
    bs = B.BatchSolver(mine)
    t_setup = time.perf_counter() - t0

    def timed(batch, fn):
        batch.restore()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()  # synchronous: returns when every member's stream is idle
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3, out

    try:
        timed(bs, lambda: bs.solve(tol=a.tol))  # warm-up: graph instantiation per handle
        dist.barrier()
        ts, res = [], None
        for _ in range(max(1, a.batch_steps)):
            dt_, (st, res) = timed(bs, lambda: bs.solve(tol=a.tol))
            ts.append(dt_)
        dist.barrier()
        t_seq, _ = timed(bs, lambda: bs.solve_sequential(tol=a.tol))
        local = {m.index: {"itr": r.itr, "conv": r.isconverged} for m, r in zip(mine, res)}
        merged = B.gather_results(local)
        out = {"solves": a.batch, "cells": sum(m.cells for m in members),
               "sizes": {str(n): sum(1 for m in members if m.nx == n) for n in B.SIZES},
               "seconds": dist.max(float(np.mean(ts))), "steps": len(ts),
               "sequential_seconds_rank0": t_seq,
               "speedup_vs_sequential": t_seq / float(np.mean(ts)),
               "setup_seconds_rank0": t_setup,
               "timing": "CUDA events around the synchronous call (includes its host-side issue of the solves)",
               "precision": "fp64", "method": "PBiCGSTAB + RB-GS(5)", "tol": a.tol,
               "sharding": f"greedy by cell count over {dist.world} rank(s)"}
        if merged is not None:
            out["iterations_total"] = int(sum(v["itr"] for v in merged.values()))
            out["all_converged"] = bool(all(v["conv"] for v in merged.values()))
        th64 = [s.get_theta() for s in bs.solvers]
    finally:
        bs.close()
    # the config's precision form: FP32 smoother inside FP64 PBiCGSTAB with FP64 restarts on the
    # true residual (H2G_MIXED), one timed call after an untimed one; max |dtheta| against FP64
    bm = B.BatchSolver(mine, precision="mixed")
    try:
        timed(bm, lambda: bm.solve(tol=a.tol))
        t_m, (st_m, res_m) = timed(bm, lambda: bm.solve(tol=a.tol))
        local_m = float(max(np.abs(s.get_theta() - t).max() for s, t in zip(bm.solvers, th64)))
        out["mixed"] = {"seconds": dist.max(t_m), "iterations_total_rank0": int(sum(r.itr for r in res_m)),
                        "restarts_total_rank0": int(sum(r.outer for r in res_m)),
                        "all_converged_rank0": bool(all(r.isconverged for r in res_m)),
                        "max_abs_dtheta_vs_fp64_K": dist.max(local_m),
                        "precision": "FP32 RB-GS smoother in FP64 PBiCGSTAB, restarted on the FP64 true residual"}
    finally:
        bm.close()
    return out


def run_adjoint(a, dist, torch, stream):
    """Gradients of J = (sum_silicon V theta^8)^(1/8) on the benchmark grid: the steady adjoint
    (forward + adjoint solve, to 1e-10) and the transient adjoint (a.adjoint_steps implicit steps
    of dt = 1e-4 s with checkpointed recomputation, to 1e-10).  CUDA events around each call."""
    import h2_b200
    from h2_b200 import adjoint as A
    from h2_b200 import model as M

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3, out

    out = {}
    m = M.build_mode3(a.nx, a.nx, a.nz)
    w = m.wk
    wts = A.silicon_weights(m.ID, m.dx, m.dy, m.dZ)
    s = h2_b200.Solver(*m.shape, stream=stream.cuda_stream)
    try:
        s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
        s.set_fields(w.lam, w.mask)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        s.snapshot()
        ts = []
        for r in range(3):
            s.snapshot(restore=True)
            dt_, (J, _, _, rf, ra) = timed(lambda: A.steady_gradient(s, wts, 8.0, tol=1e-10))
            if r:
                ts.append(dt_)
        out["steady"] = {"seconds": dist.max(float(np.mean(ts))), "J": J, "forward_iterations": rf.itr,
                         "adjoint_iterations": ra.itr, "tol": 1e-10}
    finally:
        s.close()
    nt = a.adjoint_steps
    mt = M.build_mode3(a.nx, a.nx, a.nz, is_steady=False, dt=1e-4)
    w = mt.wk
    s = h2_b200.Solver(*mt.shape, stream=stream.cuda_stream)
    try:
        s.set_grid(mt.ZC, mt.dZ, mt.dx, mt.dy, mt.dt, mt.HC, False)
        s.set_fields(w.lam, w.mask, w.rho, w.cp)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        s.set_hsrc(w.hsrc)
        s.snapshot()
        t_fwd, (st, res, stats) = timed(lambda: s.transient(mt.bcs, nt, tol=1e-10, smoother="gs"))
        s.snapshot(restore=True)
        k = max(1, int(np.ceil(np.sqrt(nt))))
        t_adj, (J, _, _, r) = timed(lambda: A.transient_gradient(s, mt.bcs, nt, wts, 8.0, tol=1e-10,
                                                                 checkpoint_every=k))
        out["transient"] = {"steps": nt, "dt": 1e-4, "seconds": dist.max(t_adj), "forward_only_seconds": t_fwd,
                            "J": J, "iterations_total": r.itr, "forward_iterations": int(stats[:, 3].sum()),
                            "checkpoint_every": k, "tol": 1e-10}
    finally:
        s.close()
    out["objective"] = "(sum over silicon cells of V theta^8)^(1/8); gradients w.r.t. hsrc per cell and ln lambda"
    return out


def main():
    a = parse()
    dist = Dist()
    if a.impl == "reference":
        run_reference(a, dist)
    else:
        run_ours(a, dist)


if __name__ == "__main__":
    main()
