"""Benchmark: BP5 p=7 CG throughput (GDOF*iterations/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one "step"): the BP5 Hex3D problem on a 40x40x40 box with interior
vertices perturbed by 0.1h (seed 1), degree p=7, stored per-node geometric
factors, FP64 Jacobi-preconditioned CG for exactly 100 iterations from x=0
with the seeded nodal forcing b = M f, f = 2u-1 (seed 0).  21,717,639
unknowns.  `value` is device-timed with every input resident in HBM (the
step resets x and r, then runs the solve); `e2e` is the same solve through
the host-buffer entry point (b copied in from pinned memory, x copied back).

With --gpus N > 1 (launched by torch.distributed.run) every rank solves its
own replica of the problem: the path has no exchange at one rank per problem,
so scaling is weak and no collective is on the data path.

--impl reference times the reference's CPU algorithm (the oracle port; the
reference itself cannot be built here) on the host cores, on a bounded sample
of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BP5 p=7 GDOF·it/s: mixed+batched vs plain FP64 CG at 1e-8 rel residual"
UNIT = "GDOF·it/s"
NX, P, PERT, PERT_SEED, RHS_SEED, ITERS = 40, 7, 0.1, 1, 0, 100
WORKLOAD = ("BP5 Hex3D p=7, 40^3 elements, interior vertices perturbed 0.1h (seed 1), stored per-node factors, "
            "FP64 Jacobi-PCG, 100 iterations per step, forcing f=2u-1 (seed 0)")
# CPU sample: the same problem family on a 20^3 sub-box (1/8 of the elements)
CPU_NX, CPU_ITERS = 20, 100
MIXED_TOL = 1e-8
# DRAM traffic of one Ax launch of this workload, from the ncu capture summarised
# in profiles/ax_bp5_p7_40cubed.md (None until captured)
AX_DRAM_BYTES = None


def ax_model_bytes(Ndofs, E, Np, Nf=1):
    # reference byte model of one non-affine Ax (BP/BP5/src/bp5Run.cpp:106-142)
    return Ndofs * 8 + (Np * 7 * 8 + 4 + Np * Nf * 4 + Np * Nf * 8) * E


def cg_model_bytes(Ndofs, E, Np, iters):
    NL = E * Np
    bax = ax_model_bytes(Ndofs, E, Np)
    bg = (Ndofs + 1) * 4 + NL * 4 + NL * 8 + Ndofs * 8
    return (4 * Ndofs * 8 + bax + bg) + (11 * Ndofs * 8 + bax + bg) * iters


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [x.strip() for x in l.split(",")]
            if len(parts) != 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_sample(steps=1, warmup=0):
    """The oracle's Jacobi-PCG on the CPU sample; returns (GDOF*it/s, cores, sample text)."""
    from oracle import oracle as O
    m = O.Mesh(CPU_NX, CPU_NX, CPU_NX, P, pert=PERT, pert_seed=PERT_SEED)
    _, b = m.rhs_random(RHS_SEED)
    inv = 1.0 / m.jacobi_diag(1.0)
    lib = O.lib()
    times = []
    for s in range(warmup + steps):
        x = np.zeros(m.Ngather)
        r = b.copy()
        t0 = time.perf_counter()
        it = lib.bpo_cg(m._h, 1.0, O._dp(x), O._dp(r), 0.0, CPU_ITERS, 1, O._dp(inv), None, None)
        t1 = time.perf_counter()
        assert it == CPU_ITERS
        if s >= warmup:
            times.append(t1 - t0)
    tot = sum(times)
    v = m.Ngather * CPU_ITERS * steps / tot / 1e9
    sample = ("oracle Jacobi-PCG (the reference's CG and BP5 kernels restated in C++/OpenMP), BP5 p=7 on a %d^3 "
              "perturbed sub-box (%d unknowns, 1/8 of the elements), %d iterations per step" %
              (CPU_NX, m.Ngather, CPU_ITERS))
    return v, O.num_threads(), sample, tot / steps


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    v, cores, sample, sec = cpu_sample(steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": "20^3 sub-box, 100 iterations per step"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ax-launches", type=int, default=20)
    ap.add_argument("--no-mixed", action="store_true", help="skip the time-to-tolerance comparison")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_setup(args.gpus)
    import benchparanumal_b200 as bp

    bp.platform_init(local)
    L = bp.lib()
    mesh = bp.Mesh(NX, NX, NX, N=P, pert=PERT, pert_seed=PERT_SEED)
    S = bp.BP(mesh, precon="JACOBI")
    Nd, E, Np = mesh.Ngather, mesh.E, mesh.Np
    b = S.rhs("RANDOM", RHS_SEED)
    x = bp.DeviceBuffer(Nd)
    r = bp.DeviceBuffer(Nd)

    def step():
        bp._check(L.bp_memset(x.ptr, 0, x.nbytes, None))
        bp._check(L.bp_memcpy_dtod(r.ptr, b.ptr, r.nbytes, None))
        st = bp.SolveStats()
        bp._check(L.bp_solver_solve(S._h, x.ptr, r.ptr, 0.0, ITERS, None, None, bp.ctypes.byref(st)))
        return st

    def ev():
        e = bp.ctypes.c_void_p()
        bp._check(L.bp_event_create(bp.ctypes.byref(e)))
        return e.value

    for _ in range(args.warmup):
        st = step()
    assert st.iterations == ITERS
    rel_res = float(np.sqrt(st.rdotr / st.rdotr0))

    # ---- device-timed region: K steps, inputs resident in HBM ----
    e0, e1 = ev(), ev()
    clocks = ClockSampler(local)
    barrier(world)
    bp.finish()
    clocks.start()
    bp._check(L.bp_event_record(e0, None))
    for _ in range(args.steps):
        step()
    bp._check(L.bp_event_record(e1, None))
    bp.finish()
    barrier(world)
    clk = clocks.stop()
    ms = bp.ctypes.c_float()
    bp._check(L.bp_event_elapsed_ms(e0, e1, bp.ctypes.byref(ms)))
    t_dev = max_over_ranks(ms.value / 1e3, world)
    value = world * Nd * ITERS * args.steps / t_dev / 1e9
    # r = b - A x (operator + gather), CG init, 4 kernels per iteration (direction, operator with p.Ap
    # partials, alpha, gather + r update), final x update
    launches_per_step = 3 + 4 * ITERS + 1

    # ---- dominant kernel: the element operator, timed alone with events (BK5 style) ----
    q = b
    AqL = bp.DeviceBuffer(mesh.NL)
    for _ in range(3):
        bp.ax_hex3d(mesh, q, AqL)
    a0, a1 = ev(), ev()
    bp._check(L.bp_event_record(a0, None))
    for _ in range(args.ax_launches):
        bp.ax_hex3d(mesh, q, AqL)
    bp._check(L.bp_event_record(a1, None))
    bp._check(L.bp_event_elapsed_ms(a0, a1, bp.ctypes.byref(ms)))
    ax_s = ms.value / 1e3 / args.ax_launches
    ax_bytes = ax_model_bytes(Nd, E, Np)
    peak, peak_kind = read_peaks()
    achieved = ax_bytes / ax_s / 1e9
    del AqL

    # ---- end to end through the host-buffer entry point ----
    bh = bp.PinnedBuffer(Nd)
    xh = bp.PinnedBuffer(Nd)
    bh.array[:] = b.download()
    S.solve_host(bh.array, xh.array, 0.0, ITERS)   # warm
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        S.solve_host(bh.array, xh.array, 0.0, ITERS)
    t1 = time.perf_counter()
    barrier(world)
    t_e2e = max_over_ranks(t1 - t0, world)
    e2e = world * Nd * ITERS * args.steps / t_e2e / 1e9

    # ---- time to 1e-8 relative residual: FP64 Jacobi-CG against the mixed solver ----
    mixed = None
    if not args.no_mixed:
        Sm = bp.BP(mesh, precon="JACOBI", precision="MIXED")

        def to_tol(solver):
            bp._check(L.bp_memset(x.ptr, 0, x.nbytes, None))
            bp._check(L.bp_memcpy_dtod(r.ptr, b.ptr, r.nbytes, None))
            st = bp.SolveStats()
            bp._check(L.bp_solver_solve(solver._h, x.ptr, r.ptr, MIXED_TOL, 50000, None, None, bp.ctypes.byref(st)))
            return st

        to_tol(S)
        to_tol(Sm)                                  # warm: graphs captured, caches primed
        barrier(world)
        st64 = to_tol(S)
        stmx = to_tol(Sm)
        t64 = max_over_ranks(st64.elapsed_ms / 1e3, world)
        tmx = max_over_ranks(stmx.elapsed_ms / 1e3, world)
        # FP64 check of the mixed solution's residual
        Ax = bp.DeviceBuffer(Nd)
        S.operator(x, Ax)
        resid = float(np.linalg.norm(b.download() - Ax.download()) / np.linalg.norm(b.download()))
        mixed = {"tolerance": MIXED_TOL,
                 "fp64": {"iterations": st64.iterations, "seconds": t64,
                          "gdof_it_s": world * Nd * st64.iterations / t64 / 1e9,
                          "relative_residual": float(np.sqrt(st64.rdotr / st64.rdotr0))},
                 "mixed": {"iterations": stmx.iterations, "reliable_updates": stmx.updates, "seconds": tmx,
                           "gdof_it_s": world * Nd * stmx.iterations / tmx / 1e9,
                           "relative_residual_fp64_check": resid},
                 "speedup_time_to_solution": t64 / tmx,
                 "speedup_gdof_it_s": (stmx.iterations / tmx) / (st64.iterations / t64)}
        del Sm, Ax

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample, _ = cpu_sample(steps=1, warmup=0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        step_bytes = cg_model_bytes(Nd, E, Np, ITERS)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded LCG forcing f=2u-1 (seed 0) on a seeded perturbed box (seed 1)",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NX, "nz": NX, "p": P, "Ndofs": Nd,
                       "iterations_per_step": ITERS, "precon": "JACOBI", "parallelism": "replicas" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (geometric factors 1.84 GB per step pass)",
                       "final_relative_residual": rel_res},
            "clocks": clk,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * Nd, "d2h_bytes_per_step": 8 * Nd},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "hbm", "kernel": "ax_tma_kernel<NQ=8,NF=1,DOT=0,R=4,double> (bp_ax_hex3d)", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": AX_DRAM_BYTES, "algorithmic_bytes": ax_bytes, "launch_ms": ax_s * 1e3},
            "model_bw_gbs": step_bytes * args.steps / (t_dev / world) / 1e9 if world == 1 else None,
            "cpu_baseline": cpu,
            "mixed_vs_fp64_to_1e-8": mixed,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
