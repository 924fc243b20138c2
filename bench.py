"""Benchmark: BP5 p=7 mixed-precision batched CG against plain FP64 CG, to 1e-8.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one "step"): the BP5 Hex3D problem on a 40x40x40 box with interior
vertices perturbed by 0.1h (seed 1), degree p=7, stored per-node geometric
factors (21,717,639 unknowns), with four right-hand sides b = M f, f = 2u-1
(LCG seeds 0..3), all four solved together by the batched mixed-precision
Jacobi-PCG (FP32 recursion and operator, FP64 reliable updates) from x = 0 to
||b - A x|| <= 1e-8 ||b|| in FP64.  `value` is GDOF*iterations/s of that step
(sum over the four systems of unknowns x iterations, divided by the
device-timed step); inputs are resident in HBM.  `e2e` is the same step with
the four b copied in from pinned host memory and the four x copied back, inside
the timed region.  The comparison the metric names, plain FP64 Jacobi-PCG on
the same problem to the same tolerance, is measured in the same run and
reported under "plain_fp64".

With --gpus N > 1 (launched by torch.distributed.run) every rank solves its
own replica of the problem: the path has no exchange at one rank per problem,
so scaling is weak and no collective is on the data path.

--impl reference times the reference's own algorithm for this path on the
host cores: plain (unpreconditioned) FP64 CG, cg::Solve of
libs/core/linearSolverCG.cpp:62-129 around the bp5AxHex3D operator and the
ogs gather, one right-hand side, restated in C++/OpenMP by the oracle (the
reference's OKL kernels need OCCA, which is absent).  It runs on the same 40^3
mesh and forcing; each step is a bounded sample of 20 CG iterations.

After the headline, the line carries the other configurations of the metric,
each solved once to 1e-8 in mixed precision and (BP3, BP6) in FP64 beside it:
BP3 p=7 over-integrated on the same perturbed box, BP6 p=15 on 24^3 affine
elements with three fields, and the batch of 64 uneven problems
(--no-extras skips them).
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
NRHS, TOL, MAXIT = 4, 1e-8, 20000
WORKLOAD = ("BP5 Hex3D p=7, 40^3 elements, interior vertices perturbed 0.1h (seed 1), stored per-node factors; "
            "4 right-hand sides f=2u-1 (seeds 0..3) solved together by the mixed-precision batched Jacobi-PCG "
            "(FP32 recursion and operator, FP64 reliable updates) to ||b-Ax|| <= 1e-8 ||b||")
# CPU legs (reference arm and cpu_baseline): the reference's plain CG on this
# same mesh and forcing, REF_ITERS iterations per step
REF_ITERS = 20
# The workload's description, identical in both arms' lines
CONFIG = {"workload": WORKLOAD, "nx": NX, "ny": NX, "nz": NX, "p": P, "Ndofs": (NX * P - 1) ** 3, "rhs": NRHS,
          "tolerance": TOL, "perturbation": PERT, "perturbation_seed": PERT_SEED, "forcing_seeds": list(range(NRHS)),
          "l2": "inputs larger than L2 (FP32 factors 0.92 GB read per packed operator apply)"}
B200_SMS = 148
# One launch of the packed FP32 element operator (4 rhs) on this workload,
# captured by ncu at full size (BK5 -nx 40 -ny 40 -nz 40 -p 7 -pt 0.1 -f RANDOM
# -fp MIXED -nr 4, one kernel, one launch): DRAM bytes read + written, and
# shared-memory wavefronts (loads + stores).  The kernel is bound by that
# pipe: one wavefront per SM and clock.
AX_DRAM_BYTES = 1396588800 + 498959616
AX_SMEM_WAVEFRONTS = 141570589
# kernel instantiations of the packed four-system FP32 operator, by autotuner form
AX_KERNELS = {"tma": "ax_tma_kernel<NQ=8,NF=1,DOT=0,R=4,float,Pack<float,4>>",
              "rb": "ax_rb_kernel<NQ=8,L=4,DOT=0>",
              "line": "ax_line_kernel<NQ=8,AFFINE=0,Pack<float,4>>",
              "mma": "ax_mma_pk4_kernel<NQ=8,DOT=0>"}


def ax_model_bytes(Ndofs, E, Np, Nf=1, s=8):
    # reference byte model of one non-affine Ax (BP/BP5/src/bp5Run.cpp:106-142)
    # with s-byte values (8: FP64 as the reference; 4: the FP32 inner operator)
    return Ndofs * s + (Np * 7 * s + 4 + Np * Nf * 4 + Np * Nf * s) * E


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
    """Max of v over the ranks (device times are reported as the slowest rank's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_info():
    """CPU model, physical cores and logical CPUs of this host."""
    model, cores = "unknown", set()
    phys = core = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name":
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
    except OSError:
        pass
    return {"model": model, "physical_cores": len(cores) or os.cpu_count(), "logical_cpus": os.cpu_count()}


def cpu_sample(steps=1, warmup=0):
    """The reference's plain CG (oracle restatement) on this workload's mesh and
    first forcing: REF_ITERS iterations from x = 0 per step, all host threads.
    Returns (GDOF*it/s, threads, sample text, seconds per step)."""
    from oracle import oracle as O
    m = O.Mesh(NX, NX, NX, P, pert=PERT, pert_seed=PERT_SEED)
    _, b = m.rhs_random(RHS_SEED)
    lib = O.lib()
    times = []
    for s in range(warmup + steps):
        x = np.zeros(m.Ngather)
        r = b.copy()
        t0 = time.perf_counter()
        it = lib.bpo_cg(m._h, 1.0, O._dp(x), O._dp(r), 0.0, REF_ITERS, 0, None, None, None)
        t1 = time.perf_counter()
        assert it == REF_ITERS
        if s >= warmup:
            times.append(t1 - t0)
    tot = sum(times)
    v = m.Ngather * REF_ITERS * steps / tot / 1e9
    info = cpu_info()
    sample = ("the reference's cg::Solve (plain FP64 CG, libs/core/linearSolverCG.cpp:62-129) with the bp5AxHex3D "
              "operator and ogs gather, restated in C++/OpenMP by the oracle, on this workload's 40^3 p=7 perturbed "
              "mesh (%d unknowns) and forcing seed %d: %d iterations from x=0 per step, %d threads on %s "
              "(%d physical cores)" % (m.Ngather, RHS_SEED, REF_ITERS, O.num_threads(), info["model"],
                                       info["physical_cores"]))
    return v, O.num_threads(), sample, tot / steps


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    v, cores, sample, sec = cpu_sample(steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
            "reference_algorithm": "plain FP64 CG (the reference's cg::Solve), one right-hand side, %d iterations "
                                   "per step; the reference has no preconditioner, mixed precision or batching"
                                   % REF_ITERS,
            "cpu": cpu_info(),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def solve_pair(bp, mesh, bpn, seed, maxit=20000):
    """One problem to 1e-8 in FP64 and in mixed precision (Jacobi-PCG), each
    after a short warm-up solve that builds its graphs and FP32 data.  Returns
    the result entry with the mixed solution's error against the FP64 one."""
    out, xs = {}, {}
    for prec in ("FP64", "MIXED"):
        S = bp.BP(mesh, bp=bpn, precon="JACOBI", precision=prec)
        b = S.rhs("RANDOM", seed)
        x, r = bp.DeviceBuffer(S.N), bp.DeviceBuffer(S.N)
        for warm in (True, False):
            x.zero()
            bp._check(bp.lib().bp_memcpy_dtod(r.ptr, b.ptr, r.nbytes, None))
            st, _, _ = S.solve(x, r, tol=TOL, maxit=30 if warm else maxit, history=False)
        # FP64 check of the returned solution: ||b - A x|| / ||b||
        bh, Ax = b.download(), bp.DeviceBuffer(S.N)
        S.operator(x, Ax)
        res = float(np.linalg.norm(bh - Ax.download()) / np.linalg.norm(bh))
        xs[prec] = x.download()
        out[prec] = {"iterations": st.iterations, "seconds": st.elapsed_ms / 1e3,
                     "gdof_it_s": S.N * st.iterations / (st.elapsed_ms / 1e3) / 1e9,
                     "fp64_relative_residual": res, "reliable_updates": st.updates}
        del S, b, x, r, Ax
    out["Ndofs"] = int(xs["FP64"].size)
    out["speedup_mixed_vs_fp64"] = out["MIXED"]["gdof_it_s"] / out["FP64"]["gdof_it_s"]
    out["mixed_error_vs_fp64_solution"] = float(np.linalg.norm(xs["MIXED"] - xs["FP64"]) /
                                                np.linalg.norm(xs["FP64"]))
    return out


def bp_problem_ndofs(p):
    """Gathered unknowns of one batch problem (a box of nx*ny*nz elements, degree N)."""
    N, nx = p["N"], p["nx"]
    return (nx * N - 1) * (p.get("ny", nx) * N - 1) * (p.get("nz", nx) * N - 1)


def extra_configs(bp, rank=0, world=1):
    """The metric's other configurations, each solved once (see the module doc)."""
    ex = {}
    m3 = bp.Mesh(NX, NX, NX, N=P, pert=PERT, pert_seed=PERT_SEED)
    ex["BP3_p7_40cubed_curved"] = dict(solve_pair(bp, m3, 3, RHS_SEED), config=(
        "BP3 Hex3D p=7, 9 Gauss points per direction, 40^3 elements perturbed 0.1h (seed 1), factors at the "
        "Gauss points; f=2u-1 (seed 0); Jacobi-PCG to 1e-8"))
    del m3
    m6 = bp.Mesh(24, 24, 24, N=15, affine=True, Nfields=3)
    ex["BP6_p15_24cubed_affine"] = dict(solve_pair(bp, m6, 6, RHS_SEED), config=(
        "BP6 Hex3D p=15, 24^3 affine elements, three fields; f=2u-1 over the gathered rows (seed 0); "
        "Jacobi-PCG to 1e-8"))
    del m6
    # the batch: at N ranks each solves the share that LPT assignment gives it,
    # with no exchange while solving; the results are gathered at the end
    from benchparanumal_b200.shard import batch_solver, solve_sharded
    probs = bp.uneven_problems()
    res, secs, mine = solve_sharded(probs, rank, world, batch_solver(TOL, 20000))
    dofit = sum(r["dof_iterations"] for r in res)
    ex["batch_64_uneven"] = {
        "config": "64 problems, p in 3..10 and n in 8..24 (LCG seed 2), perturbation 0.1h (seeds 100+i), 4 rhs "
                  "each (seeds 1000+4i+k); mixed-precision batched Jacobi-PCG to 1e-8",
        "parallelism": ("1 GPU" if world == 1 else
                        "%d ranks, problems assigned longest-processing-time first, no exchange while solving" % world),
        "systems": sum(p["nrhs"] for p in probs),
        "Ndofs_total": int(sum(bp_problem_ndofs(p) * p["nrhs"] for p in probs)),
        "seconds": secs, "gdof_it_s": dofit / secs / 1e9,
        "problems": [{k: r[k] for k in ("N", "n", "iterations", "max_relative_residual")} for r in res]}
    return ex


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--ax-launches", type=int, default=20)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, world, local = dist_setup(args.gpus)
    import benchparanumal_b200 as bp

    bp.platform_init(local)
    L = bp.lib()
    prob = {"nx": NX, "N": P, "pert": PERT, "pert_seed": PERT_SEED, "nrhs": NRHS, "rhs_seed": RHS_SEED}
    B = bp.Batch([prob], precon="JACOBI", precision="MIXED")
    Nd = B.Ngather[0]
    assert Nd == CONFIG["Ndofs"]

    def ev():
        e = bp.ctypes.c_void_p()
        bp._check(L.bp_event_create(bp.ctypes.byref(e)))
        return e.value

    def step():
        return B.solve(tol=TOL, maxit=MAXIT)[0]

    for _ in range(args.warmup):
        st = step()
    dofit = sum(Nd * s.iterations for s in st)
    rel_res = max(float(np.sqrt(s.rdotr / s.rdotr0)) for s in st)
    launches_per_step = sum(s.kernel_launches for s in st)

    # ---- device-timed region: K steps, inputs resident in HBM ----
    e0, e1 = ev(), ev()
    clocks = ClockSampler(local)
    barrier(world)
    bp.finish()
    clocks.start()
    bp._check(L.bp_event_record(e0, None))
    for _ in range(args.steps):
        st = step()
    bp._check(L.bp_event_record(e1, None))
    bp.finish()
    barrier(world)
    clk = clocks.stop()
    ms = bp.ctypes.c_float()
    bp._check(L.bp_event_elapsed_ms(e0, e1, bp.ctypes.byref(ms)))
    t_dev = max_over_ranks(ms.value / 1e3, world)
    assert sum(Nd * s.iterations for s in st) == dofit
    value = world * dofit * args.steps / t_dev / 1e9

    # ---- end to end: the four b from pinned host memory in, the four x out ----
    bh = [bp.PinnedBuffer(Nd) for _ in range(NRHS)]
    xh = [bp.PinnedBuffer(Nd) for _ in range(NRHS)]
    dev = []
    for k in range(NRHS):
        xp, bptr = bp.ctypes.c_void_p(), bp.ctypes.c_void_p()
        bp._check(L.bp_batch_vectors(B._h, k, bp.ctypes.byref(xp), bp.ctypes.byref(bptr)))
        dev.append((xp.value, bptr.value))
        bh[k].array[:] = B.vectors(k)[1]
    nbytes = 8 * Nd

    def e2e_step():
        for k in range(NRHS):
            bp._check(L.bp_memcpy_htod(dev[k][1], bh[k].array.ctypes.data, nbytes, None))
        B.solve(tol=TOL, maxit=MAXIT)
        for k in range(NRHS):
            bp._check(L.bp_memcpy_dtoh(xh[k].array.ctypes.data, dev[k][0], nbytes, None))
        bp.finish()

    e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    t1 = time.perf_counter()
    barrier(world)
    t_e2e = max_over_ranks(t1 - t0, world)
    e2e = world * dofit * args.steps / t_e2e / 1e9
    # FP64 check of the returned solutions
    Ax = bp.DeviceBuffer(Nd)
    xd = bp.DeviceBuffer(Nd)
    resid = []
    for k in range(NRHS):
        xd.upload(xh[k].array)
        B.operator(k, xd, Ax)
        resid.append(float(np.linalg.norm(bh[k].array - Ax.download()) / np.linalg.norm(bh[k].array)))

    # ---- the comparison: plain FP64 Jacobi-PCG on the same problem and tolerance ----
    mesh = bp.Mesh(NX, NX, NX, N=P, pert=PERT, pert_seed=PERT_SEED)
    S = bp.BP(mesh, precon="JACOBI")
    b0 = S.rhs("RANDOM", RHS_SEED)
    x = bp.DeviceBuffer(Nd)
    r = bp.DeviceBuffer(Nd)

    def fp64_solve(tol, maxit):
        bp._check(L.bp_memset(x.ptr, 0, x.nbytes, None))
        bp._check(L.bp_memcpy_dtod(r.ptr, b0.ptr, r.nbytes, None))
        st = bp.SolveStats()
        bp._check(L.bp_solver_solve(S._h, x.ptr, r.ptr, tol, maxit, None, None, bp.ctypes.byref(st)))
        return st

    fp64_solve(TOL, MAXIT)
    st64 = fp64_solve(TOL, MAXIT)
    t64 = max_over_ranks(st64.elapsed_ms / 1e3, world)
    plain = {"iterations": st64.iterations, "seconds": t64, "gdof_it_s": world * Nd * st64.iterations / t64 / 1e9,
             "relative_residual": float(np.sqrt(st64.rdotr / st64.rdotr0))}
    # and the reference's own step, exactly 100 FP64 iterations (bp5Run.cpp:71-95)
    fp64_solve(0.0, ITERS)
    st100 = fp64_solve(0.0, ITERS)
    plain["fixed_100_iterations_gdof_it_s"] = world * Nd * ITERS / (st100.elapsed_ms / 1e3) / 1e9

    # ---- dominant kernel of the step: the packed FP32 element operator on the four
    # right-hand sides (what each iteration of the batched solve launches), timed
    # alone; beside it the same operator with the CG direction update fused in
    # (bp_cg_direction_ax_f32_multi, opt-in in the solver: slower, measured) ----
    v = mesh.view
    ng = mesh.E * mesh.Np
    ops = {"wJ": bp.DeviceBuffer(ng, np.float32), "ggeo": bp.DeviceBuffer(6 * ng, np.float32),
           "gllw": bp.DeviceBuffer(mesh.Nq, np.float32), "D": bp.DeviceBuffer(mesh.Nq * mesh.Nq, np.float32)}
    for name, n in (("wJ", ng), ("ggeo", 6 * ng), ("gllw", mesh.Nq), ("D", mesh.Nq * mesh.Nq)):
        bp.convert_f64_f32(getattr(v, name), n, ops[name])
    b32 = bp.DeviceBuffer(Nd, np.float32)
    bp.convert_f64_f32(b0, Nd, b32)
    packed = np.repeat(b32.download(), NRHS)   # interleaved: row r, system k at r*NRHS + k
    vec = {k: bp.DeviceBuffer.from_host(packed) for k in ("r", "p0", "p1", "x")}
    invD32 = bp.DeviceBuffer.from_host(np.full(Nd, 0.5, np.float32))
    own = bp.DeviceBuffer(mesh.NL, np.int32)
    bp.ogs_owner_map(mesh, own)
    parts = bp.DeviceBuffer((mesh.E + 1) * NRHS)
    AqL = bp.DeviceBuffer(mesh.NL * NRHS, np.float32)
    coef_a, coef_b = [1e-3] * NRHS, [0.5] * NRHS

    def fused():
        bp.cg_direction_ax_f32_multi(mesh, NRHS, own, ops, coef_a, coef_b, vec["r"], invD32, vec["p0"], vec["p1"],
                                     vec["x"], AqL, parts)

    def timed(fn):
        for _ in range(3):
            fn()
        a0, a1 = ev(), ev()
        bp._check(L.bp_event_record(a0, None))
        for _ in range(args.ax_launches):
            fn()
        bp._check(L.bp_event_record(a1, None))
        bp._check(L.bp_event_elapsed_ms(a0, a1, bp.ctypes.byref(ms)))
        return ms.value / 1e3 / args.ax_launches

    fused_s = timed(fused)
    ax_s = timed(lambda: bp.ax_hex3d_f32_multi(mesh, NRHS, vec["p1"], AqL, ops))
    # the form the autotuner chose for this launch (packed FP32 group, not fused)
    ax_form = bp.tune_report(1, P, 1, False, 4, NRHS, 0, mesh.E)[0]
    E, Np = mesh.E, mesh.Np
    # reference model of the operator with 4-byte values, the q and Aq terms once per
    # right-hand side; the fused step adds the direction update's vectors: r, x
    # (read and write) and the new p per system, invD once
    ax_bytes = ax_model_bytes(Nd, E, Np, s=4) + (NRHS - 1) * (Nd * 4 + E * Np * 4)
    fused_bytes = ax_bytes + NRHS * Nd * 4 * 4 + Nd * 4
    peak, peak_kind = read_peaks()
    achieved = ax_bytes / ax_s / 1e9
    smem_mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    smem_bound_ms = AX_SMEM_WAVEFRONTS / (B200_SMS * smem_mhz * 1e6) * 1e3
    del AqL, ops, vec, invD32, own, parts, b32

    # free the headline's buffers before the other configurations
    del S, b0, x, r, Ax, xd, mesh, B
    extras = None
    if not args.no_extras:
        extras = extra_configs(bp, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, cores, sample, _ = cpu_sample(steps=1, warmup=0)
        cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner / f64 refinement",
            "data": "synthetic: seeded LCG forcing f=2u-1 (seeds 0..3) on a seeded perturbed box (seed 1)",
            "config": CONFIG,
            "results": {"iterations_per_system": [s.iterations for s in st],
                        "reliable_updates_per_system": [s.updates for s in st],
                        "final_relative_residual_max": rel_res,
                        "fp64_check_relative_residual": resid,
                        "parallelism": "replicas" if world > 1 else "1 GPU"},
            "clocks": clk,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": NRHS * 8 * Nd,
                    "d2h_bytes_per_step": NRHS * 8 * Nd},
            "gpu_launches": launches_per_step * args.steps,
            "plain_fp64": plain,
            "speedup_vs_plain_fp64": value / plain["gdof_it_s"],
            "roofline": {"bound": "hbm",
                         "kernel": AX_KERNELS.get(ax_form, str(ax_form)) + " (bp_ax_hex3d_f32_multi, 4 rhs)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "algorithmic_bytes": ax_bytes,
                         # DRAM bytes and wavefronts were captured with ncu on the TMA form
                         "traffic": AX_DRAM_BYTES if ax_form == "tma" else None,
                         "launch_ms": ax_s * 1e3,
                         "fused_direction_step": {"kernel": "bp_cg_direction_ax_f32_multi (4 rhs)",
                                                  "launch_ms": fused_s * 1e3, "algorithmic_bytes": fused_bytes,
                                                  "achieved": fused_bytes / fused_s / 1e9},
                         # the roof that binds this kernel: shared-memory wavefronts at one per SM and clock
                         # (clock: the median SM clock sampled during the timed step, else the maximum)
                         "smem": {"wavefronts": AX_SMEM_WAVEFRONTS, "sm_mhz": smem_mhz,
                                  "bound_ms": smem_bound_ms, "frac": smem_bound_ms / (ax_s * 1e3)}
                         if ax_form == "tma" else None},
            "cpu_baseline": cpu,
            "cpu": cpu_info(),
            "configs": extras,
        }
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
