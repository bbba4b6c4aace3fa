#!/usr/bin/env python
"""KKT LDL^T factor+solve throughput on B200.

Workload: the 256 x 256 plane-stress PDE-constrained KKT system
(amigo_b200.workloads.plane_stress_kkt: n = 329,732, 6.09e6 nonzeros, five
right-hand sides: a unit load plus four N(0,1) columns), AMD ordering, the
reference solver's settings (ustab 0.01, pivot_tol 1e-14). One step = one
numeric factorization + one 5-RHS solve; the symbolic analysis runs once per
pattern outside the timed region, as in the interior-point loop. The timed
factorizations reuse the pivot order recorded at a neighbouring iterate (the
same pattern with perturbed values; SparseLDL.reuse_pivot_order); the line
also reports the first factorization's order (the reference's pivot sequence
replayed) and a record taken from the benchmark values themselves.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). With N > 1 (torchrun) every rank factors its
own replica (a single factorization does not shard), value = all ranks'
steps / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "KKT LDLᵀ factor+solve/s at 1e-10 backward err: mixed-prec vs FP64, 1 B200"
UNIT = "factor+solve/s"
BERR_TARGET = 1e-10
L2_BYTES = 126 * 1024 * 1024
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def host_info() -> dict:
    """The host the CPU baseline ran on: CPU model, logical cores, and the
    BLAS the compiled reference links (OpenBLAS from the image's opencv
    wheel, see oracle/Makefile)."""
    cpu = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    cpu = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu": cpu, "nproc": os.cpu_count() or 1,
            "blas": "OpenBLAS 0.3.15 (LP64, opencv-python-headless wheel)"}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "source": "measured"}
    except Exception:
        return dict(FALLBACK_PEAKS, source="fallback")


class ClockSampler:
    """nvidia-smi sampling during the timed region (median SM clock and the
    throttle reasons seen)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, enabled: bool = True):
        self.enabled = enabled
        self.idx = device_index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        if not self.enabled:
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.enabled:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"]}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t is not None:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def backward_error(system, x, b) -> float:
    r = b - system.matvec(x)
    kn = system.inf_norm()
    num = np.abs(r).max(axis=0)
    den = kn * np.abs(x).max(axis=0) + np.abs(b).max(axis=0)
    return float(np.max(num / den))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_sample(system, threads: int, budget_s: float, max_steps: int, warmup: int):
    """Time the reference's own SparseLDL (compiled from its sources into
    oracle/_ref) on the host: factor + 5-RHS solve of the same system."""
    from oracle import ref

    env_threads = str(threads)
    os.environ["OMP_NUM_THREADS"] = env_threads
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    r = ref.RefLDL(system.rowp, system.cols, order=ref.ORDER_AMD, openmp=threads > 1)
    for _ in range(warmup):
        r.factor(system.vals, system.diag)
        r.solve(system.rhs)
    times = []
    t_all = time.perf_counter()
    x = None
    while len(times) < max_steps:
        t0 = time.perf_counter()
        r.factor(system.vals, system.diag)
        x = r.solve(system.rhs)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s:
            break
    inertia = r.inertia()
    r.close()
    return times, inertia, x


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU SparseLDL with all host threads."""
    if rank != 0:
        return 0
    from amigo_b200.workloads import plane_stress_kkt
    from oracle import ref

    if not ref.available(openmp=True):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/liboracle_ref_omp.so not built"}))
        return 0
    s = plane_stress_kkt(args.nel)
    cores = os.cpu_count() or 1
    budget = float(os.environ.get("REFERENCE_BUDGET_S", "150"))
    times, inertia, x = cpu_reference_sample(s, cores, budget, args.steps, min(args.warmup, 1))
    ms = 1e3 * float(np.mean(times))
    value = 1e3 / ms
    sample = (f"{len(times)} of {args.steps} requested factor+5-RHS solves of the full "
              f"system (time budget {budget:.0f} s), after {min(args.warmup, 1)} warm-up")
    berr = backward_error(s, x, s.rhs)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": len(times), "warmup": min(args.warmup, 1),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"plane-stress KKT {args.nel}x{args.nel} (n={s.n}, nnz={s.nnz}), "
                               "5 RHS, AMD", "nrhs": 5, "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "host": host_info(),
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "inertia": list(inertia), "backward_error": berr,
    }
    print(json.dumps(line))
    return 0


def run_reference_batched(args, world, rank):
    """The reference arm of the batched workload: one serial SparseLDL per
    system, the systems spread over all host cores by a thread pool (the
    compiled reference releases the interpreter lock while it factors).
    Each step factors and solves a bounded sample of the batch, the time
    scaled to the whole batch."""
    if rank != 0:
        return 0
    from concurrent.futures import ThreadPoolExecutor

    from amigo_b200.workloads import batched_optimal_control
    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/liboracle_ref.so not built"}))
        return 0
    # one thread per system: BLAS inside each call stays single-threaded
    # (read when the library is first loaded in this process)
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    systems = batched_optimal_control(num_systems=args.systems, seed=0)
    cores = os.cpu_count() or 1
    handles = [ref.RefLDL(q.rowp, q.cols, order=ref.ORDER_AMD) for q in systems]

    def one(i):
        q = systems[i]
        handles[i].factor(q.vals, q.diag)
        return i, handles[i].solve(q.rhs[:, :1]), handles[i].inertia()

    budget = float(os.environ.get("REFERENCE_BUDGET_S", "60"))
    per_step = max(1, budget / max(1, args.steps + 1))
    times, results = [], {}
    with ThreadPoolExecutor(max_workers=cores) as pool:
        for step in range(args.steps + 1):  # the first pass is the warm-up
            t0 = time.perf_counter()
            done = 0
            futs = [pool.submit(one, i) for i in range(len(systems))]
            for f in futs:
                i, x, inertia = f.result()
                results[i] = (x, inertia)
                done += 1
                if time.perf_counter() - t0 > per_step:
                    break
            for f in futs:
                f.cancel()
            while any(not f.done() for f in futs):
                time.sleep(0.001)
            if step > 0:
                times.append((time.perf_counter() - t0) / done * len(systems))
    ms = 1e3 * float(np.mean(times))
    value = 1e3 / ms
    berr = max(backward_error(systems[i], x, systems[i].rhs[:, :1])
               for i, (x, _) in results.items())
    ok = all(tuple(inertia) == systems[i].expected_inertia
             for i, (_, inertia) in results.items())
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "batch factor+solve/s",
        "n_gpus": world, "steps": len(times), "warmup": 1, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{len(systems)} independent optimal-control KKT systems, "
                               "one RHS each, AMD, FP64",
                   "parallelism": f"one system per host thread, {cores} threads"},
        "cpu_baseline": {"value": value, "unit": "batch factor+solve/s", "cores": cores,
                         "kind": "reference", "host": host_info(),
                         "sample": f"systems completed within {per_step:.0f} s per step, "
                                   "scaled to the batch"},
        "e2e": {"value": value, "unit": "batch factor+solve/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "backward_error": berr, "inertia_all_expected": ok,
    }
    print(json.dumps(line))
    return 0


def perturbed_iterate(system, seed: int = 123, eps_vals: float = 0.01, eps_sigma: float = 0.3):
    """Values of the same pattern standing for a neighbouring interior-point
    iterate: every stored entry scaled by 1 + eps_vals N(0,1) (the same
    factor for (i, j) and (j, i), so the matrix stays symmetric) and every
    positive diagonal entry (Sigma) by exp(eps_sigma N(0,1))."""
    rng = np.random.default_rng(seed)
    r = np.repeat(np.arange(system.n), np.diff(system.rowp))
    key = r.astype(np.int64) * system.n + system.cols
    tkey = system.cols.astype(np.int64) * system.n + r
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], tkey)]
    f = rng.standard_normal(system.nnz)
    f = 0.5 * (f + f[pos])
    v = system.vals * (1.0 + eps_vals * f)
    d = system.diag.copy()
    m = d > 0
    d[m] *= np.exp(eps_sigma * rng.standard_normal(int(m.sum())))
    return v, d


def measure_batched(args, dev):
    """The batched workload beside the headline: 512 optimal-control systems
    (N ~ U{50..400}, nx = 6, nu = 3, one RHS each) in one handle; one step
    = factor + solve of all of them, device-resident inputs, CUDA events."""
    import torch

    from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDLBatch, Vector
    from amigo_b200.workloads import batched_optimal_control

    systems = batched_optimal_control(num_systems=512, seed=0)
    mats = [CSRMat(q.n, q.n, q.rowp, q.cols, torch.as_tensor(q.vals, device=dev))
            for q in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    diag = Vector(torch.as_tensor(np.concatenate([q.diag for q in systems]), device=dev))
    b = torch.as_tensor(np.concatenate([q.rhs[:, 0] for q in systems]), device=dev)
    x = torch.empty_like(b)

    def step():
        batch.factor(diag)
        x.copy_(b)
        batch.solve(x)

    for _ in range(args.warmup):
        step()
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = batch.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (batch.launch_count() - launches0) / args.steps
    xh = x.cpu().numpy()
    berr = max(backward_error(q, xs.reshape(-1, 1), q.rhs[:, :1])
               for q, xs in zip(systems, batch.split(xh)))
    ok = all(tuple(int(v) for v in i) == q.expected_inertia
             for i, q in zip(batch.system_inertia(), systems))
    batch.close()
    return {"value": 1e3 / ms, "unit": "batch factor+solve/s", "ms_per_step": ms,
            "systems": len(systems), "n_total": int(sum(q.n for q in systems)),
            "gpu_launches_per_step": launches, "backward_error": berr,
            "inertia_all_expected": bool(ok),
            "what": "512 optimal-control systems, N ~ U{50..400}, nx 6, nu 3, one RHS each, "
                    "AMD, FP64, one batch handle; level-scheduled launches"}


def run_ours(args, world, rank, local):
    import torch

    from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDL, Vector
    from amigo_b200.workloads import plane_stress_kkt

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    s = plane_stress_kkt(args.nel)
    nrhs = s.rhs.shape[1]
    vals = torch.as_tensor(s.vals, device=dev)
    diag = torch.as_tensor(s.diag, device=dev)
    b = torch.as_tensor(np.ascontiguousarray(s.rhs.T), device=dev).t()  # column-major
    x = torch.empty_like(b)
    x = x.t().contiguous().t()
    ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, vals), order=OrderingType.AMD)
    dvec = Vector(diag)
    stream = torch.cuda.current_stream(dev)

    def step():
        ldl.factor(dvec)
        x.copy_(b)
        ldl.solve(x)

    def timed(k):
        """K steps between CUDA events on the launching stream, the ranks
        lined up by a barrier; device milliseconds, max over ranks."""
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    ref_order = same_values = None
    if not args.headline_only:
        # (1) the reference's pivot order: every factorization starts from
        # the symbolic supernodes and replays the reference's delays
        for _ in range(args.warmup):
            step()
        ms_ref_order = timed(args.steps)
        ref_order = {
            "value": world * args.steps / (ms_ref_order / 1e3),
            "ms_per_step": ms_ref_order / args.steps,
            "backward_error": backward_error(s, x.cpu().numpy(), s.rhs),
            "delayed_pivots": ldl.stats()["delayed"],
            "what": "every factorization from the symbolic supernodes, the reference's "
                    "pivot sequence replayed (the first factorization of a pattern)"}

        # (2) the record of a factorization of these very values: the
        # fastest case of pivot-order reuse (every recorded pivot passes)
        ldl.factor(dvec)
        ldl.reuse_pivot_order()
        for _ in range(args.warmup):
            step()
        ms_same = timed(args.steps)
        same_values = {
            "value": world * args.steps / (ms_same / 1e3),
            "ms_per_step": ms_same / args.steps,
            "backward_error": backward_error(s, x.cpu().numpy(), s.rhs),
            "delayed_pivots": ldl.stats()["delayed"],
            "what": "record taken from a factorization of the benchmark matrix itself (the "
                    "best case of reuse, e.g. inertia-correction refactorizations)"}

    # (3) the headline: the pivot order recorded at a neighbouring
    # interior-point iterate (the same pattern, other values), as a
    # refactorization loop that calls reuse_pivot_order after a factorization
    # and then factors the next iterate's matrix
    pv, pd = perturbed_iterate(s)
    ldl.set_pivot_record(None)
    vals.copy_(torch.as_tensor(pv, device=dev))
    diag.copy_(torch.as_tensor(pd, device=dev))
    ldl.factor(dvec)
    ldl.reuse_pivot_order()
    vals.copy_(torch.as_tensor(s.vals, device=dev))
    diag.copy_(torch.as_tensor(s.diag, device=dev))
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local, enabled=not args.no_clocks)
    launches0 = ldl.launch_count()
    sampler.start()
    ms_total = timed(args.steps)
    clocks = sampler.stop()
    launches = ldl.launch_count() - launches0
    ms_max = ms_total
    # accuracy and work of the last timed step
    xh = x.cpu().numpy()
    berr = backward_error(s, xh, s.rhs)
    inertia = ldl.get_inertia()
    stats = ldl.stats()
    work = ldl.work()
    # kernel-class times for the roofline: the same K steps again with the
    # library's per-class CUDA events on (they add host work between
    # launches, so the headline value above is timed without them)
    prof = None
    if not args.no_profile_pass:
        ldl.set_profiling(True)
        ldl.reset_profile()
        for _ in range(args.steps):
            step()
        torch.cuda.synchronize()
        prof = ldl.profile()
        ldl.set_profiling(False)
    value = world * args.steps / (ms_max / 1e3)

    # (4) mixed precision on the headline's pivot order: contribution-block tiles on
    # the tensor cores, FP64-refined solves, FP64 redo when the inertia
    # differs from the FP64 factorization's or the refinement stalls
    mixed = None
    if not args.no_mixed:
        ldl.set_precision("mixed", refine_iters=5, refine_tol=BERR_TARGET)
        for _ in range(args.warmup):
            step()
        redo0 = ldl.last_refinement()["fp64_redos"]
        ms_mixed = timed(args.steps)
        info = ldl.last_refinement()
        berr_mixed = backward_error(s, x.cpu().numpy(), s.rhs)
        mixed = {
            "value": world * args.steps / (ms_mixed / 1e3),
            "ms_per_step": ms_mixed / args.steps, "backward_error": berr_mixed,
            "berr_target_met": bool(berr_mixed <= BERR_TARGET),
            "inertia": list(ldl.get_inertia()),
            "fp64_redos_in_timed_steps": info["fp64_redos"] - redo0,
            "refinement_iterations": info["iterations"],
            "vs_fp64_same_pivot_order": ms_max / ms_mixed,
            "what": "contribution-block tiles of the big fronts' trailing updates as 3xTF32 on "
                    "tcgen05 (FP32 accumulation in tensor memory), solves refined in FP64 to "
                    "1e-10; a factorization whose inertia differs from the FP64 one is redone "
                    "in FP64 (on this KKT family FP32-level rounding flips tiny pivots)"}
        ldl.set_precision("fp64")

    # the batched workload beside the headline (one GPU)
    batched = None
    if world == 1 and not (args.no_batched or args.headline_only):
        ldl.close()
        torch.cuda.empty_cache()
        batched = measure_batched(args, dev)

    # end to end through the public API with host buffers (pinned), the same
    # reuse of the previous factorization's pivot order (the device-buffer
    # handle is released first: each holds the factor pools of this system)
    ldl.close()
    torch.cuda.empty_cache()
    e2e_value, berr_e2e = None, None
    hv = torch.empty(s.nnz, dtype=torch.float64, pin_memory=True)
    hd = torch.empty(s.n, dtype=torch.float64, pin_memory=True)
    hx = torch.empty((nrhs, s.n), dtype=torch.float64, pin_memory=True)
    hv.numpy()[:] = s.vals
    hd.numpy()[:] = s.diag
    host_ldl = SparseLDL(CSRMat(s.n, s.n, s.rowp, s.cols, hv.numpy()), order=OrderingType.AMD)
    hvec = Vector(hd.numpy())
    xf = hx.numpy().T  # n x nrhs, column-major view of pinned memory

    def e2e_step():
        host_ldl.factor(hvec)
        xf[...] = s.rhs
        host_ldl.solve(xf)

    if not args.no_e2e:
        # the same pivot order as the headline: recorded at the neighbouring
        # iterate's values, then the benchmark values
        hv.numpy()[:] = pv
        hd.numpy()[:] = pd
        host_ldl.factor(hvec)
        host_ldl.reuse_pivot_order()
        hv.numpy()[:] = s.vals
        hd.numpy()[:] = s.diag
        for _ in range(max(1, min(args.warmup, 2))):
            e2e_step()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1e3
        te = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        if world > 1:
            torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
        e2e_value = world * args.steps / (float(te.item()) / 1e3)
        berr_e2e = backward_error(s, np.array(xf), s.rhs)
    h2d = (s.nnz + s.n + s.n * nrhs) * 8
    d2h = s.n * nrhs * 8
    host_ldl.close()

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    # roofline of the dominant kernel class: device time from CUDA events the
    # library records on its stream around each class over the timed region;
    # algorithmic work per step from the factorization's own counters
    peaks = load_peaks()
    roof = None
    algo = {
        # dense partial factorizations outside the big-front path (flops)
        "fronts": ("tensor", work["flops"] - work["panel_flops"] - work["update_flops"]
                   - work["cluster_flops"]),
        # big fronts: panels and their trailing updates (flops; with pivot
        # reuse one cooperative launch per level does both)
        "big_panel": ("tensor", work["panel_flops"] + work["update_flops"]),
        # whole fronts factored in a cluster's distributed shared memory
        "cluster_fronts": ("tensor", work["cluster_flops"]),
        # rank-kw updates: trailing lower triangle read + written, panels read
        "big_update": ("hbm", work["update_bytes"]),
        # contribution blocks read into the fronts (bytes)
        "big_assembly": ("hbm", stats["cb_bytes"]),
        # every factor entry read once per sweep, plus the update vectors
        "solve_forward": ("hbm", stats["L_bytes"]),
        "solve_backward": ("hbm", stats["L_bytes"]),
    }
    for p_ in prof or []:
        p_["bound"], w = algo[p_["name"]]
        p_["work_per_step"] = w
    dom = max(prof, key=lambda p_: p_["ms"]) if prof else None
    fp64_peak_tflops = 37.0  # B200 datasheet FP64 (no FP64 peak is measured on this pool)
    if dom is not None:
        per_launch_ms = dom["ms"] / max(1, dom["launches"])
        total_work = dom["work_per_step"] * args.steps
        if dom["bound"] == "hbm":
            achieved = total_work / max(1e-12, dom["ms"] / 1e3) / 1e9
            roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None}
        else:
            achieved = total_work / max(1e-12, dom["ms"] / 1e3) / 1e12
            roof = {"bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"],
                    "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops"],
                    "traffic": None,
                    "fp64_frac": achieved / fp64_peak_tflops,
                    "note": "FP64 arithmetic: frac is against the bf16 dense peak the "
                            "contract names; fp64_frac against the B200 datasheet FP64 "
                            "peak (37 TFLOP/s, not measured here)"}
        roof.update({"kernel": dom["name"], "launches": dom["launches"],
                     "ms_per_launch": per_launch_ms, "peak_source": peaks["source"],
                     "traffic_note": "null: the dominant class is one cooperative launch per "
                                     "tree level; its full ncu capture (128x128, "
                                     "profiles/app_level_kernel_plane_stress_128.txt) is "
                                     "L2-resident, 6.7 MB DRAM read per level launch, so no "
                                     "full-size DRAM figure is scaled from it",
                     "timing": "profile pass of the same steps, CUDA events per kernel class"})

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import ref

        if ref.available():
            times, cinertia, _ = cpu_reference_sample(s, 1, 30.0, 1, 0)
            cms = 1e3 * float(np.mean(times))
            cpu = {"value": 1e3 / cms, "unit": UNIT, "cores": 1, "kind": "reference", "host": host_info(),
                   "sample": f"{len(times)} factor+5-RHS solve of the full system, serial "
                             "build, OPENBLAS_NUM_THREADS=1",
                   "inertia": list(cinertia)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {
            "workload": f"plane-stress KKT {args.nel}x{args.nel} (n={s.n}, nnz={s.nnz}), "
                        f"{nrhs} RHS, AMD ordering, FP64 factor+solve",
            "nrhs": nrhs, "parallelism": "replicas" if world > 1 else "single GPU",
            "pivot_order": "recorded at a neighbouring interior-point iterate (the same "
                           "pattern; entries scaled by 1 + 0.01 N(0,1), Sigma by "
                           "exp(0.3 N(0,1))) and reused for the benchmark matrix "
                           "(SparseLDL.reuse_pivot_order, as a refactorization loop does); "
                           "every candidate is still tested against its whole column and "
                           "delayed when it fails",
            "l2": "inputs and per-step factor traffic larger than L2 (126 MB); no flush",
        },
        "fp64_reference_order": ref_order,
        "pivot_record_from_same_values": same_values,
        "mixed_precision": mixed,
        "batched_workload": batched,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "backward_error": berr_e2e},
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "backward_error": berr,
        "berr_target_met": bool(berr <= BERR_TARGET),
        "inertia": list(inertia),
        "expected_inertia": list(s.expected_inertia),
        "factor_flops_executed": stats["flops"],
        "max_front": stats["max_front"],
        "delayed_pivots": stats["delayed"],
        "a_posteriori_panels": {k: work[k] for k in ("app_panels", "app_rejected",
                                                     "app_block_delays")},
        "profile": prof,
    }
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_batched(args, world, rank, local):
    """Secondary workload: many independent optimal-control KKT systems of
    uneven size (N ~ U{50..400}, nx = 6, nu = 3, one RHS each), factored and
    solved together in one handle. One step = factor + solve of all systems.
    With N ranks the batch is split by system over the GPUs (balanced by
    size, amigo_b200.shard), no exchange on the data path, and the step time
    is the slowest rank's (strong scaling of one batch). Not the headline
    metric; printed in the same JSON shape."""
    import torch

    from amigo_b200.shard import gather_by_system, shard_systems
    from amigo_b200.sparse_ldl import CSRMat, OrderingType, SparseLDLBatch, Vector
    from amigo_b200.workloads import batched_optimal_control

    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    all_systems = batched_optimal_control(num_systems=args.systems, seed=0)
    idx, systems = shard_systems(all_systems, rank, world)
    mats = [CSRMat(q.n, q.n, q.rowp, q.cols, torch.as_tensor(q.vals, device=dev))
            for q in systems]
    batch = SparseLDLBatch(mats, order=OrderingType.AMD)
    diag = Vector(torch.as_tensor(np.concatenate([q.diag for q in systems]), device=dev))
    bh = np.concatenate([q.rhs[:, 0] for q in systems])
    b = torch.as_tensor(bh, device=dev)
    x = torch.empty_like(b)

    def step():
        batch.factor(diag)
        x.copy_(b)
        batch.solve(x)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = batch.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t = torch.tensor([e0.elapsed_time(e1) / args.steps], device=dev, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = float(t.item())
    launches = batch.launch_count() - launches0
    xh = x.cpu().numpy()
    berrs = [backward_error(q, xs.reshape(-1, 1), q.rhs[:, :1])
             for q, xs in zip(systems, batch.split(xh))]
    inertias = [tuple(int(v) for v in i) for i in batch.system_inertia()]
    # per-system results of every rank, in the batch's order (host gather)
    results = gather_by_system(list(zip(inertias, berrs)), idx, len(all_systems))
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    berr = max(r[1] for r in results)
    ok = all(r[0] == q.expected_inertia for r, q in zip(results, all_systems))
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        from oracle import ref

        if ref.available():
            # serial reference, one system after another, on a bounded sample
            t_all, done, n_done = time.perf_counter(), 0.0, 0
            for q in all_systems:
                r = ref.RefLDL(q.rowp, q.cols, order=ref.ORDER_AMD)
                t0 = time.perf_counter()
                r.factor(q.vals, q.diag)
                r.solve(q.rhs[:, :1])
                done += time.perf_counter() - t0
                r.close()
                n_done += 1
                if time.perf_counter() - t_all > 20.0:
                    break
            per_batch = done / n_done * len(all_systems)
            cpu = {"value": 1.0 / per_batch, "unit": "batch factor+solve/s", "cores": 1,
                   "kind": "reference", "host": host_info(),
                   "sample": f"{n_done} of {len(all_systems)} systems, serial, scaled to the batch"}
    n_total = sum(q.n for q in all_systems)
    line = {
        "metric": METRIC, "value": 1e3 / ms, "unit": "batch factor+solve/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(all_systems)} independent optimal-control KKT systems "
                               f"(n total {n_total}), one RHS each, AMD, FP64",
                   "parallelism": f"systems split over {world} GPUs" if world > 1
                   else "single GPU, one handle",
                   "systems_per_s": len(all_systems) * 1e3 / ms},
        "cpu_baseline": cpu, "gpu_launches": launches, "backward_error": berr,
        "berr_target_met": bool(berr <= BERR_TARGET), "inertia_all_expected": ok,
    }
    print(json.dumps(line))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nel", type=int, default=256, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    # a single factor+solve for profiler launch lists
    ap.add_argument("--no-e2e", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-profile-pass", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-clocks", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-mixed", action="store_true", help=argparse.SUPPRESS)
    # profiling runs: only the headline's pivot order (no reference-order and
    # same-values arms, no batched workload)
    ap.add_argument("--headline-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-batched", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--workload", choices=["plane_stress", "batched"], default="plane_stress",
                    help=argparse.SUPPRESS)
    ap.add_argument("--systems", type=int, default=512, help=argparse.SUPPRESS)
    args = ap.parse_args(argv)
    world, rank, local = dist_setup()
    if args.workload == "batched":
        if args.impl == "reference":
            return run_reference_batched(args, world, rank)
        return run_batched(args, world, rank, local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
