"""Benchmark of the FP64 FR residual (rhs_func) on the large blast workload.

Workload: 2D radial blast on [0,1]^2, 1024 x 1024 quads, GLL p = 5 (36 points per
element), HLLC, Van der Waals gas (a = 0.05, b = 0.02, gamma = 1.4): 37,748,736
nodes, 150,994,944 DOF, a 1.21 GB FP64 state (larger than the 126 MB L2, so no
flush is needed between steps).  One step = one rhs = -R(U) over the whole mesh.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one process per GPU, each rank on its own replica of
the workload (weak scaling); rank 0 prints one JSON line.  --impl reference
times the reference's own residual code (fr_sdg's include/*.hpp built into
oracle/_ref) on the same mesh on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DOF-residuals/s (FP64 FR residual, rhs_func)"
UNIT = "DOF-residuals/s"
WORKLOAD = ("blast_vdw_1024x1024_p5 (2D radial blast, HLLC, Van der Waals a=0.05 b=0.02, spectral filter with "
            "the shock sensor)")


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), for the CPU-baseline record."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Nominal dense FP64 rate of a B200 (vector and tensor pipes alike); the measured FP64
# denominator is a DGEMM timed by the bench itself (dgemm_tflops).
FP64_NOMINAL_TFLOPS = 37.0


def dgemm_tflops(device, n: int = 8192, reps: int = 5) -> float:
    """FP64 matrix-multiply rate of this GPU (cuBLAS DGEMM through torch.mm, n x n,
    CUDA events): the measured FP64 denominator beside the nominal one."""
    import torch

    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    c = torch.mm(a, b)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.mm(a, b, out=c)
    e1.record()
    torch.cuda.synchronize()
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 * reps / (e0.elapsed_time(e1) / 1e3) / 1e12


def flops_per_full_launch():
    """Operations of one 1024^2 residual of the workload, counted on the reference
    algorithm (oracle/count_flops.py -> profiles/fr2d_kernel_blast_flops.txt)."""
    f = Path(__file__).resolve().parent / "profiles" / "fr2d_kernel_blast_flops.txt"
    try:
        for line in f.read_text().splitlines():
            if line.startswith("flops_per_full_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def traffic_per_launch():
    """DRAM bytes per launch of the residual kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "fr2d_kernel_blast_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_full_launch:"):
            return float(line.split(":", 1)[1].strip())
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 25 ms during the timed
    region: the sampler is started and has delivered a first sample before the region
    begins; only samples stamped inside the region count (the first one after it when
    the region is shorter than the interval)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, interval_ms: int = 25):
        self.gpu = gpu_index
        self.interval_ms = interval_ms
        self.proc = None
        self.samples = []
        self.t0 = self.t1 = None

    def _reader(self):
        for line in self.proc.stdout:
            if line.strip():
                self.samples.append((time.monotonic(), line))

    def __enter__(self):
        import threading

        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._reader, daemon=True)
            self.thread.start()
            deadline = time.monotonic() + 10.0
            while not self.samples and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def __exit__(self, *exc):
        self.t1 = time.monotonic()
        if self.proc:
            # one more sample after the region, for regions shorter than the interval
            deadline = time.monotonic() + 1.0
            n = len(self.samples)
            while len(self.samples) == n and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)
        inside = [l for t, l in self.samples if self.t0 <= t <= self.t1]
        if not inside:
            inside = [l for t, l in self.samples if t > self.t1][:1]
        self.lines = inside

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_residual_rate(threads: int, target_s: float = 3.0, rows: int = 64, max_reps: int = 20):
    """Oracle (CPU restatement) residual rate on a bounded sample of the workload:
    a 1024 x `rows` element strip of the same mesh spacing and state."""
    import numpy as np

    from fr_sdg_b200.workloads import blast_large
    from oracle.oracle import Oracle

    wl = blast_large()
    cfg = wl.cfg
    full = wl.init("cpu").numpy()
    n = cfg.poly_deg + 1
    per_row = cfg.n_elems[0] * n * n * 4
    j0 = cfg.n_elems[1] // 2 - rows // 2
    U = np.ascontiguousarray(full[j0 * per_row:(j0 + rows) * per_row])
    del full
    cfg.n_elems[1] = rows
    cfg.box_length[1] = rows / 1024.0
    o = Oracle(cfg, threads=threads)
    o.residual(0.0, U)  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        o.residual(0.0, U)
        reps += 1
        el = time.perf_counter() - t0
        if el >= target_s or reps >= max_reps:
            break
    dofs = U.size
    return dofs * reps / el, {"sample": f"{reps} residual(s) of a 1024x{rows}-element strip of the workload "
                                        f"({dofs} DOF each), {el:.1f} s wall",
                              "cores": threads}


def repo_libraries_loaded() -> list[str]:
    """Shared libraries of this repository mapped into the process (Linux)."""
    out = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            path = line.split()[-1] if line.strip() else ""
            if path.endswith(".so") and path.startswith(str(ROOT)):
                out.add(str(Path(path).relative_to(ROOT)))
    except OSError:
        pass
    return sorted(out)


def reference_input(elements: int):
    """The workload's configuration and initial state built without libfrsdg.so:
    the reference's defaults (oracle/reference.py::default_config) and the GLL
    nodes of the reference's own GLL class (oracle/_ref)."""
    from fr_sdg_b200.workloads import blast_large
    from oracle import reference as REF

    wl = blast_large(elements, defaults=REF.default_config, gll_nodes=REF.reference_element(5)[0])
    return wl, wl.init("cpu").numpy()


def run_reference(args, ws, rank):
    """--impl reference: fr_sdg's own rhs_func path (the reference's include/*.hpp compiled
    into oracle/_ref/libfrsdg_ref.so: DMDA ghost scatter, residual_kernel, VecScale) on
    the full workload mesh, on every host thread (one block of element rows per thread,
    as one MPI rank each would own).  Rank 0 alone runs it; the other ranks exit."""
    if rank != 0:
        return 0
    from oracle import reference as REF

    if not REF.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfrsdg_ref.so was not built "
                                                               "(the reference tree was absent at build time)"}))
        return 0
    threads = os.cpu_count() or 1
    wl, U = reference_input(args.elements)
    F = np.empty_like(U)
    ref = REF.Reference(wl.cfg, threads=threads)
    for _ in range(args.warmup):
        ref.rhs(0.0, U, F)
    step_s = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s0 = time.perf_counter()
        ref.rhs(0.0, U, F)
        step_s.append(time.perf_counter() - s0)
    el = time.perf_counter() - t0
    value = U.size * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.elements == 1024 else f"{WORKLOAD} at {args.elements}^2",
                   "elements": [args.elements, args.elements], "poly_deg": 5, "dofs_per_rank": int(U.size),
                   "parallelism": f"{threads} host threads, one block of element rows each (as MPI ranks)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "cpu_model": cpu_model(),
                         "sample": f"the full {args.elements}^2 mesh ({U.size} DOF) per step: rhs_func of fr_sdg's "
                                   "own include/*.hpp (DMDA ghost scatter, residual_kernel, VecScale) built into "
                                   "oracle/_ref/libfrsdg_ref.so against stand-ins for PETSc/Eigen/Boost; "
                                   f"median step {statistics.median(step_s) * 1e3:.0f} ms"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_loaded": repo_libraries_loaded(),
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_to_t_end(device, t_end: float = 0.25, max_steps: int = 4000) -> dict:
    """Config 4 to t_end in FP64 and in the mixed form: time to t_end of all instances
    together, finiteness per instance and the per-instance density L2 of mixed - FP64
    (absolute and relative to the FP64 density's L2 norm)."""
    import torch

    from fr_sdg_b200.batch import BatchedInstances, density_l2, load_manifest

    specs = load_manifest()
    out, finals = {}, {}
    for mixed in (False, True):
        bi = BatchedInstances(specs, device, mixed=mixed)
        r = bi.run_persistent(t_end, n_steps=max_steps)
        finite = [s.status() == 0 and bool(torch.isfinite(U).all()) for _, s, U, _ in bi.items]
        finals[mixed] = [(wl.cfg, U) for wl, _, U, _ in bi.items]
        out["mixed" if mixed else "fp64"] = {
            "seconds": r.seconds, "instances": r.instances, "dofs": r.dofs, "finite_instances": int(sum(finite)),
            "steps_min_max": [min(r.steps), max(r.steps)], "graph_replays": bi.replays,
            "stopped_before_t_end": bi.stalled,
            "stage_dof_residuals_per_s": r.stage_residuals / r.seconds, "tuning": bi.tuning}
        bi.close()
    errs, rels = [], []
    for (cfg, Ud), (_, Um) in zip(finals[False], finals[True]):
        e = density_l2(cfg, Um, Ud)
        errs.append(e)
        rels.append(e / density_l2(cfg, Ud, torch.zeros_like(Ud)))
    out.update({
        "t_end": t_end, "max_replays": max_steps,
        "scheme": "SSP-RK3, spectral filter + positivity limiter (floor 1e-6) on every stage, CFL 0.1 "
                  "(dt = CFL h / ((2p+1) max(|v|+c)) per instance, re-evaluated on the device after every step; "
                  "an instance whose step falls below 1e-3 of its first stops); the batch engine: one launch "
                  "per order group and stage plus the limiter pass, the post-step in the last stage's "
                  "epilogue, one CUDA graph per step of all instances, device clocks, autotuned tiles "
                  "(the autotuner's first pass is inside the timed region)",
        "mixed_vs_fp64_density_l2": {"max": max(errs), "median": statistics.median(errs),
                                     "relative_max": max(rels), "relative_median": statistics.median(rels),
                                     "per_instance": [float(f"{e:.3e}") for e in errs]},
    })
    return out


def run_ours(args, ws, rank, local):
    import torch

    from fr_sdg_b200 import FRSolver
    from fr_sdg_b200.workloads import blast_large

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()

    # N > 1: one mesh of elements x (elements * N) rows, a row block of elements^2 per
    # rank (weak scaling); every step exchanges one ghost element row with each
    # neighbour over NCCL and evaluates the residual of the owned rows.
    blk = None
    if ws > 1:
        from fr_sdg_b200.partition import exchange_ghost_rows, row_blocks

        wl = blast_large(args.elements, ny=args.elements * ws)
        blk = row_blocks(args.elements * ws, ws, periodic_y=False)[rank]
        solver = FRSolver(wl.cfg)
        solver.set_row_window(*blk.window())
        U = wl.init(f"cuda:{local}", rows=(blk.row_base, blk.rows))
        row_len = U.numel() // blk.rows
    else:
        wl = blast_large(args.elements)
        solver = FRSolver(wl.cfg)
        U = wl.init(f"cuda:{local}")
    F = torch.empty_like(U)
    dofs = U.numel() if blk is None else blk.owned * row_len
    stream = torch.cuda.current_stream()

    def step():
        if blk is not None:
            exchange_ghost_rows(U, blk, row_len)
        solver.rhs_func(0.0, U, F)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for k in range(args.steps):
            if blk is not None:
                exchange_ghost_rows(U, blk, row_len)
            starts[k].record(stream)
            solver.rhs_func(0.0, U, F)
            ends[k].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    barrier()
    elapsed_ms = t0.elapsed_time(t1)
    launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    if dist:
        t = torch.tensor([elapsed_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = ws * dofs * args.steps / (elapsed_ms / 1e3)
    bad = solver.status()

    # ---- the same residual in FP32 (FP32 state), and the RK stage in FP64 and in the
    # mixed form (FP32 arithmetic on the FP64 state, node primitives recovered in FP64),
    # device-resident
    mixed = None
    if not args.no_mixed and ws == 1:
        U32 = U.float()
        F32 = torch.empty_like(U32)
        out = torch.empty_like(U)

        def event_ms(fn):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            for _ in range(args.steps):
                fn()
            m1.record(stream)
            torch.cuda.synchronize()
            return m0.elapsed_time(m1) / args.steps

        mms = event_ms(lambda: solver.residual_kernel_f32(0.0, U32, F32))
        sms = event_ms(lambda: solver.rk_stage(0.0, U, out, gamma=1e-3, a=U, alpha=1.0))
        xms = event_ms(lambda: solver.rk_stage_mixed(0.0, U, out, gamma=1e-3, a=U, alpha=1.0))
        mixed = {"fp32_residual_ms": mms, "fp32_dof_residuals_per_s": ws * dofs / (mms / 1e3),
                 "speedup_vs_fp64": (elapsed_ms / args.steps) / mms,
                 "fp64_stage_ms": sms, "mixed_stage_ms": xms, "mixed_stage_speedup": sms / xms}
        # the FP32 residual with its derivative contractions on the tensor cores (tcgen05,
        # split TF32, cfg.mixed_tc = 1; p = 4 to 7)
        if 4 <= wl.cfg.poly_deg <= 7:
            saved_tc = wl.cfg.mixed_tc
            wl.cfg.mixed_tc = 1
            with FRSolver(wl.cfg) as ts:
                tms = event_ms(lambda: ts.residual_kernel_f32(0.0, U32, F32))
                txms = event_ms(lambda: ts.rk_stage_mixed(0.0, U, out, gamma=1e-3, a=U, alpha=1.0))
            wl.cfg.mixed_tc = saved_tc
            mixed["tensor_cores"] = {"fp32_residual_ms": tms, "fp32_dof_residuals_per_s": ws * dofs / (tms / 1e3),
                                     "mixed_stage_ms": txms,
                                     "path": "tcgen05.mma kind::tf32, operands split hi + lo, FP32 accumulation"}
        # the last SSP-RK3 stage with the post-step (spectral filter + positivity limiter)
        # in its epilogue against the stage and the post-step as two launches
        if blk is None:
            from fr_sdg_b200 import _abi as A

            pcfg = wl.cfg
            saved = (pcfg.apply_filter, pcfg.apply_weno, pcfg.pp_limit)
            pcfg.apply_filter, pcfg.apply_weno, pcfg.pp_limit = 1, 0, 1
            with FRSolver(pcfg) as ps:
                mid = torch.empty_like(U)
                kw = dict(gamma=1e-6, a=U, alpha=1.0 / 3.0, b=U, beta=2.0 / 3.0)
                fused = event_ms(lambda: ps.rk_stage_fused(0.0, U, out, A.STAGE_POST_STEP, **kw))
                sep = event_ms(lambda: (ps.rk_stage(0.0, U, mid, **kw), ps.apply_stabilization_to(mid, out)))
                lim_sep = event_ms(lambda: (ps.rk_stage(0.0, U, out, **kw), ps.pp_limit(out)))
                del mid
            pcfg.apply_filter, pcfg.apply_weno, pcfg.pp_limit = saved
            mixed["stage_epilogue"] = {"workload": "the blast state, spectral filter + positivity limiter",
                                       "fused_stage_post_step_ms": fused, "stage_then_post_step_ms": sep,
                                       "stage_then_limiter_ms": lim_sep}
        del U32, F32, out

    # ---- end to end through the host-buffer entry point
    e2e = None
    if not args.no_e2e and blk is not None:
        # host vectors through the public API: pinned U -> device, ghost exchange,
        # residual, rhs -> pinned host
        Uh = U.cpu().pin_memory()
        Fh = torch.empty_like(Uh).pin_memory()
        ke = max(1, min(args.steps, args.e2e_steps))
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            U.copy_(Uh, non_blocking=True)
            step()
            Fh.copy_(F, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = e0.elapsed_time(e1)
        t = torch.tensor([ems], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
        e2e = {"value": ws * dofs * ke / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": Uh.numel() * 8,
               "d2h_bytes_per_step": Fh.numel() * 8, "steps": ke,
               "path": "pinned host U -> device, NCCL ghost-row exchange, frsdg_rhs, rhs -> pinned host (per rank)"}
    elif not args.no_e2e:
        Uh = U.cpu().pin_memory()
        Fh = torch.empty_like(Uh).pin_memory()
        solver.rhs_func_host(0.0, Uh, Fh)  # allocates the staging buffers once
        ke = max(1, min(args.steps, args.e2e_steps))
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ke):
            solver.rhs_func_host(0.0, Uh, Fh)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ems], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": ws * dofs * ke / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": Uh.numel() * 8,
               "d2h_bytes_per_step": Fh.numel() * 8, "steps": ke,
               "path": "frsdg_rhs_host (pinned host U -> device -> rhs -> pinned host)"}
        # the bound of this path: the same bytes copied both ways at once, pinned host
        # memory, no compute (the residual hides behind the transfers when the step
        # takes as long as the copies alone)
        dU, dF = torch.empty_like(U), torch.empty_like(U)
        cs1, cs2 = torch.cuda.Stream(), torch.cuda.Stream()

        def copies():
            with torch.cuda.stream(cs1):
                dU.copy_(Uh, non_blocking=True)
            with torch.cuda.stream(cs2):
                Fh.copy_(dF, non_blocking=True)

        copies()
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        for _ in range(ke):
            copies()
        torch.cuda.synchronize()
        cms = (time.perf_counter() - c0) * 1e3 / ke
        e2e["copy_bound"] = {"ms_per_step": cms, "gb_per_s_both_directions": 2 * Uh.numel() * 8 / cms / 1e6,
                             "value": ws * dofs / (cms / 1e3), "frac": (ws * dofs * ke / (ems / 1e3)) /
                             (ws * dofs / (cms / 1e3))}
        del dU, dF

    # ---- roofline of the residual kernel
    peak, peak_kind = measured_peaks()
    alg_bytes = dofs * 8 * 2  # read U, write rhs (affine mesh: metrics are constants)
    mean_launch_s = statistics.mean(launch_ms) / 1e3
    achieved = alg_bytes / mean_launch_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_per_launch(), "peak_kind": peak_kind, "kernel": "fr2d_kernel<double,6,VdW,HLLC,affine>",
            "algorithmic_bytes_per_launch": alg_bytes, "mean_launch_ms": mean_launch_s * 1e3}
    # the FP64 compute bound beside it: operations of the reference algorithm per launch
    fl = flops_per_full_launch()
    roof_fp64 = None
    if fl is not None:
        fl *= (args.elements / 1024) ** 2
        tf = fl / mean_launch_s / 1e12
        try:
            dg = dgemm_tflops(f"cuda:{local}")
        except Exception:  # an extra figure must not cost the headline line
            dg = None
        roof_fp64 = {"bound": "fp64", "achieved": tf, "peak": dg or FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": tf / (dg or FP64_NOMINAL_TFLOPS),
                     "peak_kind": "measured: cuBLAS DGEMM 8192^2 (torch.mm), burst" if dg else "nominal",
                     "nominal_peak": FP64_NOMINAL_TFLOPS, "frac_of_nominal": tf / FP64_NOMINAL_TFLOPS,
                     "flops_per_launch": fl, "flop_per_algorithmic_byte": fl / alg_bytes,
                     "count": "reference algorithm restated by the oracle, counting scalar (oracle/count_flops.py)"}

    # ---- time to t_end.  (1) The blast's own schedule (SSP-RK3, 200 steps, WENO with
    # the shock sensor), a throughput figure: the reference algorithm itself turns this
    # configuration non-finite (no positivity limiter), so it is not a converged run.
    # (2) The curved isentropic vortex (64^2, p = 4, RK4, CFL 0.05) to t = 10 with its
    # L2 density error against the exact translated vortex.
    t_end = None
    if not args.no_t_end and ws == 1:
        try:
            from fr_sdg_b200.integrate import Integrator, cfl_time_step, l2_error, node_jacobian
            from fr_sdg_b200.workloads import exact_vortex, node_coords, pack2d, vortex_curved

            def timed(fn):
                barrier()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                res = fn()
                e1.record(stream)
                torch.cuda.synchronize()
                barrier()
                ms = e0.elapsed_time(e1)
                if dist:
                    tt = torch.tensor([ms], device=f"cuda:{local}")
                    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                    ms = float(tt.item())
                return res, ms

            # the first CUDA-graph capture of a process sets up the graph memory pool; do it
            # once outside the timed runs
            _warm = torch.zeros(8, device=f"cuda:{local}")
            _g = torch.cuda.CUDAGraph()
            _side = torch.cuda.Stream()
            _side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(_side):
                _g.capture_begin()
                _warm.add_(1.0)
                _g.capture_end()
            torch.cuda.current_stream().wait_stream(_side)
            _g.replay()
            torch.cuda.synchronize()
            del _g, _warm
            U1 = wl.init(f"cuda:{local}")
            dt = wl.time_step(U1)
            integ = Integrator(solver, "ssprk3")
            integ.step(U1, 0.0, dt)  # warm (allocates the stage buffers)
            U1.copy_(wl.init(f"cuda:{local}"))
            solver.status()
            st, ms = timed(lambda: integ.run(U1, dt, n_steps=wl.n_steps))
            blast = {"seconds": ms / 1e3, "steps": st.steps, "dt": dt, "scheme": "SSP-RK3, spectral filter with the shock sensor (the filter overrides WENO) + positivity "
                                "limiter, CFL 0.1 with the (2p+1) rule; the post-step in the last stage's epilogue",
                     "stage_dof_residuals_per_s": ws * dofs * 3 * st.steps / (ms / 1e3),
                     "finite": solver.status() == 0}
            del U1, integ
            vw = vortex_curved()
            with FRSolver(vw.cfg) as vs:
                V = vw.init(f"cuda:{local}")
                vdt = vw.time_step(V)
                vint = Integrator(vs, "rk4")
                vint.step(V, 0.0, vdt)
                V.copy_(vw.init(f"cuda:{local}"))
                vst, vms = timed(lambda: vint.run(V, vdt, t_end=vw.t_end, graph=True))
                x, y = node_coords(vw.cfg, f"cuda:{local}")
                err = l2_error(vw.cfg, V, pack2d(*exact_vortex(vst.t, x, y)), node_jacobian(vw.cfg, V.device))
                vortex = {"workload": vw.name, "seconds": vms / 1e3, "steps": vst.steps, "t_end": vst.t, "dt": vdt,
                          "scheme": "RK4, CUDA graphs of 64 steps", "l2_density_error_vs_exact": float(err[0]),
                          "finite": vs.status() == 0}
            # (3) The 1D Sod tube (200 elements, p = 3, SSP-RK3 + WENO, t = 0.2): launch-latency
            # bound, so the full steps replay CUDA graphs; L1 density error against the exact
            # Riemann solution (Toro, ch. 4).
            from fr_sdg_b200 import refelem
            from fr_sdg_b200.exact_riemann import sod_exact
            from fr_sdg_b200.workloads import sod1d
            sw = sod1d()
            with FRSolver(sw.cfg) as ss:
                S = sw.init(f"cuda:{local}")
                sdt = sw.time_step(S)
                sint = Integrator(ss, "ssprk3")
                sint.step(S, 0.0, sdt)
                S.copy_(sw.init(f"cuda:{local}"))
                sst, sms = timed(lambda: sint.run(S, sdt, t_end=sw.t_end, graph=True))
                xs, _ = node_coords(sw.cfg, "cpu")
                n1 = sw.cfg.poly_deg + 1
                rho = S.view(-1, 3, n1)[:, 0].cpu().numpy()
                w1 = np.array(refelem.reference_element(sw.cfg.poly_deg)[1]) * 0.5 / sw.cfg.n_elems[0]
                l1 = float(np.sum(w1[None, :] * np.abs(rho - sod_exact(xs.numpy(), sst.t))))
                sod = {"workload": sw.name, "seconds": sms / 1e3, "steps": sst.steps, "t_end": sst.t, "dt": sdt,
                       "scheme": "SSP-RK3, spectral filter + positivity limiter, CFL 0.1 with the (2p+1) rule, "
                                 "CUDA graphs of 64 steps",
                       "l1_density_error_vs_exact": l1, "finite": ss.status() == 0}
            # (4) The vortex again in mixed precision (FP32 residuals, FP64 stage sums)
            with FRSolver(vw.cfg) as vs:
                V = vw.init(f"cuda:{local}")
                vint = Integrator(vs, "rk4", mixed=True)
                vint.step(V, 0.0, vdt)
                V.copy_(vw.init(f"cuda:{local}"))
                mst, mms2 = timed(lambda: vint.run(V, vdt, t_end=vw.t_end, graph=True))
                merr = l2_error(vw.cfg, V, pack2d(*exact_vortex(mst.t, x, y)), node_jacobian(vw.cfg, V.device))
                vortex_mixed = {"workload": vw.name, "seconds": mms2 / 1e3, "steps": mst.steps, "t_end": mst.t,
                                "scheme": "RK4 mixed (FP32 residual, FP64 stages), CUDA graphs of 64 steps",
                                "l2_density_error_vs_exact": float(merr[0]), "finite": vs.status() == 0}
            # (5) The batched uneven workload: 512 seeded circular explosions (32^2..128^2,
            # p = 2..6, ideal / Van der Waals, spectral filter + positivity limiter, CFL 0.1
            # with the (2p+1) rule) each marched to t_end = 0.25 with its own time step,
            # in FP64 and in the mixed form (FP32 residuals, FP64 stage sums), with the
            # density L2 difference of the two per instance.
            batched = batched_to_t_end(f"cuda:{local}")
            def implicit_figures():
                # (6) The implicit path on the bump channel (256 x 64, p = 3, 1,048,576 DOF): the
                # complex-step JVP, the two preconditioner set-ups and applies, and one backward-
                # Euler step with Newton-GMRES and block Gauss-Seidel.
                from fr_sdg_b200.implicit import BackwardEulerNewtonKrylov
                from fr_sdg_b200.workloads import bump_channel

                bw = bump_channel()
                with FRSolver(bw.cfg) as bs:
                    B = bw.init(f"cuda:{local}")
                    Vb = torch.rand_like(B)
                    Jb = torch.empty_like(B)
                    Zb = torch.empty_like(B)
                    bs.pre_jv_eval(0.0, B, 10.0)
                    bs.matmult(Vb, Jb)

                    def rep(fn, n):
                        _, ms_ = timed(lambda: [fn() for _ in range(n)])
                        return ms_ / n

                    jvp_ms = rep(lambda: bs.matmult(Vb, Jb), 20)
                    bs.pc_setup(0.0, 10.0, B)
                    pcj_setup_ms = rep(lambda: bs.pc_setup(0.0, 10.0, B), 3)
                    pcj_apply_ms = rep(lambda: bs.pc_apply(Vb, Zb), 20)
                    bs.pc_setup_gs(0.0, 10.0, B)
                    pcg_setup_ms = rep(lambda: bs.pc_setup_gs(0.0, 10.0, B), 3)
                    pcg_apply_ms = rep(lambda: bs.pc_apply(Vb, Zb), 20)
                    nk = BackwardEulerNewtonKrylov(bs, restart=60, gmres_rtol=1e-6, max_gmres=600, newton_rtol=1e-8,
                                                   precondition="gs")
                    nst, nms = timed(lambda: nk.step(B, 0.0, 0.01))
                    implicit = {"workload": bw.name, "dofs": B.numel(), "jvp_ms": jvp_ms,
                                "jvp_dof_per_s": B.numel() / (jvp_ms / 1e3),
                                "block_jacobi": {"setup_ms": pcj_setup_ms, "apply_ms": pcj_apply_ms},
                                "block_gauss_seidel": {"setup_ms": pcg_setup_ms, "apply_ms": pcg_apply_ms},
                                "backward_euler_step": {"dt": 0.01, "seconds": nms / 1e3,
                                                        "newton_iterations": nst.newton_iterations,
                                                        "gmres_iterations": nst.gmres_iterations,
                                                        "f_drop": nst.f_norms[-1] / nst.f_norms[0]},
                                "finite": bs.status() == 0}
                    # pseudo-transient march of the bump to a 1e-10 residual drop: backward
                    # Euler, one inexact Newton step each (GMRES(60), at most 200 iterations:
                    # 3.3 s against 4.2-5.1 s with 400), the aggregate coarse level
                    # (4 x 4 elements) in front of block Gauss-Seidel
                    from fr_sdg_b200.implicit import march_to_steady

                    S0 = bw.init(f"cuda:{local}")
                    nk2 = BackwardEulerNewtonKrylov(bs, restart=60, max_gmres=200, max_newton=1, precondition="gs",
                                                    coarse=(4, 4))
                    sst, sms = timed(lambda: march_to_steady(bs, S0, dt0=0.05, drop=1e-10, max_steps=60, newton=nk2,
                                                             max_rejections=30, max_growth=3.0, reject_growth=1.5))
                    implicit["steady_state"] = {
                        "seconds": sms / 1e3, "pseudo_time_steps": sst.steps, "rejected": sst.rejected,
                        "newton_iterations": sst.newton_iterations, "gmres_iterations": sst.gmres_iterations,
                        "residual_drop": sst.residual_drop, "converged": sst.residual_drop <= 1e-10,
                        "ms_per_gmres_iteration": sms / max(sst.gmres_iterations, 1),
                        "scheme": "SER pseudo time (dt0 0.05, growth <= 3, steps that grow the residual 1.5x "
                                  "rejected), GMRES(60) <= 200, aggregate coarse level 4x4 + block Gauss-Seidel"}
                return implicit

            try:
                implicit = implicit_figures()
            except Exception as exc:  # an extra figure must not cost the headline line
                implicit = {"error": f"{type(exc).__name__}: {exc}"}
            t_end = {"vortex_curved_64x64_p4": vortex, "vortex_curved_64x64_p4_mixed": vortex_mixed,
                     "blast_200_steps": blast, "sod1d_200_p3": sod, "batched_uneven_512": batched,
                     "implicit_bump_256x64_p3": implicit}
        except Exception as exc:  # the extra runs must not cost the headline line
            t_end = {"error": f"{type(exc).__name__}: {exc}"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle

        oracle.lib()
        threads = os.cpu_count() or 1
        r1, info1 = cpu_residual_rate(1, target_s=10.0, rows=16, max_reps=20)
        cpu = {"value": r1, "unit": UNIT, "cores": 1, "kind": "port", "cpu_model": cpu_model(),
               "sample": info1["sample"] + "; oracle restatement of the reference residual, 1 thread"}
        if args.cpu_all_cores:
            rN, infoN = cpu_residual_rate(threads, target_s=10.0, max_reps=20)
            cpu["all_cores"] = {"value": rN, "cores": threads, "sample": infoN["sample"]}

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.elements == 1024 else f"{WORKLOAD} at {args.elements}^2",
                   "elements": [args.elements, args.elements * ws], "poly_deg": 5, "dofs_per_rank": dofs,
                   "state_bytes": dofs * 8,
                   "l2": f"inputs ({dofs * 8 / 1e9:.2f} GB) larger than L2 (126 MB); no flush",
                   "parallelism": (f"row-block domain decomposition x{ws} ({args.elements}x{args.elements * ws} "
                                   "elements, one ghost element row exchanged with each neighbour per step over NCCL)")
                   if ws > 1 else "single GPU"},
        "clocks": clk.summary(), "gpu_launches": args.steps, "roofline": roof, "roofline_fp64": roof_fp64, "e2e": e2e,
        "cpu_baseline": cpu, "bad_density_nodes": bad, "time_to_t_end": t_end, "mixed_precision": mixed,
    }
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--elements", type=int, default=1024, help="elements per direction (1024 = the workload)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-t-end", action="store_true", help="skip the 200-step time-to-t_end run")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP32 / mixed-precision residual figures")
    ap.add_argument("--cpu-all-cores", action="store_true")
    args = ap.parse_args(argv)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    return run_ours(args, ws, rank, local)


if __name__ == "__main__":
    sys.exit(main())
