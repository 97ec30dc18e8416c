"""The batched uneven workload: many independent small FR problems run together.

Instances are circular explosions (ProblemFactory2D<CircularExplosion>,
factory.hpp:400-465) on [-1,1]^2 with Rusanov fluxes and outflow boundaries, drawn
with numpy.random.default_rng(20261203) in the order {Nx, p, gas kind, gamma | (a, b),
r0, p_out} per instance: Nx = Ny in {32, 48, 64, 96, 128}, p in {2..6}, ideal gas with
gamma ~ U[1.3, 1.67] or Van der Waals with a ~ U[0.01, 0.1], b ~ U[0.01, 0.05],
gamma = 1.4; density 1 / 0.125 and pressure 1 / p_out ~ U[0.05, 0.2] inside / outside
r0 ~ U[0.3, 0.5].  The draws are committed as data/batched_uneven_512.json.

Each instance has its own handle, state and time step (CFL on its own mesh).  They
advance concurrently on a pool of CUDA streams, every instance replaying its own CUDA
graph of 64 SSP-RK3 steps, so small meshes overlap on the GPU instead of leaving it
idle one launch at a time.
"""
from __future__ import annotations

import json
import time
from dataclasses import asdict, dataclass
from pathlib import Path

import numpy as np
import torch

from .integrate import Integrator, cfl_time_step
from .solver import FRSolver
from .workloads import SHOCK_STAB, Workload, circular_explosion

SEED = 20261203
SIZES = (32, 48, 64, 96, 128)
MANIFEST = Path(__file__).resolve().parent / "data" / "batched_uneven_512.json"


@dataclass(frozen=True)
class InstanceSpec:
    n_elems: int
    p: int
    gas: str
    gamma: float
    vdw_a: float
    vdw_b: float
    r0: float
    p_out: float


def draw_instances(n: int = 512, seed: int = SEED) -> list[InstanceSpec]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ne = int(rng.choice(SIZES))
        p = int(rng.integers(2, 7))
        vdw = bool(rng.integers(0, 2))
        if vdw:
            gamma, a, b = 1.4, float(rng.uniform(0.01, 0.1)), float(rng.uniform(0.01, 0.05))
        else:
            gamma, a, b = float(rng.uniform(1.3, 1.67)), 0.0, 0.0
        r0 = float(rng.uniform(0.3, 0.5))
        p_out = float(rng.uniform(0.05, 0.2))
        out.append(InstanceSpec(ne, p, "vdw" if vdw else "ideal", gamma, a, b, r0, p_out))
    return out


def write_manifest(specs: list[InstanceSpec], path: Path = MANIFEST) -> None:
    path.write_text(json.dumps({"seed": SEED, "instances": [asdict(s) for s in specs]}, indent=1) + "\n")


def load_manifest(path: Path = MANIFEST) -> list[InstanceSpec]:
    return [InstanceSpec(**d) for d in json.loads(path.read_text())["instances"]]


def instance_workload(spec: InstanceSpec, stab: str = "filter") -> Workload:
    """stab = "filter": the configured spectral filter; "weno": WENO + shock sensor with
    the filter off (the settings of the reference's shock runs)."""
    # the filter's cut-off mode is 2 (filter.hpp defaults); at p = 2 that is the top
    # mode and the filter strength formula divides 0 by 0, so p = 2 instances cut at 1
    wl = circular_explosion(spec.n_elems, spec.p, spec.gas, spec.gamma, (spec.vdw_a, spec.vdw_b), spec.r0,
                            spec.p_out, filt_cut_off=min(2, spec.p - 1))
    if stab == "weno":
        c = wl.cfg
        c.apply_filter = 0
        c.apply_weno = 1
        c.weno_gamma = SHOCK_STAB["weno_gamma"]
        c.shock_threshold = SHOCK_STAB["threshold"]
        c.shock_theta = SHOCK_STAB["theta"]
    return wl


class DeviceBatch:
    """A batch of instances advanced by the library (frsdg_batch): every SSP-RK3 stage of
    all instances of a group is one launch, one step of the whole batch is replayed as a
    CUDA graph until every instance reaches its t_end, and an autotuner picks each
    group's tile and persistent-CTA count.  items: (FRSolver, state, dt, t_end).
    dt_scale: per item, adaptive steps dt = dt_scale / max(|v| + c) after every step."""

    def __init__(self, items, mixed: bool = False, dt_scale=None):
        import ctypes as C

        from . import _abi as A

        self._A, self._C = A, C
        self.items = list(items)
        n = len(self.items)
        hs = (C.c_void_p * n)(*[s._h.value if hasattr(s._h, "value") else s._h for s, _, _, _ in self.items])
        us = (C.c_void_p * n)(*[U.data_ptr() for _, U, _, _ in self.items])
        dts = (C.c_double * n)(*[float(dt) for _, _, dt, _ in self.items])
        tends = (C.c_double * n)(*[float(te) for _, _, _, te in self.items])
        scales = (C.c_double * n)(*[float(x) for x in dt_scale]) if dt_scale is not None else None
        self._h = C.c_void_p()
        A.check(A.lib().frsdg_batch_create(hs, n, us, dts, scales, tends, int(mixed), C.byref(self._h)),
                "frsdg_batch_create")

    def close(self) -> None:
        if self._h:
            self._A.lib().frsdg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> None:
        self._A.check(self._A.lib().frsdg_batch_step(self._h, torch.cuda.current_stream().cuda_stream),
                      "frsdg_batch_step")

    def run(self, max_steps: int = 0) -> int:
        """Replay steps until every instance reaches its t_end (or max_steps > 0 steps)."""
        C = self._C
        k = C.c_int64()
        self._A.check(self._A.lib().frsdg_batch_run(self._h, int(max_steps), C.byref(k),
                                                    torch.cuda.current_stream().cuda_stream), "frsdg_batch_run")
        return int(k.value)

    def times(self):
        """(t, active, steps) of every instance."""
        C, n = self._C, len(self.items)
        t, act, st = (C.c_double * n)(), (C.c_int32 * n)(), (C.c_int64 * n)()
        self._A.check(self._A.lib().frsdg_batch_times(self._h, t, act, st), "frsdg_batch_times")
        return list(t), [bool(a) for a in act], list(st)

    def tuning(self) -> list[dict]:
        C = self._C
        g = C.c_int32()
        self._A.check(self._A.lib().frsdg_batch_groups(self._h, C.byref(g)), "frsdg_batch_groups")
        out = []
        for i in range(g.value):
            n, var, grid, tiles, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
            self._A.check(self._A.lib().frsdg_batch_tuning(self._h, i, C.byref(n), C.byref(var), C.byref(grid),
                                                           C.byref(tiles), C.byref(ms)), "frsdg_batch_tuning")
            out.append({"order_n": n.value, "tile_variant": var.value, "ctas": grid.value, "tiles": tiles.value,
                        "stage_ms": ms.value})
        return out


def density_l2(cfg, U: torch.Tensor, V: torch.Tensor) -> float:
    """GLL-quadrature L2 norm of the density difference of two states of one instance
    (physical measure: detJ of the affine map, (h_x/2)(h_y/2))."""
    from .refelem import reference_element

    n = cfg.poly_deg + 1
    w = torch.tensor(reference_element(cfg.poly_deg)[1], dtype=torch.float64, device=U.device)
    jac = (0.5 * cfg.box_length[0] / cfg.n_elems[0]) * (0.5 * cfg.box_length[1] / cfg.n_elems[1])
    d = (U.view(-1, n, n, 4)[..., 0] - V.view(-1, n, n, 4)[..., 0])
    return float(torch.sqrt(jac * ((w[:, None] * w[None, :])[None] * d * d).sum()))


@dataclass
class BatchResult:
    instances: int
    dofs: int
    stage_residuals: float    # sum over instances of DOFs x stages
    seconds: float
    finite: int               # instances whose health word stayed clear
    steps: list
    capture_seconds: float = 0.0  # host time spent capturing the graphs (before timing)


class BatchedInstances:
    """All instances of a batch, resident on one GPU."""

    def __init__(self, specs: list[InstanceSpec], device, stab: str = "filter", streams: int = 16, init=None,
                 mixed: bool = False, pp_eps: float | None = None):
        """init(cfg, device) -> state replaces the explosion initial states (tests).
        mixed: FP32 residuals with FP64 stage sums (Integrator(mixed=True)).
        pp_eps: the positivity limiter's floor, replacing the workload's."""
        self.device = torch.device(device)
        self.items = []
        for sp in specs:
            wl = instance_workload(sp, stab)
            if pp_eps is not None:
                wl.cfg.pp_eps = pp_eps
            s = FRSolver(wl.cfg)
            U = wl.init(self.device) if init is None else init(wl.cfg, self.device)
            self.items.append((wl, s, U, Integrator(s, "ssprk3", mixed=mixed)))
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(streams)]

    @property
    def dofs(self) -> int:
        return sum(U.numel() for _, _, U, _ in self.items)

    def close(self) -> None:
        for _, s, _, _ in self.items:
            s.close()
        self.items = []

    def run_persistent(self, t_end: float | None, n_steps: int | None = None, adaptive: bool = True) -> BatchResult:
        """The whole batch through the library's batch engine (DeviceBatch): one launch per
        group and stage, one CUDA graph per step replayed until every instance reaches
        t_end (or for n_steps steps); device-timed, the autotuner's first pass included.
        adaptive: each instance's step follows its current wave speed (the workload's CFL
        rule on max |v| + c of the state after every step)."""
        cur = torch.cuda.current_stream(self.device)
        for _, s, _, _ in self.items:
            s.status()
        dts = [cfl_time_step(wl.cfg, U, wl.cfl, wl.cfl_rule) for wl, _, U, _ in self.items]
        te = t_end if t_end is not None else 1e300  # finite: the clocks' tolerance scales with t_end
        scales = None
        if adaptive:
            scales = []
            for wl, _, _, _ in self.items:
                c = wl.cfg
                h = min(c.box_length[0] / c.n_elems[0], c.box_length[1] / c.n_elems[1])
                scales.append(wl.cfl * h / ((2 * c.poly_deg + 1) if wl.cfl_rule == "dg" else 1.0))
        db = DeviceBatch([(s, U, dt, te) for (wl, s, U, it), dt in zip(self.items, dts)], mixed=self.items[0][3].mixed,
                         dt_scale=scales)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        k = db.run(n_steps or 0)
        e1.record(cur)
        torch.cuda.synchronize(self.device)
        self.times, _, steps = db.times()
        self.replays = k  # replays of the step graph (inactive instances skip theirs)
        # instances that stopped before t_end (adaptive step below its floor)
        self.stalled = sum(1 for t in self.times if t < te * (1.0 - 1e-14)) if t_end is not None else 0
        self.tuning = db.tuning()
        db.close()
        finite = sum(1 for _, s, _, _ in self.items if s.status() == 0)
        stage = float(sum(3 * n * U.numel() for n, (_, _, U, _) in zip(steps, self.items)))
        return BatchResult(len(self.items), self.dofs, stage, e0.elapsed_time(e1) / 1e3, finite, steps, 0.0)

    def run(self, t_end: float | None, cfl: float | None = None, graph: bool = True, n_steps: int | None = None,
            steps_per_graph: int = 64) -> BatchResult:
        """Advance every instance to t_end (or by n_steps steps) with its own CFL time
        step; device-timed from the first launch to the last completion over all
        streams.  With n_steps and graph=True every instance's graph of
        steps_per_graph steps is captured before the timed region, which then holds
        only graph replays (and the eager leftover steps)."""
        cur = torch.cuda.current_stream(self.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _, s, _, _ in self.items:
            s.status()
        dts = [cfl_time_step(wl.cfg, U, wl.cfl if cfl is None else cfl, wl.cfl_rule) for wl, _, U, _ in self.items]
        graphs, t_cap = None, 0.0
        if graph and t_end is None and n_steps is not None and n_steps >= steps_per_graph:
            c0 = time.perf_counter()
            graphs = []
            for k, ((_, _, U, it), dt) in enumerate(zip(self.items, dts)):
                st = self.streams[k % len(self.streams)]
                st.wait_stream(cur)
                with torch.cuda.stream(st):
                    graphs.append(it.capture(U, dt, steps_per_graph))
            for st in self.streams:
                cur.wait_stream(st)
            torch.cuda.synchronize(self.device)
            t_cap = time.perf_counter() - c0
        e0.record(cur)
        steps = []
        for k, ((wl, s, U, it), dt) in enumerate(zip(self.items, dts)):
            st = self.streams[k % len(self.streams)]
            st.wait_stream(cur)
            with torch.cuda.stream(st):
                if graphs is None:
                    steps.append(it.run(U, dt, t_end=t_end, n_steps=n_steps, graph=graph,
                                        steps_per_graph=steps_per_graph).steps)
                    continue
                reps = n_steps // steps_per_graph
                for _ in range(reps):
                    graphs[k].replay()
                t = 0.0
                for _ in range(reps * steps_per_graph):
                    t += dt
                for _ in range(n_steps - reps * steps_per_graph):
                    it.step(U, t, dt)
                    t += dt
                steps.append(n_steps)
        for st in self.streams:
            cur.wait_stream(st)
        e1.record(cur)
        torch.cuda.synchronize(self.device)
        del graphs
        finite = sum(1 for _, s, _, _ in self.items if s.status() == 0)
        stage = float(sum(3 * n * U.numel() for n, (_, _, U, _) in zip(steps, self.items)))
        return BatchResult(len(self.items), self.dofs, stage, e0.elapsed_time(e1) / 1e3, finite, steps, t_cap)
