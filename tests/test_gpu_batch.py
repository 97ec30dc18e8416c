"""GPU: instances advanced together on a stream pool with graph replays end in the
same state as each advanced alone and eagerly, on the drawn meshes and gases from
smooth seeded states."""
import pytest
import torch

from tests.helpers import random_state, rel_err

from fr_sdg_b200 import FRSolver
from fr_sdg_b200.batch import BatchedInstances, instance_workload, load_manifest
from fr_sdg_b200.integrate import Integrator, cfl_time_step

pytestmark = pytest.mark.gpu


def test_batched_matches_standalone(cuda):
    specs = [s for s in load_manifest() if s.n_elems <= 48][:6]
    init = lambda cfg, dev: torch.from_numpy(random_state(cfg, cfg.n_elems[0] + cfg.poly_deg, amp=0.05,
                                                          smooth=True)).to(dev)
    b = BatchedInstances(specs, cuda, streams=3, init=init)
    try:
        r = b.run(None, 0.02, n_steps=12, steps_per_graph=4)
        assert r.steps == [12] * len(specs) and r.finite == len(specs)
        for sp, (wl, _, U, _) in zip(specs, b.items):
            w2 = instance_workload(sp)
            with FRSolver(w2.cfg) as s:
                V = init(w2.cfg, cuda)
                Integrator(s, "ssprk3").run(V, cfl_time_step(w2.cfg, V, 0.02, w2.cfl_rule), n_steps=12)
                assert torch.equal(U, V), sp
    finally:
        b.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_device_batch_matches_integrator(mixed, cuda):
    """frsdg_batch (one launch per group and stage, device clocks, graph replay) ends in the
    per-instance integrator's state, the clipped final step included.  The batch kernels
    compile the same element code as the single-instance kernels but into other kernels,
    where the compiler may contract a different set of products into FMAs, so the two
    agree to rounding (1e-13 of max|U| in FP64, 1e-9 for the FP32 arithmetic of the mixed
    form after eleven steps), not bit for bit."""
    from fr_sdg_b200.batch import DeviceBatch

    specs = [s for s in load_manifest() if s.n_elems <= 48][:8]
    init = lambda cfg, dev: torch.from_numpy(random_state(cfg, cfg.n_elems[0] + cfg.poly_deg, amp=0.05,
                                                          smooth=True)).to(dev)
    items, refs = [], []
    for sp in specs:
        w = instance_workload(sp)
        s = FRSolver(w.cfg)
        U = init(w.cfg, cuda)
        dt = cfl_time_step(w.cfg, U, 0.05, w.cfl_rule)
        items.append((s, U, dt, 10.5 * dt))
        V = U.clone()
        Integrator(s, "ssprk3", mixed=mixed).run(V, dt, t_end=10.5 * dt)
        refs.append(V)
    db = DeviceBatch(items, mixed=mixed)
    try:
        steps = db.run()
        assert steps >= 11
        t, active, nsteps = db.times()
        assert not any(active)
        assert nsteps == [11] * len(items)  # ten full steps and the clipped one
        tol = 1e-9 if mixed else 1e-13
        for (s, U, dt, te), V, ti in zip(items, refs, t):
            assert ti == te
            err = rel_err(U.cpu().numpy(), V.cpu().numpy())
            assert err <= tol, f"batch vs integrator: rel err {err:.3e}"
            assert s.status() == 0
        tuned = db.tuning()
        assert tuned and all(g["ctas"] > 0 and g["tile_variant"] in (0, 1) for g in tuned)
    finally:
        db.close()
        for s, _, _, _ in items:
            s.close()


def test_device_batch_explosions_stay_finite(cuda):
    """Drawn circular explosions (spectral filter + positivity limiter, CFL 0.1 with the
    (2p+1) rule) through the batch engine to t = 0.05: every instance admissible."""
    specs = [s for s in load_manifest() if s.n_elems <= 64][:24]
    b = BatchedInstances(specs, cuda)
    try:
        dt0 = [cfl_time_step(wl.cfg, U, wl.cfl, wl.cfl_rule) for wl, _, U, _ in b.items]
        r = b.run_persistent(0.05)
        assert r.finite == len(specs)
        assert all(t == 0.05 for t in b.times)
        # adaptive steps follow the wave speed, which the explosions change by a few times
        for k, d in zip(r.steps, dt0):
            assert 0.05 / d / 4 <= k <= 4 * 0.05 / d + 1
        for _, _, U, _ in b.items:
            q = U.view(-1, 4)
            assert bool(torch.isfinite(U).all()) and float(q[:, 0].min()) > 0.0
    finally:
        b.close()
