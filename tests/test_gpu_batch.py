"""GPU: instances advanced together on a stream pool with graph replays end in the
same state as each advanced alone and eagerly, on the drawn meshes and gases from
smooth seeded states."""
import pytest
import torch

from tests.helpers import random_state

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
