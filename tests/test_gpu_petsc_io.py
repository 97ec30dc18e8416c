"""PETSc binary solution files written from the GPU: the device packer byte for byte
against numpy's big-endian encoding, and SolutionMonitor files read back with the
reference tools' reader (restated in oracle/petsc_binary.py)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from fr_sdg_b200 import FRSolver
from fr_sdg_b200.integrate import Integrator, cfl_time_step
from fr_sdg_b200.petsc_io import SolutionMonitor, pack_record
from fr_sdg_b200.workloads import sod1d, vortex_curved
from oracle.petsc_binary import last_vector, read_all_vectors, record_bytes

pytestmark = pytest.mark.gpu


def _bits(n: int, seed: int) -> np.ndarray:
    """n doubles from random 64-bit patterns (NaN payloads, infinities, subnormals and
    signed zeros included), so the packer is checked on every byte value."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 2 ** 63, size=n, dtype=np.int64).view(np.float64).copy()
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -2.2250738585072014e-308, 1.0])
    x[: min(n, special.size)] = special[: min(n, special.size)]
    if n > 8:
        x[8:: 3] = -x[8:: 3]
    return x


@pytest.mark.parametrize("index_bytes", [4, 8])
@pytest.mark.parametrize("n", [0, 1, 7, 1000, 3_000_001])
def test_pack_bit_exact(cuda, n, index_bytes):
    x = _bits(n, seed=n + index_bytes)
    rec = pack_record(torch.from_numpy(x).to(cuda), index_bytes)
    torch.cuda.synchronize()
    assert rec.cpu().numpy().tobytes() == record_bytes(x, index_bytes)


def test_pack_rejects_bad_arguments(cuda):
    x = torch.zeros(17, dtype=torch.float64, device=cuda)
    out = torch.empty(8 + 8 * 16 + 8, dtype=torch.uint8, device=cuda)
    from fr_sdg_b200 import _abi as A
    lib = A.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # misaligned destination and source are refused on the host, before any launch
    assert lib.frsdg_petsc_vec_pack(x.data_ptr(), 16, 4, out.data_ptr() + 4, stream) == A.ERR_ARG
    assert lib.frsdg_petsc_vec_pack(x.data_ptr() + 4, 8, 4, out.data_ptr(), stream) == A.ERR_ARG
    assert lib.frsdg_petsc_vec_pack(x.data_ptr(), 16, 3, out.data_ptr(), stream) == A.ERR_ARG
    with pytest.raises(ValueError):
        pack_record(x.float())


def test_monitor_records_every_interval(cuda, tmp_path):
    """interval 2 over 5 steps writes steps 0, 2, 4 and the final step 5, each equal to
    the eager run's state at that step."""
    wl = vortex_curved(n_elems=8, p=3)
    with FRSolver(wl.cfg) as s:
        U0 = wl.init(cuda)
        dt = wl.time_step(U0)
        ref, U = [U0.clone()], U0.clone()
        it = Integrator(s, "rk4")
        for k in range(5):
            it.step(U, k * dt, dt)
            ref.append(U.clone())
        f = tmp_path / "vortex.bin"
        U = U0.clone()
        with SolutionMonitor(f, interval=2) as m:
            st = Integrator(s, "rk4").run(U, dt, n_steps=5, monitor=m)
        assert st.steps == 5 and m.records == 4
        got = read_all_vectors(f)
        assert len(got) == 4
        for vec, k in zip(got, (0, 2, 4, 5)):
            assert np.array_equal(vec.astype(np.float64), ref[k].cpu().numpy()), k


def test_monitor_final_only_with_graph(cuda, tmp_path):
    """interval -1 + skip_initial (the reference tools' settings): one record, the final
    state, also when the steps replay CUDA graphs and the last step is clipped."""
    wl = sod1d()
    with FRSolver(wl.cfg) as s:
        U0 = wl.init(cuda)
        dt = wl.time_step(U0)
        t_end = 20.5 * dt
        Ue, Ug = U0.clone(), U0.clone()
        Integrator(s, "ssprk3").run(Ue, dt, t_end=t_end)
        f = tmp_path / "sod.bin"
        with SolutionMonitor(f, interval=-1, skip_initial=True) as m:
            st = Integrator(s, "ssprk3").run(Ug, dt, t_end=t_end, graph=True, steps_per_graph=8, monitor=m)
        assert st.steps == 21 and m.records == 1
        assert len(read_all_vectors(f)) == 1
        assert np.array_equal(last_vector(f).astype(np.float64), Ue.cpu().numpy())
        assert torch.equal(Ue, Ug)
