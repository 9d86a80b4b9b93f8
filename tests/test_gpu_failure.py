"""Failure detection without a GPU fault: the batched relaxation's bounded
waits are made to run out on purpose and must end the run with
MG_ERR_TIMEOUT, leaving the GPU usable.

* The iteration budget of one launch (mg_batch_set_limits) set to 2 loop
  iterations: the while node's loop test stops the graph with cells still
  running, and the host reports the spent budget.
* The grid-barrier wait of the whole-GPU step set to 0 s: the first CTA to
  wait at a barrier gives up at once, sets the error word, every other wait
  sees it and returns, the loop test stops, the host reports the timeout.

After each, the same batch with default limits relaxes to the same result as
a fresh batch, so the context and the device state are intact."""
import tempfile

import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu


def _mb():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200

    return mapp_b200


def _builder(mb):
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=2, style="DMD_I")
    return mb.system_from_workload(w)


def _relaxed(mb, builder, cells, launch=None):
    B = mb.Batch(builder)
    for c in cells:
        B.add_cell(c)
    B.set_params(5, 40, 1e-5, 1e-8, 60)
    if launch:
        B.set_launch(*launch)
    B.relax()
    out = [B.cell_result(k) for k in range(len(cells))]
    B.close()
    return out


def _same(a, b):
    for (xa, fa, ra), (xb, fb, rb) in zip(a, b):
        assert ra["iterations"] == rb["iterations"]
        # the last line search can end on the minimum step (3) in one run and
        # on the energy tolerance (5) in another: the energies it compares are
        # sums of FP64 atomics, equal only to the last bits between runs
        assert ra["code"] == rb["code"] or {ra["code"], rb["code"]} == {3, 5}
        assert np.max(np.abs(xa - xb)) <= 1e-9


def test_iteration_budget_runs_out():
    mb = _mb()
    builder = _builder(mb)
    cells = [fx.make_dmd_cell(3, 3, 3, sigma=0.03, seed=5 + k) for k in range(3)]
    B = mb.Batch(builder)
    for c in cells:
        B.add_cell(c)
    B.set_params(5, 40, 1e-5, 1e-8, 60)
    B.set_limits(iteration_budget=2)
    with pytest.raises(mb.MGError) as e:
        B.relax()
    assert e.value.code == mb.MG_ERR_TIMEOUT and "iteration budget" in str(e.value)
    B.set_limits(iteration_budget=0)
    B.relax()
    again = [B.cell_result(k) for k in range(len(cells))]
    B.close()
    _same(again, _relaxed(mb, builder, cells))


def test_grid_barrier_wait_runs_out():
    mb = _mb()
    builder = _builder(mb)
    cells = [fx.make_dmd_cell(4, 4, 4, sigma=0.03, seed=21)]
    whole = (0, 0, 1024, mb.MG_LAUNCH_WHOLE_GPU)
    B = mb.Batch(builder)
    B.add_cell(cells[0])
    B.set_params(5, 40, 1e-5, 1e-8, 60)
    B.set_launch(*whole)
    B.set_limits(barrier_wait_s=0.0)
    with pytest.raises(mb.MGError) as e:
        B.relax()
    assert e.value.code == mb.MG_ERR_TIMEOUT and "grid barrier" in str(e.value)
    B.set_limits(barrier_wait_s=2.0)
    B.relax()
    again = [B.cell_result(0)]
    B.close()
    _same(again, _relaxed(mb, builder, cells, launch=whole))


def test_limits_rejected():
    mb = _mb()
    builder = _builder(mb)
    B = mb.Batch(builder)
    with pytest.raises(mb.MGError):
        B.set_limits(iteration_budget=-1)
    with pytest.raises(mb.MGError):
        B.set_limits(barrier_wait_s=-1.0)
