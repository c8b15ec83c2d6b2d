"""GPU: synchronisation modes of the persistent PCG kernels.

Mode 0 meets at a grid-wide counter barrier and then reads the reduction
slots; mode 1 polls per-instance slots (the read is the wait).  Both sum the
same partials in the same order, so every solver kernel must give
bit-identical iterates in both modes; in mode 1 each instance of a packed
batch stops on its own."""
import numpy as np
import pytest

from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu

# (solver path, kernel): register-resident and streamed persistent
KERNELS = [(0, "resident"), (2, "streamed")]


def _run(sc, path, mode, steps, warm="zero", offs=None):
    g = GpuCloth(sc, max_iter=20000, rel_tol=1e-6, warm_start="zero", instances=offs)
    g.sim.set_tuning(path)
    g.sim.set_sync_mode(mode)
    g.sim.set_solver(20000, 1e-6, warm)
    its = g.run(steps)
    return g, its


@pytest.mark.parametrize("path,kernel", KERNELS)
def test_sync_modes_give_identical_iterates(path, kernel):
    sc = scenes.config_large(side=48, steps=5)
    runs = []
    for mode in (0, 1):
        g, its = _run(sc, path, mode, 5)
        assert g.sim.solver_info()[0] == kernel and g.sim.sync_mode() == mode
        assert g.stats()[2] == capi.SOLVE_CONVERGED
        runs.append((its, g.positions(), g.velocities()))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


@pytest.mark.parametrize("path,kernel", KERNELS)
@pytest.mark.parametrize("warm", ["previous", "previous_scaled"])
def test_sync_modes_agree_with_warm_starts(path, kernel, warm):
    sc = scenes.config_small(steps=12)
    a, ia = _run(sc, path, 0, 12, warm=warm)
    b, ib = _run(sc, path, 1, 12, warm=warm)
    assert np.array_equal(ia, ib)
    assert np.array_equal(a.positions(), b.positions())


@pytest.mark.parametrize("path,kernel", KERNELS)
def test_polled_batch_matches_individual_solves(path, kernel):
    inst = scenes.batch_instances(count=5, seed=21, lo=8, hi=30, steps=3, max_iter=20000)
    sc, offs = scenes.concat(inst)
    g, _ = _run(sc, path, 1, 3, offs=offs)
    assert g.sim.solver_info()[0] == kernel
    it_b, rr_b, st_b = g.sim.instance_stats()
    assert (st_b == capi.SOLVE_CONVERGED).all() and (rr_b <= 1e-6).all()
    assert len(set(it_b.tolist())) > 1  # instances stop at their own counts
    pb = g.positions()
    for b, s in enumerate(inst):
        one, _ = _run(s, path, 1, 3)
        assert np.abs(pb[offs[b]:offs[b + 1]] - one.positions()).max() < 1e-5
        assert abs(int(it_b[b]) - one.stats()[0]) <= max(3, 0.02 * one.stats()[0])


def test_sync_mode_argument_checked():
    g = GpuCloth(scenes.config_small(steps=1), max_iter=100, rel_tol=1e-6, warm_start="zero")
    with pytest.raises(ValueError):
        g.sim.set_sync_mode(2)
