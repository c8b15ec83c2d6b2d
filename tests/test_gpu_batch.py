"""Batched solve: several cloth instances of uneven size packed into one
particle buffer and solved by one persistent PCG launch with per-instance
convergence must reproduce solving each instance on its own."""
import numpy as np
import pytest

from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu


def packed(count, seed, lo=8, hi=24):
    inst = scenes.batch_instances(count=count, seed=seed, lo=lo, hi=hi, steps=4, max_iter=20000)
    sc, offs = scenes.concat(inst)
    return inst, sc, offs


@pytest.mark.parametrize("path", [0, 2])
def test_batch_matches_individual_solves(path):
    inst, sc, offs = packed(6, seed=11)
    g = GpuCloth(sc, max_iter=20000, rel_tol=1e-8, warm_start="zero", instances=offs)
    g.sim.set_tuning(path)
    g.run(3, record_iters=False)
    pb = g.positions()
    it_b, rr_b, st_b = g.sim.instance_stats()
    assert (st_b == capi.SOLVE_CONVERGED).all() and (rr_b <= 1e-8).all()
    for b, s in enumerate(inst):
        one = GpuCloth(s, max_iter=20000, rel_tol=1e-8, warm_start="zero")
        one.sim.set_tuning(path)
        one.run(3, record_iters=False)
        assert np.abs(pb[offs[b]:offs[b + 1]] - one.positions()).max() < 1e-5
        # per-instance convergence: same iteration count as alone, up to
        # reduction-order round-off
        assert abs(int(it_b[b]) - one.stats()[0]) <= max(3, 0.02 * one.stats()[0])


def test_batch_instances_converge_independently():
    inst, sc, offs = packed(5, seed=12, lo=6, hi=40)
    g = GpuCloth(sc, max_iter=20000, rel_tol=1e-6, warm_start="zero", instances=offs)
    # the first step from the stress-free rest state of these regular grids
    # converges in one iteration for every instance (the FP64 oracle too), so
    # the counts are compared on the second step
    g.step()
    g.step()
    it, rr, st = g.sim.instance_stats()
    assert len(it) == 5 and (st == capi.SOLVE_CONVERGED).all()
    assert len(set(it.tolist())) > 1  # uneven sizes converge at different counts
    tot_it, tot_rr, tot_st = g.stats()
    assert tot_it == it.max() and tot_st == capi.SOLVE_CONVERGED


def test_batch_rejects_cross_instance_triangle():
    inst, sc, offs = packed(2, seed=13)
    tris = np.concatenate([sc["tris"], [[0, 1, int(offs[1])]]]).astype(np.int32)
    sc = dict(sc, tris=tris, edges=scenes.unique_edges(tris))
    g = GpuCloth(sc, max_iter=100, rel_tol=1e-6, warm_start="zero", instances=offs)
    with pytest.raises(ValueError):
        g.step()


def test_batch_dump_is_in_caller_order():
    inst, sc, offs = packed(3, seed=14)
    g = GpuCloth(sc, max_iter=20000, rel_tol=1e-8, warm_start="zero", instances=offs)
    g.step()
    diag, rp, col, vals, rhs, dx = g.dump()
    assert diag.shape[0] == sc["pos"].shape[0]
    one = GpuCloth(inst[1], max_iter=20000, rel_tol=1e-8, warm_start="zero")
    one.step()
    d1, rp1, col1, v1, rhs1, dx1 = one.dump()
    lo, hi = offs[1], offs[2]
    np.testing.assert_array_equal(diag[lo:hi], d1)
    np.testing.assert_array_equal(rhs[lo:hi], rhs1)
    np.testing.assert_array_equal(col[rp[lo]:rp[hi]] - lo, col1)
