"""The CTA-local Chebyshev preconditioner of the register-resident kernel:
the same converged solutions as block-Jacobi PCG (the oracle's), iteration
counts as the oracle's restatement of the same preconditioner, and the warm
starts, batches and determinism that the default path has."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu


def oracle_sim(sc, tol, warm="zero", fp64=True, degree=0, block_rows=512, max_iter=20000):
    n = sc["pos"].shape[0]
    s = O.OracleCloth(fp64)
    s.set_material(sc["density"], 0.0, sc["gravity"])
    s.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    s.set_mesh(sc["tris"])
    im = s.redistribute_mass(sc["density"])
    s.set_state(sc["pos"], sc["vel"], im)
    s.build_springs(sc["k_spring"])
    s.build_stretch(sc["k_stretch"])
    s.set_pins(sc["pin_idx"], sc["pin_targets"], sc.get("k_pin", 1e6))
    s.set_solver(max_iter, tol, warm)
    s.set_preconditioner(degree, 30.0, block_rows)
    return s


def gpu(sc, degree, order=0, **kw):
    g = GpuCloth(sc, **kw)
    if order:
        g.sim.set_row_order(order)
    if degree:
        g.sim.set_preconditioner("chebyshev", degree, 30.0)
    return g


def trajectories(sc, steps, degree, order=0, warm="zero", tol=1e-7):
    """Positions after `steps` of the preconditioned GPU run, of the
    block-Jacobi GPU run at the same tolerance, and of the FP64 oracle."""
    a = gpu(sc, degree, order, max_iter=20000, rel_tol=tol, warm_start=warm)
    b = gpu(sc, 0, 0, max_iter=20000, rel_tol=tol, warm_start=warm)
    o = oracle_sim(sc, 1e-11)
    for _ in range(steps):
        a.step()
        b.step()
        o.step(sc["dt"])
        assert a.stats()[2] == capi.SOLVE_CONVERGED
    return a, a.positions(), b.positions(), o.state()[0]


@pytest.mark.parametrize("side", [10, 64])
@pytest.mark.parametrize("degree", [3, 9])
def test_chebyshev_solutions_and_iterations(side, degree):
    sc = scenes.config_small(side=side, steps=4)
    g = gpu(sc, degree, max_iter=20000, rel_tol=1e-7)
    g.step()
    kind, deg, ratio, used = g.sim.preconditioner()
    assert (kind, deg, used) == ("chebyshev", degree, 1)
    block_rows = g.sim.solver_info()[2]  # one CTA's rows
    o = oracle_sim(sc, 1e-11)
    o.step(sc["dt"])
    assert np.abs(g.dump()[5] - o.dump_system()[5]).max() < 2e-6
    # a stop at rel-res 1e-7 bounds dx only as loosely as cond(A) allows: the
    # preconditioned run must stay as close to the FP64 solution as the
    # block-Jacobi run stopped at the same residual
    _, pc, bj, ref = trajectories(sc, 4, degree)
    assert np.abs(pc - ref).max() <= max(3.0 * np.abs(bj - ref).max(), 2e-5)
    # same preconditioner on the CPU (FP32 port), same state: similar counts
    c = oracle_sim(sc, 1e-7, fp64=False, degree=degree, block_rows=block_rows)
    c.set_state(*[a.astype(np.float32) for a in (g.positions(), g.velocities())], g.inv_mass.cpu().numpy())
    g.step()
    c.step(sc["dt"])
    gi, ci = g.stats()[0], c.stats()[0]
    # FP32 on both sides, different summation orders (the per-block lambda
    # estimates differ in the last bits): counts within 15%
    assert abs(gi - ci) <= 0.15 * ci + 2
    b = oracle_sim(sc, 1e-7, fp64=False)
    b.set_state(*[a.astype(np.float32) for a in (g.positions(), g.velocities())], g.inv_mass.cpu().numpy())
    b.step(sc["dt"])
    assert gi < 0.75 * b.stats()[0]  # fewer iterations than block-Jacobi


@pytest.mark.parametrize("warm", ["previous", "previous_scaled"])
def test_chebyshev_warm_starts(warm):
    sc = scenes.config_small(side=32, steps=10)
    _, pc, bj, ref = trajectories(sc, 10, 5, warm=warm)
    assert np.abs(pc - ref).max() <= max(3.0 * np.abs(bj - ref).max(), 2e-5)


@pytest.mark.parametrize("degree", [0, 5])
def test_spatial_row_order(degree):
    """Rows reordered into compact blocks: same system and solutions as the
    caller's order, with (for the CTA-local preconditioner) fewer iterations."""
    sc = scenes.config_small(side=64, steps=3)
    a = gpu(sc, degree, order=1, max_iter=20000, rel_tol=1e-7)
    b = gpu(sc, degree, order=0, max_iter=20000, rel_tol=1e-7)
    a.step()
    b.step()
    rows = a.sim.row_of_particles(sc["pos"].shape[0])
    assert sorted(rows.tolist()) == list(range(len(rows))) and (rows != np.arange(len(rows))).any()
    da, db = a.dump(), b.dump()
    np.testing.assert_array_equal(da[1], db[1])  # pattern in particle order
    np.testing.assert_array_equal(da[2], db[2])
    assert np.abs(da[0] - db[0]).max() <= 1e-6 * np.abs(db[0]).max()
    assert np.abs(da[3] - db[3]).max() <= 1e-6 * np.abs(db[3]).max()
    assert np.abs(da[5] - db[5]).max() < 2e-6
    _, pc, bj, ref = trajectories(sc, 3, degree, order=1)
    assert np.abs(pc - ref).max() <= max(3.0 * np.abs(bj - ref).max(), 2e-5)
    if degree:
        assert a.stats()[0] <= b.stats()[0]


def test_chebyshev_in_a_batch_matches_single_runs():
    scs = [scenes.config_small(side=s, steps=3) for s in (12, 20, 9)]
    sc, offs = scenes.concat(scs)
    g = gpu(sc, 5, max_iter=20000, rel_tol=1e-7, instances=offs)
    g.run(3, record_iters=False)
    assert g.sim.preconditioner()[3]
    st = g.sim.instance_stats()
    assert all(s == capi.SOLVE_CONVERGED for s in st[2])
    for k, s in enumerate(scs):
        one = gpu(s, 5, max_iter=20000, rel_tol=1e-7)
        one.run(3, record_iters=False)
        # the same kernel on different CTA partitions: reductions sum in a
        # different order and the solves stop on different iterates (rel-res
        # 1e-7), which three steps of this cloth amplify to ~2e-5 m
        np.testing.assert_allclose(g.positions()[offs[k]:offs[k + 1]], one.positions(), atol=5e-5)


def test_chebyshev_is_deterministic_and_other_kernels_keep_block_jacobi():
    sc = scenes.config_small(side=48, steps=3)
    runs = []
    for _ in range(2):
        g = gpu(sc, 7, max_iter=400, rel_tol=0.0)
        g.run(3, record_iters=False)
        runs.append(g.positions())
    np.testing.assert_array_equal(runs[0], runs[1])
    g = gpu(sc, 7, max_iter=20000, rel_tol=1e-7)
    g.sim.set_tuning(2)  # streamed kernel
    g.step()
    assert g.sim.preconditioner()[3] == 0
    with pytest.raises(ValueError):
        g.sim.set_preconditioner("chebyshev", 4, 30.0)  # even degree
