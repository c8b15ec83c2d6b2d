"""GPU: the autotuner times every applicable solver configuration on the
current state without advancing the simulation, keeps the fastest, and the
tuned solver continues the same trajectory."""
import numpy as np
import pytest

from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("warm", ["zero", "previous"])
def test_autotune_restores_state_and_keeps_the_fastest(warm):
    sc = scenes.config_large(side=40, steps=6)
    g = GpuCloth(sc, max_iter=20000, rel_tol=1e-6, warm_start=warm)
    ref = GpuCloth(sc, max_iter=20000, rel_tol=1e-6, warm_start=warm)
    g.run(2)
    ref.run(2)
    p0, v0 = g.positions(), g.velocities()
    table = g.sim.autotune(sc["dt"], repetitions=1)
    # the simulation did not advance
    np.testing.assert_array_equal(g.positions(), p0)
    np.testing.assert_array_equal(g.velocities(), v0)
    kernels = {t["kernel"] for t in table}
    assert {"resident", "streamed", "loop"} <= kernels and len(table) >= 6
    assert all(t["status"] == capi.SOLVE_CONVERGED for t in table)
    best = min(table, key=lambda t: t["solve_ms"])
    g.step()
    assert g.sim.solver_info()[0] == best["kernel"]
    assert g.sim.sync_mode() == best["sync"]
    ref.step()
    for _ in range(3):
        g.step()
        ref.step()
    assert g.stats()[2] == capi.SOLVE_CONVERGED
    assert np.abs(g.positions() - ref.positions()).max() < 1e-4


def test_autotune_argument_checks():
    g = GpuCloth(scenes.config_small(steps=1), max_iter=100, rel_tol=1e-6, warm_start="zero")
    with pytest.raises(ValueError):
        g.sim.autotune(0.0)
    with pytest.raises(ValueError):
        g.sim.autotune(0.01, repetitions=0)
