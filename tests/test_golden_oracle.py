"""Pins the CPU oracle to the reference's own outputs (golden fixtures made
by running the compiled reference ClothSimulator on a B200): assembled
system, converged solution and trajectory, from the same states."""
import numpy as np
import pytest

import oracle.oracle as O
from golden_util import (DUMPS, TOL_BLOCK_REL, TOL_DX_CONVERGED, TOL_RHS_ABS, TOL_TRAJ, TRAJECTORIES, load,
                         rel, scene_for)


def oracle_from(sc, fx, pre, springs, fp64=True, tol=1e-12, iters=20000, warm="zero"):
    s = O.OracleCloth(fp64)
    s.set_material(sc["density"], 0.0, sc["gravity"])
    s.set_state(sc["pos"], sc["vel"], fx[pre + "inv_mass"])
    s.set_mesh(sc["tris"])
    s.set_options(springs, False, 1e-6)
    s.build_springs(float(sc["k_spring"]))
    s.build_stretch(float(sc["k_stretch"]))
    if sc.get("k_shear") is not None:
        s.build_shear(float(sc["k_shear"]))
    if sc.get("k_bend") is not None:
        s.build_bending(float(sc["k_bend"]))
    s.set_pins(sc["pin_idx"], sc["pin_targets"], sc["k_pin"])
    s.set_solver(iters, tol, warm)
    return s


def test_inverse_mass_matches_reference():
    for name in ("ref_grid10_springs.npz", "ref_grid16_springs.npz"):
        fx = load(name)
        sc = scene_for(name)
        pre = "it1000_" if "grid10" in name else ""
        s = O.OracleCloth(True)
        s.set_state(sc["pos"], sc["vel"])
        s.set_mesh(sc["tris"])
        np.testing.assert_allclose(s.redistribute_mass(sc["density"]), fx[pre + "inv_mass"], rtol=2e-6)


@pytest.mark.parametrize("fixture,pre,springs,steps,converged", DUMPS)
def test_oracle_system_matches_reference(fixture, pre, springs, steps, converged):
    fx = load(fixture)
    sc = scene_for(fixture)
    for k in steps:
        s = oracle_from(sc, fx, pre, springs)
        s.set_state(fx[f"{pre}s{k}_pos"], fx[f"{pre}s{k}_vel"], fx[pre + "inv_mass"])
        s.step(sc["dt"])
        diag, rp, col, vals, rhs, dx = s.dump_system()
        np.testing.assert_array_equal(rp, fx[f"{pre}s{k}_row_offsets"])
        np.testing.assert_array_equal(col, fx[f"{pre}s{k}_col_indices"])
        assert rel(fx[f"{pre}s{k}_diag"], diag) < TOL_BLOCK_REL
        assert rel(fx[f"{pre}s{k}_values"], vals) < TOL_BLOCK_REL
        assert np.abs(fx[f"{pre}s{k}_rhs"] - rhs).max() < TOL_RHS_ABS
        if converged:
            assert np.abs(fx[f"{pre}s{k}_dx"] - dx).max() < TOL_DX_CONVERGED


@pytest.mark.parametrize("fixture,pre,steps", TRAJECTORIES)
def test_oracle_trajectory_matches_reference(fixture, pre, steps):
    fx = load(fixture)
    sc = scene_for(fixture)
    for fp64 in (True, False):
        s = oracle_from(sc, fx, pre, True, fp64=fp64, tol=1e-10, iters=20000)
        for _ in range(steps):
            s.step(sc["dt"])
        assert np.abs(s.state()[0] - fx[pre + "final_pos"]).max() < TOL_TRAJ
