"""Pins the oracle's contact terms to the reference's own outputs: fixtures
made by the compiled reference ClothSimulator on a B200 with static shapes
(plane + box, Coulomb friction) and with self-collision (its detector's
contact list recorded beside each dumped system).

From each recorded pre-step state the oracle assembles the same system
(diagonal incl. contact blocks, off-diagonal blocks, rhs incl. penalty,
lagged friction and the Coulomb projection) and solves it; the self-contact
step after a warm-started one uses the reference's own warm residual
(residual mode 1: the contact operator's off-diagonal part left out of
r0 = b - A x0, src/solver/pcg_solver.cu:512-513)."""
import numpy as np
import pytest

import oracle.oracle as O
from golden_util import (CONTACT_DUMPS, SELF_CONTACT, TOL_BLOCK_REL, TOL_DX_CONVERGED, grid10_contact, load,
                         rel, self_contacts, two_sheets)

# rhs of contact steps: penalty forces reach ~1e2 N, FP32 round-off ~1e-5 of that
TOL_RHS_REL = 2e-6


def oracle_for(sc, inv, tol=1e-12, iters=20000, warm="zero"):
    s = O.OracleCloth(True)
    s.set_material(sc["density"], 0.0, sc["gravity"])
    s.set_state(sc["pos"], sc["vel"], inv)
    s.set_mesh(sc["tris"])
    s.set_options(True, False, 1e-6)
    s.build_springs(float(sc["k_spring"]))
    s.build_stretch(float(sc["k_stretch"]))
    if len(sc["pin_idx"]):
        s.set_pins(sc["pin_idx"], sc["pin_targets"], sc["k_pin"])
    O.add_static_shapes(s, sc)
    s.set_solver(iters, tol, warm)
    return s


def check_system(fx, k, got, dx_tol=TOL_DX_CONVERGED, dx_rel=0.0):
    diag, rp, col, vals, rhs, dx = got
    np.testing.assert_array_equal(rp, fx[f"s{k}_row_offsets"])
    np.testing.assert_array_equal(col, fx[f"s{k}_col_indices"])
    assert rel(fx[f"s{k}_diag"], diag) < TOL_BLOCK_REL
    assert rel(fx[f"s{k}_values"], vals) < TOL_BLOCK_REL
    assert np.abs(fx[f"s{k}_rhs"] - rhs).max() <= TOL_RHS_REL * np.abs(rhs).max() + 5e-4
    if dx_tol is not None:
        assert np.abs(fx[f"s{k}_dx"] - dx).max() < dx_tol + dx_rel * np.abs(dx).max()


@pytest.mark.parametrize("fixture,steps", CONTACT_DUMPS)
def test_static_contact_system_matches_reference(fixture, steps):
    fx = load(fixture)
    sc = grid10_contact()
    touched = 0
    for k in steps:
        s = oracle_for(sc, fx["inv_mass"])
        s.set_state(fx[f"s{k}_pos"], fx[f"s{k}_vel"], fx["inv_mass"])
        s.step(sc["dt"])
        got = s.dump_system()
        check_system(fx, k, got)
        # the contact blocks are there: the diagonal exceeds inertia + elastic
        touched += int((fx[f"s{k}_pos"][:, 1] < 0.12).any())
    assert touched >= 3  # the dumped steps include contact, not only free fall


def test_self_contact_system_matches_reference():
    fixture, steps = SELF_CONTACT
    fx = load(fixture)
    sc = two_sheets()
    assert fx["s0_cpairs"].shape[0] > 50  # the sheets start in contact
    for k in steps:
        s = oracle_for(sc, fx["inv_mass"], warm="user")
        s.set_state(fx[f"s{k}_pos"], fx[f"s{k}_vel"], fx["inv_mass"])
        if k == 0:
            s.set_warm_guess(np.zeros_like(fx["s0_pos"], np.float64))
        elif f"s{k - 1}_dx" in fx:
            s.set_warm_guess(fx[f"s{k - 1}_dx"].astype(np.float64))
        s.set_contacts(**self_contacts(fx, k, sc), residual_mode=1)
        s.step(sc["dt"])
        known_guess = k == 0 or f"s{k - 1}_dx" in fx
        # the warm-started steps are metres long (next test); the FP32
        # reference and the FP64 oracle agree to ~2e-5 of the step there
        check_system(fx, k, s.dump_system(), dx_tol=TOL_DX_CONVERGED if known_guess else None, dx_rel=5e-5)


@pytest.mark.parametrize("k", [1, 2])
def test_self_contact_warm_residual_mode_matters(k):
    """The reference's warm-started steps solve (A + C) x = b + C_off x0:
    fed back through (A + C)^-1 C_off, the previous dx grows the step from
    3 mm (step 0, zero guess) to metres.  Residual mode 1 reproduces the
    reference; mode 0 (the full residual) keeps step 1 at the millimetre scale."""
    fixture, _ = SELF_CONTACT
    fx = load(fixture)
    sc = two_sheets()
    ref = np.abs(fx[f"s{k}_dx"]).max()
    assert ref > 100 * np.abs(fx["s0_dx"]).max()
    out = {}
    for mode in (0, 1):
        s = oracle_for(sc, fx["inv_mass"], warm="user")
        s.set_state(fx[f"s{k}_pos"], fx[f"s{k}_vel"], fx["inv_mass"])
        s.set_warm_guess(fx[f"s{k - 1}_dx"].astype(np.float64))
        s.set_contacts(**self_contacts(fx, k, sc), residual_mode=mode)
        s.step(sc["dt"])
        dx = s.dump_system()[5]
        out[mode] = (np.abs(dx - fx[f"s{k}_dx"]).max(), np.abs(dx).max())
    assert out[1][0] < 5e-5 * ref
    assert out[0][0] > 0.1 * ref
    if k == 1:  # from the sane state of step 1; step 2 starts from the reference's blown-up state
        assert out[0][1] < 0.05
