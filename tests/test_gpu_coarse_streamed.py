"""GPU: the streamed kernel's two-level preconditioner (block-Jacobi plus the
coarse level of translation and linear fields on blocks of ~5120 rows, A_c
inverted densely every step) against the FP64 oracle's restatement of the
same operator on the same blocks."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    O.set_threads(O.max_threads())
    yield


def gpu(sc, pc=True, warm="zero", tol=1e-6):
    g = GpuCloth(sc, max_iter=60000, rel_tol=tol, warm_start=warm)
    g.sim.set_tuning(2)  # the streamed kernel
    g.sim.set_row_order(1)
    if pc:
        g.sim.set_preconditioner("chebyshev_coarse", 7, 60.0)
    return g


def permuted(sc, order):
    """The scene renumbered in `order` (order[new] = old particle)."""
    inv = np.empty_like(order)
    inv[order] = np.arange(order.shape[0])
    out = dict(sc)
    out["pos"] = sc["pos"][order]
    out["vel"] = sc["vel"][order]
    out["tris"] = inv[sc["tris"]].astype(np.int32)
    out["pin_idx"] = inv[sc["pin_idx"]].astype(np.int32)
    e_new = scenes.unique_edges(out["tris"])
    if np.ndim(sc["k_spring"]):
        n = sc["pos"].shape[0]
        e_old = np.asarray(sc["edges"], np.int64)
        key = np.minimum(e_old[:, 0], e_old[:, 1]) * n + np.maximum(e_old[:, 0], e_old[:, 1])
        a, b = order[e_new[:, 0]], order[e_new[:, 1]]
        key_new = np.minimum(a, b) * n + np.maximum(a, b)
        srt = np.argsort(key)
        out["k_spring"] = np.asarray(sc["k_spring"], np.float32)[srt[np.searchsorted(key[srt], key_new)]]
    out["edges"] = e_new
    return out


def oracle_sim(sc, tol, coarse_rows=0, state=None):
    n = sc["pos"].shape[0]
    s = O.OracleCloth(True)
    s.set_material(sc["density"], sc.get("damping", 0.0), sc["gravity"])
    s.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    s.set_mesh(sc["tris"])
    s.set_options(True, False, sc.get("det_eps", 1e-6))
    im = s.redistribute_mass(sc["density"])
    s.set_state(sc["pos"], sc["vel"], im)
    s.build_springs(sc["k_spring"])
    s.build_stretch(sc["k_stretch"])
    s.set_pins(sc["pin_idx"], sc["pin_targets"], sc.get("k_pin", 1e6))
    if state is not None:  # the step from a given state, rest shapes from the scene's
        s.set_state(state[0], state[1], im)
    s.set_solver(400000, tol, "zero")
    if coarse_rows:
        s.set_preconditioner(0, 60.0, 512, "linear", coarse_rows)
    return s


def test_streamed_coarse_steps_match_fp64_oracle_and_its_iterations():
    # 192^2: 144 CTAs of 256 rows, coarse blocks of 20 CTAs = 5120 rows
    # (eight blocks, the last one of 4 CTAs), 96 unknowns
    sc = scenes.config_large(side=192)
    g = gpu(sc)
    n = sc["pos"].shape[0]
    errs, its, oits = [], [], []
    for _ in range(3):
        p0, v0 = g.positions().astype(np.float32), g.velocities().astype(np.float32)
        g.step()
        it, rr, st = g.stats()
        assert st == capi.SOLVE_CONVERGED and rr <= 1e-6
        assert g.sim.solver_info()[0] == "streamed" and g.sim.preconditioner()[3] == 3
        its.append(it)
        o = oracle_sim(sc, 1e-10, state=(p0, v0))
        o.step(sc["dt"])
        errs.append(float(np.abs(g.positions() - o.state()[0]).max()))
    # the same operator in the oracle, on the device's row blocks
    order = np.argsort(g.sim.row_of_particles(n))
    ps = permuted(sc, order)
    o = oracle_sim(ps, 1e-6, coarse_rows=5120)
    for _ in range(3):
        o.step(sc["dt"])
        oits.append(o.stats()[0])
    # the dense FP64 Gauss-Jordan inverse against the exact inverse of the
    # device's own A_c with its relative diagonal shift of 1e-5 (rows rounded
    # to FP32 once)
    info, ac, ainv = g.sim.debug_coarse()
    assert (info["on"], info["fields"], info["blocks"]) == (1, 4, 8)
    keep = np.diag(ac) != 0
    A = ac[np.ix_(keep, keep)].astype(np.float64)
    inv = np.linalg.inv(A + 1e-5 * np.diag(np.diag(A)))
    np.testing.assert_allclose(ainv[np.ix_(keep, keep)], inv, rtol=1e-4, atol=1e-6 * np.abs(inv).max())
    print(f"streamed two-level: one-step max|dx| vs FP64 {errs}, iterations {its}, oracle {oits}")
    assert max(errs) < 1e-5  # metres, as the benchmarked configurations
    for a, b in zip(its, oits):
        assert abs(a - b) <= 0.2 * b


def test_streamed_coarse_cuts_iterations_and_keeps_warm_starts_exact():
    sc = scenes.config_large(side=192)
    plain, two = gpu(sc, pc=False), gpu(sc)
    for _ in range(3):
        plain.step()
        two.step()
    assert two.sim.preconditioner()[3] == 3 and plain.sim.preconditioner()[3] == 0
    assert plain.stats()[0] > 3 * two.stats()[0]
    for warm in ("previous", "previous_scaled"):
        w = gpu(sc, warm=warm)
        for _ in range(3):
            p0, v0 = w.positions().astype(np.float32), w.velocities().astype(np.float32)
            w.step()
            assert w.stats()[2] == capi.SOLVE_CONVERGED
        o = oracle_sim(sc, 1e-10, state=(p0, v0))
        o.step(sc["dt"])
        assert np.abs(w.positions() - o.state()[0]).max() < 1e-5


def test_streamed_coarse_is_deterministic():
    sc = scenes.config_large(side=128)
    a, b = gpu(sc), gpu(sc)
    for _ in range(3):
        a.step()
        b.step()
    assert a.sim.preconditioner()[3] == 3
    assert np.array_equal(a.positions(), b.positions())
