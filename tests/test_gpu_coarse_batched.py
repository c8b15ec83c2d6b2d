"""GPU: the streamed kernel's coarse level for batches (coarse blocks inside
instances, one per CTA segment of an instance or a run of them, at most 8 per
instance: translation and linear fields, A_c block-diagonal by instance, each
instance's dense inverse formed on its own) on zero-guess solves of several
instances: the converged states against the block-Jacobi batch and the FP64
oracle, the iteration counts against the oracle's restatement of the same
operator on the device's blocks per instance, the per-instance inverses
against the exact inverses of the device's own matrices, and bitwise
repeatability."""
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


def packed(count, seed, lo, hi):
    inst = scenes.batch_instances(count=count, seed=seed, lo=lo, hi=hi, steps=4, max_iter=60000)
    sc, offs = scenes.concat(inst)
    return inst, sc, offs


def batch(sc, offs, pc=True, warm="zero", tol=1e-7):
    g = GpuCloth(sc, max_iter=60000, rel_tol=tol, warm_start=warm, instances=offs)
    g.sim.set_tuning(2)  # the streamed kernel
    if pc:
        g.sim.set_preconditioner("chebyshev_coarse", 7, 60.0)
    return g


def inst_rows(offs):
    """First internal row of every instance (each starts on a fresh 32-row
    slice), and the padded total."""
    n = np.diff(np.asarray(offs, np.int64))
    return np.concatenate([[0], np.cumsum((n + 31) // 32 * 32)])


def inst_bounds(g, offs):
    """Per instance, the device's coarse block starts relative to the
    instance's first row (ending with its row count)."""
    rows = g.sim.debug_coarse_rows()
    r0 = inst_rows(offs)
    out = []
    for b in range(len(offs) - 1):
        starts = [int(r) - int(r0[b]) for r in rows[:-1] if r0[b] <= r < r0[b + 1]]
        out.append(starts + [int(offs[b + 1] - offs[b])])
    return out


def oracle_inst(sc, tol, state, coarse):
    """One instance's step from `state` in the FP64 oracle; `coarse`: None,
    or the restatement of the batched level on the given block starts
    (block-Jacobi plus translation and linear fields per block)."""
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
    s.set_state(state[0], state[1], im)
    s.set_solver(400000, tol, "zero")
    if coarse is not None:
        s.set_preconditioner(0, 60.0, 512, "linear", 0)
        s.set_coarse_bounds(coarse)
    return s


def test_batched_coarse_matches_oracle_and_its_iterations():
    # six instances of 24^2..64^2 particles (ragged: padding rows inside the
    # batch), three steps
    inst, sc, offs = packed(6, seed=21, lo=24, hi=64)
    g = batch(sc, offs)
    errs, bad = [], []
    for step in range(3):
        p0, v0 = g.positions().astype(np.float32), g.velocities().astype(np.float32)
        g.step()
        assert g.sim.solver_info()[0] == "streamed" and g.sim.preconditioner()[3] == 3
        it, rr, st = g.sim.instance_stats()
        assert (st == capi.SOLVE_CONVERGED).all() and (rr <= 1e-7).all()
        pos = g.positions()
        bounds = inst_bounds(g, offs)
        for b, s in enumerate(inst):
            a, e = int(offs[b]), int(offs[b + 1])
            state = (p0[a:e], v0[a:e])
            o = oracle_inst(s, 1e-11, state, coarse=None)
            o.step(s["dt"])
            errs.append(float(np.abs(pos[a:e] - o.state()[0]).max()))
            if step > 0:  # from rest the first step converges in a handful of iterations
                c = oracle_inst(s, 1e-7, state, coarse=bounds[b])
                c.step(s["dt"])
                ci = c.stats()[0]
                if abs(int(it[b]) - ci) > 0.25 * ci + 3:
                    bad.append((step, b, int(it[b]), ci))
    print(f"batched two-level: blocks per instance {[len(x) - 1 for x in bounds]}, max|dx| vs FP64 "
          f"{max(errs):.3g}, iteration mismatches {bad}")
    assert max(len(x) - 1 for x in bounds) > 1  # blocks inside instances
    assert max(errs) < 1e-5
    assert not bad


def test_batched_coarse_cuts_iterations():
    inst, sc, offs = packed(8, seed=22, lo=32, hi=96)
    plain, two = batch(sc, offs, pc=False), batch(sc, offs)
    errs = {}
    for step in range(3):
        for name, g in (("plain", plain), ("two", two)):
            p0, v0 = g.positions().astype(np.float32), g.velocities().astype(np.float32)
            g.step()
            assert (g.sim.instance_stats()[2] == capi.SOLVE_CONVERGED).all()
            if step == 2:  # the last step of each against the FP64 oracle from its own state
                pos = g.positions()
                errs[name] = max(
                    float(np.abs(pos[offs[b]:offs[b + 1]] - _oracle_step(s, p0, v0, offs, b)).max())
                    for b, s in enumerate(inst))
    assert two.sim.preconditioner()[3] == 3 and plain.sim.preconditioner()[3] == 0
    ip, it = plain.sim.instance_stats()[0], two.sim.instance_stats()[0]
    big = np.argmax(offs[1:] - offs[:-1])
    print(f"iterations block-Jacobi {ip.tolist()}, two-level {it.tolist()}, one-step errors {errs}")
    assert it[big] < 0.6 * ip[big], (it, ip)
    assert it.max() < 0.6 * ip.max()
    # both solves stop at the same relative residual; the two-level state is
    # as close to the FP64 solution as the block-Jacobi one
    assert errs["two"] <= max(3.0 * errs["plain"], 2e-5)


def _oracle_step(s, p0, v0, offs, b):
    a, e = int(offs[b]), int(offs[b + 1])
    o = oracle_inst(s, 1e-11, (p0[a:e], v0[a:e]), coarse=None)
    o.step(s["dt"])
    return o.state()[0]


def test_batched_coarse_inverse_blocks():
    inst, sc, offs = packed(5, seed=23, lo=20, hi=48)
    g = batch(sc, offs)
    for _ in range(2):
        g.step()
    info, ac, ainv = g.sim.debug_coarse()
    rows = g.sim.debug_coarse_rows()
    assert (info["on"], info["fields"], info["blocks"]) == (1, 4, len(rows) - 1)
    r0 = inst_rows(offs)
    nblk = [int(((rows[:-1] >= r0[b]) & (rows[:-1] < r0[b + 1])).sum()) for b in range(5)]
    assert sum(nblk) == info["blocks"] and 1 <= max(nblk) <= 12
    first = np.concatenate([[0], np.cumsum(nblk)])
    for b in range(5):
        sl = slice(12 * first[b], 12 * first[b + 1])
        A = ac[sl, sl].astype(np.float64)
        assert np.all(ac[sl, :sl.start] == 0) and np.all(ac[sl, sl.stop:] == 0)
        assert np.all(ainv[sl, :sl.start] == 0) and np.all(ainv[sl, sl.stop:] == 0)
        keep = np.diag(A) != 0
        Ak = A[np.ix_(keep, keep)]
        inv = np.linalg.inv(Ak + 1e-5 * np.diag(np.diag(Ak)))
        np.testing.assert_allclose(ainv[sl, sl][np.ix_(keep, keep)], inv, rtol=1e-4, atol=1e-6 * np.abs(inv).max())


def test_batched_coarse_is_deterministic_and_needs_the_zero_guess():
    inst, sc, offs = packed(4, seed=24, lo=24, hi=48)
    a, b = batch(sc, offs), batch(sc, offs)
    for _ in range(3):
        a.step()
        b.step()
    assert np.array_equal(a.positions(), b.positions())
    # warm starts keep block-Jacobi on batches
    w = batch(sc, offs, warm="previous")
    w.step()
    assert w.sim.preconditioner()[3] == 0
    assert (w.sim.instance_stats()[2] == capi.SOLVE_CONVERGED).all()
