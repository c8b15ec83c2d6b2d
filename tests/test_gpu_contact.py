"""GPU parity of the contact terms against the CPU oracle, through the C ABI.

Static shapes (planes, boxes, Coulomb friction) are row-local terms of the
fused assembly; the contact operator is a device-resident contact list whose
per-row slot lists the step rebuilds every frame and whose off-diagonal
blocks ride inside the solver SpMVs.

Tolerances: FP32 assembly against the FP64 oracle (relative 2e-6 on the
system blocks); converged solves at rel-res 1e-8 agree to ~1e-7 m.  With
friction the stick / slip switch of the Coulomb cone makes trajectories
chaotic (the FP32 oracle leaves the FP64 one by centimetres within 20 steps
of this scene), so friction is checked step by step from the GPU's own
state; the frictionless trajectory is compared over the whole drop (the FP32
/ FP64 oracle spread there is 7e-4 m).
"""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu

PATHS = [0, 1, 2]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    yield


def make(sc, path=0, **kw):
    g = GpuCloth(sc, **kw)
    g.sim.set_tuning(path)
    return g


def oracle_sim(sc, tol=1e-10, max_iter=20000, warm="zero", fp64=True):
    n = sc["pos"].shape[0]
    s = O.OracleCloth(fp64)
    s.set_material(sc["density"], sc.get("damping", 0.0), sc["gravity"])
    s.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    s.set_mesh(sc["tris"])
    im = s.redistribute_mass(sc["density"])
    s.set_state(sc["pos"], sc["vel"], im)
    if sc.get("k_spring") is not None:
        s.build_springs(sc["k_spring"])
    if sc.get("k_stretch") is not None:
        s.build_stretch(sc["k_stretch"])
    if len(sc["pin_idx"]):
        s.set_pins(sc["pin_idx"], sc["pin_targets"], sc.get("k_pin", 1e6))
    O.add_static_shapes(s, sc)
    s.set_solver(max_iter, tol, warm)
    return s


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def compare_step(g, sc, inv, tol_blocks=2e-6, tol_rhs=1e-5, tol_dx=2e-5, contacts=None):
    """Steps the GPU once and an oracle set to the GPU's state; compares."""
    one = oracle_sim(sc)
    one.set_state(g.positions().astype(np.float32), g.velocities().astype(np.float32), inv)
    if contacts is not None:
        one.set_contacts(**contacts)
    one.step(sc["dt"])
    g.step()
    diag, rp, col, vals, rhs, dx = g.dump()
    od, orp, ocol, ovals, orhs, odx = one.dump_system()
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert rel(diag, od) < tol_blocks
    assert rel(vals, ovals) < tol_blocks
    # relative to the largest force, plus the FP32 round-off of near-zero
    # elastic forces at rest (5e-4 N, as in the contact-free parity tests)
    assert np.abs(rhs - orhs).max() <= tol_rhs * np.abs(orhs).max() + 5e-4
    assert np.abs(dx - odx).max() < tol_dx
    return one


@pytest.mark.parametrize("path", PATHS)
def test_static_contact_frictionless_trajectory(path):
    sc = scenes.config_contact(friction=0.0)
    g = make(sc, path, max_iter=20000, rel_tol=1e-8)
    o = oracle_sim(sc, tol=1e-10)
    for _ in range(sc["steps"]):
        g.step()
        o.step(sc["dt"])
        assert g.stats()[2] == capi.SOLVE_CONVERGED
    p, _ = o.state()
    assert np.abs(g.positions() - p).max() < 2e-3
    # it did land: the centre rests on the table top, the rim lower
    y = g.positions()[:, 1]
    assert y.min() < 0.1 and y.max() < 0.16


@pytest.mark.parametrize("path", PATHS)
def test_static_contact_friction_system_matches_oracle(path):
    sc = scenes.config_contact(friction=0.3)
    g = make(sc, path, max_iter=20000, rel_tol=1e-8)
    inv = g.inv_mass.cpu().numpy()
    o = oracle_sim(sc, tol=1e-10)
    for k in range(30):
        if k in (8, 14, 22, 29):  # falling, first contact, sliding, settling
            compare_step(g, sc, inv)
        else:
            g.step()
        o.step(sc["dt"])
        if k == 11:
            # before the cone starts switching the runs stay together
            assert np.abs(g.positions() - o.state()[0]).max() < 1e-3


def test_static_contact_pybind_facade_matches_capi():
    sc = scenes.config_contact(friction=0.3, steps=12)
    a = make(sc, 0, max_iter=20000, rel_tol=1e-8)
    b = GpuCloth(sc, max_iter=20000, rel_tol=1e-8, api="pybind")
    assert b.sim.static_plane_count() == 1 and b.sim.static_box_count() == 1
    assert b.sim.static_contact_friction() == pytest.approx(0.3)
    for _ in range(12):
        a.step()
        b.step()
    np.testing.assert_array_equal(a.positions(), b.positions())


def test_static_shape_changes_take_effect():
    sc = scenes.config_contact(friction=0.0, steps=20)
    g = make(sc, 0, max_iter=20000, rel_tol=1e-8)
    g.run(12, record_iters=False)
    g.sim.clear_static_shapes()
    assert g.sim.static_shape_counts() == (0, 0)
    o = oracle_sim(dict(sc, planes=[], boxes=[]))
    inv = g.inv_mass.cpu().numpy()
    o.set_state(g.positions().astype(np.float32), g.velocities().astype(np.float32), inv)
    g.step()
    o.step(sc["dt"])
    assert np.abs(g.positions() - o.state()[0]).max() < 1e-6
    assert g.sim.static_contact() == pytest.approx((0.01, 1.0e4, 0.0, 1.0e-4))


# ---------------------------------------------------------------------------
# contact operator
# ---------------------------------------------------------------------------

def contact_list(n, m, seed, depth=0.002, bad=None):
    rng = np.random.default_rng(seed)
    pairs = np.stack([rng.choice(n, 4, replace=False) for _ in range(m)]).astype(np.int32)
    b = rng.dirichlet(np.ones(3), m)
    w = np.concatenate([np.ones((m, 1)), -b], 1)
    nrm = rng.normal(size=(m, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    weights = np.concatenate([w, nrm, rng.uniform(0.5, 1.5, (m, 1)) * depth], 1).astype(np.float32)
    u = rng.normal(scale=2e-4, size=(m, 3))
    slips = np.concatenate([u, np.linalg.norm(u, axis=1, keepdims=True)], 1).astype(np.float32)
    ks = rng.uniform(2e3, 6e3, m).astype(np.float32)
    if bad is not None:
        pairs[bad, 2] = n + 3  # out of range with a non-zero weight: dropped
    return pairs, weights, slips, ks


class DeviceContacts:
    def __init__(self, pairs, weights, slips, ks, count):
        import torch

        self.pairs = torch.from_numpy(pairs).cuda()
        self.weights = torch.from_numpy(weights).cuda()
        self.slips = torch.from_numpy(slips).cuda()
        self.ks = torch.from_numpy(ks).cuda()
        self.count = torch.tensor([count], dtype=torch.int32, device="cuda")
        self.m = pairs.shape[0]

    def attach(self, sim, stiffness=4.0e3, per_contact=False, mu=0.0, mode=0, slips=True):
        sim.set_contact_op(self.pairs.data_ptr(), self.weights.data_ptr(), self.count.data_ptr(), self.m,
                           stiffness, self.ks.data_ptr() if per_contact else 0,
                           self.slips.data_ptr() if slips else 0, mu, 1.0e-4, mode)


def oracle_contacts(pairs, weights, slips, ks, count, stiffness=4.0e3, per_contact=False, mu=0.0, mode=0,
                    n=None):
    keep = np.arange(pairs.shape[0]) < count
    if n is not None:
        keep &= ((pairs >= 0) & (pairs < n)).all(1)
    return dict(pairs=pairs[keep], weights=weights[keep], stiffness=stiffness,
                stiffnesses=ks[keep] if per_contact else None, slips=slips[keep], friction=mu,
                residual_mode=mode)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("per_contact,mu", [(False, 0.0), (True, 0.25)])
def test_contact_operator_system_and_solve_match_oracle(path, per_contact, mu):
    sc = scenes.config_small(steps=10)
    n = sc["pos"].shape[0]
    pairs, weights, slips, ks = contact_list(n, 40, seed=11, bad=7)
    dc = DeviceContacts(pairs, weights, slips, ks, count=35)
    g = make(sc, path, max_iter=20000, rel_tol=1e-8)
    dc.attach(g.sim, per_contact=per_contact, mu=mu)
    inv = g.inv_mass.cpu().numpy()
    oc = oracle_contacts(pairs, weights, slips, ks, 35, per_contact=per_contact, mu=mu, n=n)
    for k in range(3):
        compare_step(g, sc, inv, contacts=oc)
        assert g.stats()[2] == capi.SOLVE_CONVERGED
    live, dropped, slots = g.sim.contact_stats()
    assert (live, dropped) == (35, 1)
    assert slots == 4 * 34  # every weight of the generated contacts is non-zero
    info = g.sim.solver_info()
    assert info[0] == ("loop" if path == 1 else "streamed")  # no register-resident kernel with contacts


@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("mode", [0, 1])
def test_contact_operator_warm_residual_modes(path, mode):
    """From the previous step's dx: mode 0 solves (A + C) x = b, mode 1 the
    reference's (A + C) x = b + C_off x0; both as the oracle.  Mode 1 feeds
    the previous dx back through (A + C)^-1 C_off, which grows it when the
    contacts dominate (here by ~470x per step), so it is compared on the
    first chained step, relative to that step's size."""
    sc = scenes.config_small(steps=10)
    n = sc["pos"].shape[0]
    pairs, weights, slips, ks = contact_list(n, 30, seed=12)
    dc = DeviceContacts(pairs, weights, slips, ks, count=30)
    g = make(sc, path, max_iter=20000, rel_tol=1e-9, warm_start="previous")
    dc.attach(g.sim, mode=mode, mu=0.2)
    o = oracle_sim(sc, tol=1e-11, warm="previous")
    o.set_contacts(**oracle_contacts(pairs, weights, slips, ks, 30, mu=0.2, mode=mode))
    sizes = []
    for _ in range(4 if mode == 0 else 2):
        g.step()
        o.step(sc["dt"])
        sizes.append(np.abs(o.dump_system()[5]).max())
    dx = g.dump()[5]
    odx = o.dump_system()[5]
    if mode == 0:
        assert np.abs(dx - odx).max() < 2e-5
        assert np.abs(g.positions() - o.state()[0]).max() < 2e-5
    else:
        assert sizes[1] > 10 * sizes[0]
        assert np.abs(dx - odx).max() < 2e-3 * sizes[1]


def test_contact_count_changes_without_a_new_operator():
    import torch

    sc = scenes.config_small(steps=10)
    n = sc["pos"].shape[0]
    pairs, weights, slips, ks = contact_list(n, 24, seed=13)
    dc = DeviceContacts(pairs, weights, slips, ks, count=24)
    g = make(sc, 0, max_iter=20000, rel_tol=1e-8)
    dc.attach(g.sim)
    inv = g.inv_mass.cpu().numpy()
    for count in (24, 9, 0, 17, 40):  # 40 > max_contacts: clamped to 24
        dc.count.fill_(count)
        torch.cuda.synchronize()
        compare_step(g, sc, inv, contacts=oracle_contacts(pairs, weights, slips, ks, min(count, 24)))
        assert g.sim.contact_stats()[0] == min(count, 24)


def test_contact_operator_is_deterministic():
    sc = scenes.config_small(steps=10)
    n = sc["pos"].shape[0]
    pairs, weights, slips, ks = contact_list(n, 64, seed=14)
    runs = []
    for _ in range(2):
        dc = DeviceContacts(pairs, weights, slips, ks, count=64)
        g = make(sc, 0, max_iter=300, rel_tol=0.0)
        dc.attach(g.sim, mu=0.3)
        g.run(3, record_iters=False)
        runs.append((g.positions(), g.dump()[0]))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_contact_operator_rejects_misaligned_buffers_and_instances():
    sc = scenes.config_small(steps=10)
    n = sc["pos"].shape[0]
    pairs, weights, slips, ks = contact_list(n, 8, seed=15)
    dc = DeviceContacts(pairs, weights, slips, ks, count=8)
    g = make(sc, 0)
    with pytest.raises(ValueError):
        g.sim.set_contact_op(dc.pairs.data_ptr() + 4, dc.weights.data_ptr(), dc.count.data_ptr(), 8, 1.0)
    with pytest.raises(ValueError):
        g.sim.set_contact_op(dc.pairs.data_ptr(), dc.weights.data_ptr(), dc.count.data_ptr(), 8, 1.0,
                             residual_mode=2)
    g.sim.set_instances([0, n])
    dc.attach(g.sim)
    with pytest.raises(ValueError):
        g.step()
    g.sim.clear_contact_op()
    g.step()
