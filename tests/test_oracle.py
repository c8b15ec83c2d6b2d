"""CPU tests of the oracle itself: analytic known-answer tests, finite
differences, PSD filtering, and whole-step sanity.  These pin the oracle's
element formulas independently of any GPU run."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import scenes


def test_spring_known_answer_stretched():
    # one spring along x stretched from L=1 to l=1.5, k=100
    x = np.array([1.5, 0, 0, 0, 0, 0.0])
    E, g, H = O.spring_eval(x, 1.0, 100.0)
    assert E == pytest.approx(0.5 * 100 * 0.25)
    np.testing.assert_allclose(g, [50, 0, 0, -50, 0, 0], atol=1e-12)
    # stretched branch: (k - kL/l) I + (kL/l) d d^T, d = x-axis
    a = 100 * 1.0 / 1.5
    Hb = np.diag([100.0, 100 - a, 100 - a])
    np.testing.assert_allclose(H[:3, :3], Hb, atol=1e-12)
    np.testing.assert_allclose(H[:3, 3:], -Hb, atol=1e-12)


def test_spring_known_answer_compressed_is_rank_one():
    x = np.array([0.5, 0, 0, 0, 0, 0.0])
    _, g, H = O.spring_eval(x, 1.0, 100.0)
    np.testing.assert_allclose(g[:3], [-50, 0, 0], atol=1e-12)
    a = 100 * 1.0 / 0.5
    np.testing.assert_allclose(H[:3, :3], np.diag([a, 0, 0]), atol=1e-12)
    assert np.linalg.eigvalsh(H).min() > -1e-9


def test_rest_shape_known_answer():
    # right triangle with legs 2 (along x) and 3 (along y)
    x = np.array([0, 0, 0, 2, 0, 0, 0, 3, 0.0])
    dm, area = O.rest_shape(x)
    assert area == pytest.approx(3.0)
    # Dm = [[2, 0], [0, 3]] -> inverse diag(1/2, 1/3)
    np.testing.assert_allclose(dm, [0.5, 0, 0, 1.0 / 3.0], atol=1e-14)


def test_rest_shape_degenerate_uses_identity():
    x = np.array([0, 0, 0, 1e-4, 0, 0, 0, 1e-4, 0.0])  # lab*v_c = 1e-8 <= 1e-6
    dm, area = O.rest_shape(x)
    np.testing.assert_allclose(dm, [1, 0, 0, 1])
    dm2, _ = O.rest_shape(x, det_eps=1e-12)
    np.testing.assert_allclose(dm2, [1e4, 0, 0, 1e4], rtol=1e-12)


def test_triangle_uniform_stretch_known_answer():
    # rest: legs 1,1; deformed: uniform stretch s along u only
    x0 = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0.0])
    dm, area = O.rest_shape(x0)
    s = 1.2
    x = x0.copy()
    x[3] *= s  # vertex 1 moved along u
    k = 7.0
    E, g, H = O.triangle_eval(x, dm, area, k)
    # wu = s * e_x, wv = e_y: cu = s - 1, cv = 0
    assert E == pytest.approx(0.5 * k * area * (s - 1) ** 2)
    # gradient: k_eff * cu * dwu[a] * e_x with dwu = (-1, 1, 0)
    ge = k * area * (s - 1)
    np.testing.assert_allclose(g, [-ge, 0, 0, ge, 0, 0, 0, 0, 0], atol=1e-12)


def _random_tri(rng, stretch):
    x0 = rng.normal(size=9)
    dm, area = O.rest_shape(x0)
    x = x0 * stretch + rng.normal(scale=0.01, size=9)
    return x, dm, area


@pytest.mark.parametrize("seed", range(5))
def test_triangle_gradient_matches_finite_differences(seed):
    rng = np.random.default_rng(seed)
    x, dm, area = _random_tri(rng, 1.3)
    k = 3.0
    _, g, _ = O.triangle_eval(x, dm, area, k)
    h = 1e-6
    fd = np.zeros(9)
    for q in range(9):
        xp, xm = x.copy(), x.copy()
        xp[q] += h
        xm[q] -= h
        fd[q] = (O.triangle_eval(xp, dm, area, k)[0] - O.triangle_eval(xm, dm, area, k)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-8)


@pytest.mark.parametrize("seed", range(5))
def test_triangle_hessian_matches_fd_when_stretched(seed):
    # both cu > 0 and cv > 0: the filtered Hessian is the exact one
    rng = np.random.default_rng(100 + seed)
    x, dm, area = _random_tri(rng, 1.4)
    k = 2.0
    _, g0, H = O.triangle_eval(x, dm, area, k)
    h = 1e-6
    fd = np.zeros((9, 9))
    for q in range(9):
        xp, xm = x.copy(), x.copy()
        xp[q] += h
        xm[q] -= h
        fd[:, q] = (O.triangle_eval(xp, dm, area, k)[1] - O.triangle_eval(xm, dm, area, k)[1]) / (2 * h)
    np.testing.assert_allclose(H, fd, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(H, H.T, atol=1e-12)


@pytest.mark.parametrize("seed", range(10))
def test_element_hessians_are_psd(seed):
    rng = np.random.default_rng(200 + seed)
    x, dm, area = _random_tri(rng, rng.uniform(0.5, 1.5))
    _, _, H = O.triangle_eval(x, dm, area, 5.0)
    assert np.linalg.eigvalsh(0.5 * (H + H.T)).min() > -1e-9 * np.abs(H).max()
    xs = rng.normal(size=6)
    _, _, Hs = O.spring_eval(xs, rng.uniform(0.2, 3.0), 10.0)
    assert np.linalg.eigvalsh(Hs).min() > -1e-9 * np.abs(Hs).max()


@pytest.mark.parametrize("seed", range(3))
def test_spring_gradient_and_hessian_fd(seed):
    rng = np.random.default_rng(300 + seed)
    x = rng.normal(size=6)
    L = 0.5 * np.linalg.norm(x[:3] - x[3:])  # stretched
    k = 4.0
    _, g, H = O.spring_eval(x, L, k)
    h = 1e-6
    for q in range(6):
        xp, xm = x.copy(), x.copy()
        xp[q] += h
        xm[q] -= h
        assert g[q] == pytest.approx((O.spring_eval(xp, L, k)[0] - O.spring_eval(xm, L, k)[0]) / (2 * h), rel=1e-6, abs=1e-8)
        np.testing.assert_allclose(H[:, q], (O.spring_eval(xp, L, k)[1] - O.spring_eval(xm, L, k)[1]) / (2 * h),
                                   rtol=1e-5, atol=1e-6)


def _dense(diag, rp, col, vals):
    n = diag.shape[0]
    A = np.zeros((3 * n, 3 * n))
    for i in range(n):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] = diag[i]
        for k in range(rp[i], rp[i + 1]):
            A[3 * i:3 * i + 3, 3 * col[k]:3 * col[k] + 3] = vals[k]
    return A


def _oracle_sim(sc, fp64=True, tol=1e-10, max_iter=5000, warm="zero"):
    n = sc["pos"].shape[0]
    sim = O.OracleCloth(fp64)
    sim.set_material(sc["density"], 0.0, sc["gravity"])
    sim.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    sim.set_mesh(sc["tris"])
    sim.set_options(True, False, sc.get("det_eps", 1e-6))
    im = sim.redistribute_mass(sc["density"])
    sim.set_state(sc["pos"], sc["vel"], im)
    sim.build_springs(sc["k_spring"])
    sim.build_stretch(sc["k_stretch"])
    sim.set_pins(sc["pin_idx"], sc["pin_targets"])
    sim.set_solver(max_iter, tol, warm)
    return sim


def test_assembled_system_is_symmetric_and_solved():
    sc = scenes.config_small(side=6)
    sim = _oracle_sim(sc)
    for _ in range(5):
        sim.step(sc["dt"])
    diag, rp, col, vals, rhs, dx = sim.dump_system()
    A = _dense(diag, rp, col, vals)
    np.testing.assert_allclose(A, A.T, atol=1e-9 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0
    r = rhs.ravel() - A @ dx.ravel()
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(rhs)
    # the oracle's SpMV agrees with the dense product
    x = np.random.default_rng(0).normal(size=dx.shape)
    np.testing.assert_allclose(sim.spmv(x).ravel(), A @ x.ravel(), rtol=1e-12, atol=1e-9)


def test_scaled_warm_start_minimises_energy_along_the_guess():
    """previous_scaled starts from c x0 with c = x0.b / x0.A x0: its energy
    1/2 x.A x - b.x is at or below both the unscaled guess's and the zero
    guess's (0).  Checked by stopping the solve at 0 iterations."""
    sc = scenes.config_small(side=8)
    starts = {}
    for mode in ("previous", "previous_scaled"):
        sim = _oracle_sim(sc, tol=1e-10, max_iter=5000, warm="previous")
        for _ in range(6):
            sim.step(sc["dt"])
        sim.set_solver(0, 0.0, mode)
        sim.step(sc["dt"])
        diag, rp, col, vals, rhs, dx = sim.dump_system()
        starts[mode] = (_dense(diag, rp, col, vals), rhs.ravel(), dx.ravel())
    A, b, x0 = starts["previous"]
    A2, b2, xs = starts["previous_scaled"]
    np.testing.assert_array_equal(A, A2)
    np.testing.assert_array_equal(b, b2)

    def energy(x):
        return 0.5 * x @ (A @ x) - b @ x

    c = (x0 @ b) / (x0 @ (A @ x0))
    np.testing.assert_allclose(xs, max(c, 0.0) * x0, rtol=1e-12, atol=1e-300)
    assert energy(xs) <= energy(x0) + 1e-15 * abs(energy(x0))
    assert energy(xs) <= 1e-15 * abs(energy(x0))


def _shear_sim(sc, shear_as_stretch):
    """Springs + a Baraff-Witkin set turned by pi/4: either through the shear
    entry point, or as the stretch set built with theta = pi/4."""
    n = sc["pos"].shape[0]
    sim = O.OracleCloth(True)
    sim.set_material(sc["density"], 0.0, sc["gravity"])
    sim.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    sim.set_mesh(sc["tris"])
    sim.set_options(True, False, 1e-6)
    im = sim.redistribute_mass(sc["density"])
    sim.set_state(sc["pos"], sc["vel"], im)
    sim.build_springs(sc["k_spring"])
    if shear_as_stretch:
        sim.build_stretch(4.0e3, theta=float(np.float32(np.pi / 4)))
    else:
        sim.build_shear(4.0e3)
    sim.set_pins(sc["pin_idx"], sc["pin_targets"])
    sim.set_solver(5000, 1e-10, "zero")
    return sim


def test_shear_set_is_the_stretch_element_turned_by_a_quarter_turn():
    # cloth_simulator.cu:423-449: shear = stretch energy on rest axes turned by pi/4
    sc = scenes.config_small(side=6)
    a, b = _shear_sim(sc, False), _shear_sim(sc, True)
    for _ in range(4):
        a.step(sc["dt"])
        b.step(sc["dt"])
    for x, y in zip(a.dump_system(), b.dump_system()):
        np.testing.assert_array_equal(x, y)


def test_shear_resists_pure_shear_that_stretch_ignores():
    # unit right triangle, simple shear x' = x + g y: the axis-aligned stretch
    # element sees |F e_u| = 1, |F e_v| = sqrt(1 + g^2) > 1; the quarter-turned
    # one sees both diagonals change length, so its energy is larger and its
    # gradient pulls the sheared vertex back
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)
    g = 0.2
    y = x.copy()
    y[2, 0] += g
    dm0, a0 = O.rest_shape(x, 1e-6, 0.0)
    dm4, a4 = O.rest_shape(x, 1e-6, float(np.pi / 4))
    e0, g0, _ = O.triangle_eval(y, dm0, a0, 1.0)
    e4, g4, _ = O.triangle_eval(y, dm4, a4, 1.0)
    lu = np.hypot(1 + 0.0, 0.0)
    lv = np.hypot(g, 1.0)
    assert e0 == pytest.approx(0.5 * a0 * (lu - 1) ** 2 + 0.5 * a0 * (lv - 1) ** 2, rel=1e-9)
    d1 = np.linalg.norm((y[1] - y[0]) / np.sqrt(2) + (y[2] - y[0]) / np.sqrt(2))
    d2 = np.linalg.norm(-(y[1] - y[0]) / np.sqrt(2) + (y[2] - y[0]) / np.sqrt(2))
    assert e4 == pytest.approx(0.5 * a4 * ((d1 - 1) ** 2 + (d2 - 1) ** 2), rel=1e-9)
    assert e4 > e0 and np.asarray(g4).reshape(3, 3)[2, 0] > 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bending_element_matches_finite_differences(seed):
    # bending_constraint.cu:46-123: theta and its shape vectors a_i = d theta / d x_i
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(12) * 0.5
    k, th0 = 2.0, 0.3
    e, g, h = O.bending_eval(x, k, th0)
    th = O.bending_angle(x)
    assert e == pytest.approx(0.5 * k * (th - th0) ** 2, rel=1e-12)
    eps = 1e-6
    fd_e = np.zeros(12)
    fd_th = np.zeros(12)
    for i in range(12):
        xp, xm = x.copy(), x.copy()
        xp[i] += eps
        xm[i] -= eps
        fd_e[i] = (O.bending_eval(xp, k, th0)[0] - O.bending_eval(xm, k, th0)[0]) / (2 * eps)
        fd_th[i] = (O.bending_angle(xp) - O.bending_angle(xm)) / (2 * eps)
    np.testing.assert_allclose(g, fd_e, atol=1e-7 * max(1.0, np.abs(g).max()))
    # Gauss-Newton Hessian k a a^T with a = d theta / d x
    np.testing.assert_allclose(h, k * np.outer(fd_th, fd_th), atol=1e-6 * max(1.0, np.abs(h).max()))
    # the off-diagonal blocks of one dihedral are not symmetric in general
    assert np.abs(h[0:3, 6:9] - h[0:3, 6:9].T).max() > 1e-3 * np.abs(h).max()


def test_dihedrals_are_the_interior_edges_of_the_mesh():
    sc = scenes.config_small(side=5)
    sim = O.OracleCloth(True)
    sim.set_state(sc["pos"], sc["vel"])
    sim.set_mesh(sc["tris"])
    sim.build_bending(1e-3)
    tris = sc["tris"]
    edges = sc["edges"]
    count = {tuple(e): 0 for e in edges}
    for t in tris:
        for a in range(3):
            u, v = sorted((int(t[a]), int(t[(a + 1) % 3])))
            count[(u, v)] += 1
    assert sim.num_dihedrals() == sum(1 for c in count.values() if c == 2)


def test_bending_at_rest_exerts_no_force():
    sc = scenes.config_small(side=5)
    n = sc["pos"].shape[0]
    sim = O.OracleCloth(True)
    sim.set_material(sc["density"], 0.0, (0.0, 0.0, 0.0))
    sim.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    sim.set_mesh(sc["tris"])
    sim.build_bending(1e-2)
    sim.set_solver(100, 1e-12, "zero")
    sim.step(sc["dt"])
    assert np.abs(sim.dump_system()[4]).max() < 1e-12


def test_lumped_mass_sums_to_density_times_area():
    sc = scenes.config_small()
    sim = O.OracleCloth(True)
    n = sc["pos"].shape[0]
    sim.set_state(sc["pos"], sc["vel"])
    sim.set_mesh(sc["tris"])
    inv = sim.redistribute_mass(0.1)
    assert (1.0 / inv).sum() == pytest.approx(0.1 * 1.0, rel=1e-5)  # 1 m^2 cloth


def test_edges_match_scene_generator():
    sc = scenes.config_small()
    sim = O.OracleCloth(True)
    sim.set_state(sc["pos"], sc["vel"])
    sim.set_mesh(sc["tris"])
    np.testing.assert_array_equal(sim.edges(), sc["edges"])


def test_free_fall_without_elastics_is_exact():
    # no elastic elements, no pins: x_{n+1} = x_n + dt v + dt^2 g exactly
    sc = scenes.config_small(side=4)
    n = sc["pos"].shape[0]
    sim = O.OracleCloth(True)
    sim.set_material(0.1, 0.0, (0, -9.81, 0))
    sim.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    sim.set_mesh(sc["tris"])
    sim.set_solver(50, 1e-12, "zero")
    dt = 0.01
    sim.step(dt)
    p, v = sim.state()
    # g and dt cross the API as float32
    g32, dt32 = float(np.float32(-9.81)), float(np.float32(dt))
    np.testing.assert_allclose(p[:, 1], sc["pos"][:, 1].astype(np.float64) + g32 * dt32 * dt32, rtol=0, atol=1e-13)
    np.testing.assert_allclose(v[:, 1], g32 * dt32, atol=1e-10)


def test_fixed_iteration_mode_runs_exact_count():
    sc = scenes.config_small(side=6)
    sim = _oracle_sim(sc, tol=0.0, max_iter=7, warm="previous")
    sim.step(sc["dt"])
    assert sim.stats()[0] == 7


def test_converged_oracle_is_tolerance_stable():
    # FP64 at rel-res 1e-6 vs 1e-10: trajectories agree to < 1e-5 m
    sc = scenes.config_small(steps=60)
    p6, _, it6 = O.run_scene(sc, fp64=True, rel_tol=1e-6, max_iter=5000)
    p10, _, _ = O.run_scene(sc, fp64=True, rel_tol=1e-10, max_iter=5000)
    assert np.abs(p6 - p10).max() < 1e-5
    assert it6.max() < 5000


def test_errors_map_to_exception_types():
    sim = O.OracleCloth(True)
    with pytest.raises(ValueError):
        sim.set_solver(max_iter=-1)
    sc = scenes.config_small(side=3)
    sim.set_state(sc["pos"], sc["vel"])
    sim.set_mesh(sc["tris"])
    with pytest.raises(ValueError):
        sim.step(0.0)
    sim.set_pins([99], [[0, 0, 0]])
    with pytest.raises(ValueError):  # out_of_range is reported as index error (rc 1)
        sim.step(0.01)


def test_thread_pool_resizes_between_runs():
    # resizing the pool after it has run jobs must not replay a finished job
    sc = scenes.config_small(side=6)
    for threads in (4, 2, 3, 1, 4):
        O.set_threads(threads)
        s = _oracle_sim(sc, tol=1e-10)
        s.step(sc["dt"])
        assert s.stats()[2] == 0
    O.set_threads(1)
