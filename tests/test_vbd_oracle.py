"""CPU checks of the cloth VBD restatement (oracle/vbd_oracle.cpp) and of
the VBD host logic of the C-ABI library (colouring, adjacency), no GPU."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes, vbd_scenes


def rot(a, axis):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K


def test_membrane_force_is_minus_energy_gradient():
    rng = np.random.default_rng(0)
    rest = np.array([[0, 0, 0], [0.1, 0, 0], [0.03, 0.08, 0]], float)
    dmi, area = vbd_scenes.rest_frames(rest, np.array([[0, 1, 2]]))
    dmi, area = dmi[0], area[0]
    x = rest @ rot(0.4, [1, 2, 3]).T + rng.normal(scale=0.01, size=(3, 3))
    mu, lam = 2.0e3, 5.0e3
    for which in range(3):
        f, h = O.vbd_membrane(which, x, x, dmi, area, mu, lam)
        g = np.zeros(3)
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[which, c] += 1e-6
            xm[which, c] -= 1e-6
            g[c] = (O.vbd_membrane_energy(xp, dmi, area, mu, lam) - O.vbd_membrane_energy(xm, dmi, area, mu, lam)) / 2e-6
        np.testing.assert_allclose(f, -g, rtol=1e-5, atol=1e-8)
        np.testing.assert_allclose(h, h.T, atol=1e-9)
        assert np.linalg.eigvalsh(h).min() > -1e-9  # projected Hessian is PSD


def test_membrane_rest_state_is_force_free_and_rotation_invariant():
    rest = np.array([[0, 0, 0], [0.1, 0, 0], [0.03, 0.08, 0]], float)
    dmi, area = vbd_scenes.rest_frames(rest, np.array([[0, 1, 2]]))
    x = rest @ rot(1.1, [0.3, -1, 2]).T + np.array([0.5, -2, 1])
    for which in range(3):
        f, _ = O.vbd_membrane(which, x, x, dmi[0], area[0], 2e3, 3e3)
        assert np.abs(f).max() < 1e-9


def test_bending_force_and_angle_gradient():
    rng = np.random.default_rng(1)
    x = np.array([[0, 0, 0.1], [0.05, 0.1, -0.08], [0, 0.0, 0], [0.1, 0.05, 0]], float) + rng.normal(scale=0.01, size=(4, 3))
    th0, L, k = 0.2, np.linalg.norm(x[3] - x[2]), 0.7
    th = O.vbd_hinge_angle(x)
    for which in range(4):
        f, h = O.vbd_bending(which, x, x, th0, L, k)
        dth = np.zeros(3)
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[which, c] += 1e-7
            xm[which, c] -= 1e-7
            dth[c] = (O.vbd_hinge_angle(xp) - O.vbd_hinge_angle(xm)) / 2e-7
        np.testing.assert_allclose(f, -k * L * (th - th0) * dth, rtol=1e-5, atol=1e-9)
        np.testing.assert_allclose(h, k * L * np.outer(dth, dth), rtol=1e-5, atol=1e-9)


def test_free_fall_is_exact_and_pinned_particles_stay():
    sc = scenes.config_small(side=6)
    vb = vbd_scenes.from_scene(sc, mu=0.0, lam=0.0, bend_k=0.0, pinned=[0])
    vb["colors"] = np.zeros(36, np.int32)  # no coupling left: one colour
    p, v = O.vbd_step(vb, vb["pos"], vb["vel"], iterations=5, dt=vb["dt"])
    g, dt = vb["gravity"].astype(float), float(np.float64(vb["dt"]))
    expect = vb["pos"].astype(float) + g * dt * dt
    expect[0] = vb["pos"][0]
    np.testing.assert_allclose(p, expect, atol=1e-12)
    np.testing.assert_allclose(v[1:], np.tile(g * dt, (35, 1)), atol=1e-9)
    np.testing.assert_array_equal(v[0], 0.0)


def test_vbd_settles_a_hanging_patch_and_fp32_port_tracks_fp64():
    sc = scenes.config_small(side=8)
    vb = vbd_scenes.from_scene(sc, pinned=[56, 63])
    c = capi.Vbd()
    c.build_cloth_coloring(vb["tri_indices"], vb["edge_indices"], 64)
    vb["colors"] = c.colors(64)
    p, v = vb["pos"].astype(float), vb["vel"].astype(float)
    q, w = p.copy(), v.copy()
    for _ in range(30):
        p, v = O.vbd_step(vb, p, v, iterations=10, dt=vb["dt"])
        q, w = O.vbd_step(vb, q, w, iterations=10, dt=vb["dt"], fp64=False)
    assert np.isfinite(p).all() and p[:, 1].min() < 0.95  # it hangs down from the two corners
    np.testing.assert_allclose(p[[56, 63]], vb["pos"][[56, 63]], atol=0)
    assert np.abs(p - q).max() < 2e-4


def test_coloring_has_no_conflicts_and_adjacency_checks():
    sc = scenes.config_small(side=12)
    vb = vbd_scenes.from_scene(sc)
    n = sc["pos"].shape[0]
    c = capi.Vbd()
    c.build_cloth_coloring(vb["tri_indices"], vb["edge_indices"], n)
    col = c.colors(n)
    assert c.num_colors() == col.max() + 1 and col.min() >= 0
    pairs = [(t[a], t[b]) for t in vb["tri_indices"] for a in range(3) for b in range(a + 1, 3)]
    pairs += [(e[a], e[b]) for e in vb["edge_indices"] for a in range(4) for b in range(a + 1, 4)]
    assert all(col[u] != col[v] for u, v in pairs)
    c.build_tri_adjacency(vb["tri_indices"], n)
    c.build_edge_adjacency(vb["edge_indices"], n)
    with pytest.raises(IndexError):
        c.build_tri_adjacency(vb["tri_indices"], n - 1)
    with pytest.raises(ValueError):
        c.set_coloring(np.array([0, -1, 2], np.int32))
