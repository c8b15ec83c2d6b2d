"""CPU checks of the oracle's contact terms: static planes / boxes
(collision/static_contact.cu) and the contact operator
(collision/contact_spmv.cu, constraint/collision/self_collision_constraint.cu).

Each check restates the reference formula in NumPy for a handful of particles
and compares it with the oracle's assembled system, or checks a property the
penalty model implies (the operator's diagonal plus off-diagonal blocks form
k (w w^T) (x) n n^T; the solve satisfies the system it states).
"""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import scenes

DT = 1.0 / 60.0


def patch(w=3, y=0.005, vel=(0.0, 0.0, 0.0)):
    pos, tris = scenes.grid_mesh(w, size=0.2, y=y)
    pos = pos.astype(np.float32)
    v = np.tile(np.asarray(vel, np.float32), (pos.shape[0], 1))
    return pos, v, tris


def make(pos, vel, tris, k_stretch=1.0e3, tol=1e-12, max_iter=5000, warm="zero"):
    s = O.OracleCloth(True)
    s.set_material(0.1, 0.0, (0.0, -9.81, 0.0))
    s.set_state(pos, vel, np.ones(pos.shape[0], np.float32))
    s.set_mesh(tris)
    im = s.redistribute_mass(0.1)
    s.set_state(pos, vel, im)
    s.build_stretch(k_stretch)
    s.set_solver(max_iter, tol, warm)
    return s


def system(s):
    s.step(DT)
    return s.dump_system()


def f1(u, eps):
    return 1.0 / u if u > eps else (-u / eps + 2.0) / eps


def test_plane_contact_adds_penalty_gradient_and_normal_block():
    pos, vel, tris = patch(y=0.004)
    k, h = 2.0e3, 0.01
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.add_static_plane((0.0, 1.0, 0.0), 0.0)
    s.set_static_contact(h, k)
    got = system(s)
    depth = float(np.float32(h)) - pos[:, 1].astype(np.float64)  # parameters cross as float32
    nrm = np.array([0.0, 1.0, 0.0])
    # rhs = inertia - grad, grad += -k depth n (static_contact.cu:186-206)
    np.testing.assert_allclose(got[4] - base[4], k * depth[:, None] * nrm, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(got[0] - base[0], k * np.einsum("i,j->ij", nrm, nrm)[None].repeat(len(pos), 0),
                               rtol=1e-12, atol=1e-9)
    np.testing.assert_array_equal(got[3], base[3])  # off-diagonal blocks untouched


def test_no_contact_above_thickness():
    pos, vel, tris = patch(y=0.05)
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.add_static_plane((0.0, 1.0, 0.0), 0.0)
    s.set_static_contact(0.01, 1.0e4, 0.5)
    got = system(s)
    for a, b in zip(got, base):
        np.testing.assert_array_equal(a, b)


def test_plane_friction_block_force_and_coulomb_cone():
    pos, vel, tris = patch(y=0.004, vel=(0.6, -0.2, 0.1))
    k, h, mu, eps = 2.0e3, 0.01, 0.4, 1.0e-4
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.add_static_plane((0.0, 1.0, 0.0), 0.0)
    s.set_static_contact(h, k, mu, eps)
    got = system(s)
    nrm = np.array([0.0, 1.0, 0.0])
    P = np.eye(3) - np.outer(nrm, nrm)
    for i in range(len(pos)):
        depth = float(np.float32(h)) - float(pos[i, 1])
        dxv = vel[i].astype(np.float64) * float(np.float32(DT))
        ut = dxv - nrm * (nrm @ dxv)
        al = float(np.float32(mu)) * k * depth * f1(np.linalg.norm(ut), float(np.float32(eps)))
        # diagonal: k n n^T + alpha (I - n n^T)
        np.testing.assert_allclose(got[0][i] - base[0][i], k * np.outer(nrm, nrm) + al * P, rtol=1e-9, atol=1e-9)
        # residual before the cone: r0 + k depth n + alpha u_t (the lagged
        # friction enters the gradient with a minus sign, static_contact.cu:208-219)
        F = base[4][i] + k * depth * nrm + al * ut
        F0 = F - k * depth * nrm
        f0n = F0 @ nrm
        fn = max(0.0, -f0n)
        if fn > 0.0:
            F0t = F0 - f0n * nrm
            ft = np.linalg.norm(F0t)
            if ft > 0.0:
                F = F - (F0t if ft <= mu * fn else (mu * fn / ft) * F0t)
        np.testing.assert_allclose(got[4][i], F, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("where,normal", [
    ((0.0, 0.095, 0.0), (0.0, 1.0, 0.0)),      # inside, nearest the +y face
    ((0.0, 0.0, -0.19), (0.0, 0.0, -1.0)),     # inside, nearest the -z face
    ((0.305, 0.105, 0.0), None),                # outside, past the +x/+y edge
])
def test_box_contact_normal_and_depth(where, normal):
    """Box SDF (static_contact.cu:56-100): inside, the nearest face; outside,
    the normalised clamped offset."""
    he = np.array([0.3, 0.1, 0.2])
    pos, vel, tris = patch(y=0.5)
    pos[0] = np.asarray(where, np.float32)
    k, h = 1.0e3, 0.01
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.add_static_box((0.0, 0.0, 0.0), he)
    s.set_static_contact(h, k)
    got = system(s)
    x = pos[0].astype(np.float64)
    d = np.abs(x) - he.astype(np.float32).astype(np.float64)
    if normal is None:
        c = np.maximum(d, 0.0)
        dist = np.linalg.norm(c)
        normal = np.sign(x) * c / dist
    else:
        dist = d.max()
    depth = float(np.float32(h)) - dist
    assert depth > 0
    np.testing.assert_allclose(got[4][0] - base[4][0], k * depth * np.asarray(normal), rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(got[0][0] - base[0][0], k * np.outer(normal, normal), rtol=1e-6, atol=1e-9)
    # the other particles lie far above the box
    np.testing.assert_array_equal(got[4][1:], base[4][1:])


def random_contacts(rng, n, m, depth=0.002, with_slip=True):
    pairs = np.stack([rng.choice(n, 4, replace=False) for _ in range(m)]).astype(np.int32)
    b = rng.dirichlet(np.ones(3), m)
    w = np.concatenate([np.ones((m, 1)), -b], 1)
    nrm = rng.normal(size=(m, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    weights = np.concatenate([w, nrm, np.full((m, 1), depth)], 1).astype(np.float32)
    slips = None
    if with_slip:
        u = rng.normal(scale=2e-4, size=(m, 3))
        slips = np.concatenate([u, np.linalg.norm(u, axis=1, keepdims=True)], 1).astype(np.float32)
    return pairs, weights, slips


def dense_contact(pairs, weights, n, k, mu=0.0, slips=None, eps=1e-4, ks=None):
    """Dense 3n x 3n penalty Hessian sum_c w w^T (x) (k n n^T + alpha (I - n n^T))."""
    mu, eps = float(np.float32(mu)), float(np.float32(eps))  # parameters cross as float32
    C = np.zeros((3 * n, 3 * n))
    g = np.zeros((n, 3))
    for c in range(len(pairs)):
        kc = float(ks[c]) if ks is not None else k
        w = weights[c, :4].astype(np.float64)
        nv = weights[c, 4:7].astype(np.float64)
        depth = float(weights[c, 7])
        al = 0.0
        u = np.zeros(3)
        if mu > 0 and slips is not None:
            al = mu * kc * depth * f1(float(slips[c, 3]), eps)
            u = slips[c, :3].astype(np.float64)
        H = kc * np.outer(nv, nv) + al * (np.eye(3) - np.outer(nv, nv))
        for a in range(4):
            g[pairs[c, a]] += w[a] * (-kc * depth * nv - al * u)
            for b in range(4):
                C[3 * pairs[c, a]:3 * pairs[c, a] + 3, 3 * pairs[c, b]:3 * pairs[c, b] + 3] += w[a] * w[b] * H
    return C, g


def dense_system(diag, rp, col, vals):
    n = diag.shape[0]
    A = np.zeros((3 * n, 3 * n))
    for i in range(n):
        A[3 * i:3 * i + 3, 3 * i:3 * i + 3] = diag[i]
        for q in range(rp[i], rp[i + 1]):
            j = col[q]
            A[3 * i:3 * i + 3, 3 * j:3 * j + 3] = vals[q]
    return A


@pytest.mark.parametrize("friction", [0.0, 0.3])
def test_contact_operator_blocks_and_gradient(friction):
    rng = np.random.default_rng(5)
    pos, vel, tris = patch(w=4, y=0.5)
    n = pos.shape[0]
    pairs, weights, slips = random_contacts(rng, n, 7)
    k = 3.0e3
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.set_contacts(pairs, weights, k, slips=slips, friction=friction)
    got = system(s)
    C, g = dense_contact(pairs, weights, n, k, friction, slips)
    # diagonal blocks baked into the system's diagonal
    for i in range(n):
        np.testing.assert_allclose(got[0][i] - base[0][i], C[3 * i:3 * i + 3, 3 * i:3 * i + 3], rtol=1e-9, atol=1e-7)
    # off-diagonal part applied as an operator
    off = C.copy()
    for i in range(n):
        off[3 * i:3 * i + 3, 3 * i:3 * i + 3] = 0.0
    Coff = np.stack([s.contact_spmv(e.reshape(-1, 3)).ravel() for e in np.eye(3 * n)], 1)
    np.testing.assert_allclose(Coff, off, rtol=1e-9, atol=1e-7)
    np.testing.assert_allclose(Coff, Coff.T, atol=1e-7)
    # gradient enters the rhs with a minus sign
    np.testing.assert_allclose(got[4] - base[4], -g, rtol=1e-9, atol=1e-7)


def test_contact_operator_per_contact_stiffness_and_skips():
    rng = np.random.default_rng(6)
    pos, vel, tris = patch(w=4, y=0.5)
    n = pos.shape[0]
    pairs, weights, _ = random_contacts(rng, n, 6, with_slip=False)
    ks = np.array([1e3, 0.0, 2e3, -5.0, np.inf, 4e3], np.float32)
    base = system(make(pos, vel, tris))
    s = make(pos, vel, tris)
    s.set_contacts(pairs, weights, 1.0e9, stiffnesses=ks)
    got = system(s)
    keep = np.array([True, False, True, False, False, True])  # finite and > 0 only
    C, g = dense_contact(pairs[keep], weights[keep], n, 0.0, ks=ks[keep])
    for i in range(n):
        np.testing.assert_allclose(got[0][i] - base[0][i], C[3 * i:3 * i + 3, 3 * i:3 * i + 3], rtol=1e-9, atol=1e-7)
    np.testing.assert_allclose(got[4] - base[4], -g, rtol=1e-9, atol=1e-7)


@pytest.mark.parametrize("mode", [0, 1])
def test_contact_solve_satisfies_its_system(mode):
    """Mode 0 solves (A + C_off) x = b from any guess; mode 1 (the
    reference's warm residual) solves (A + C_off) x = b + C_off x0."""
    rng = np.random.default_rng(7)
    pos, vel, tris = patch(w=4, y=0.5)
    n = pos.shape[0]
    pairs, weights, slips = random_contacts(rng, n, 5)
    s = make(pos, vel, tris, tol=1e-13, max_iter=20000, warm="user")
    x0 = rng.normal(scale=1e-3, size=(n, 3))
    s.set_warm_guess(x0)
    s.set_contacts(pairs, weights, 5.0e3, slips=slips, friction=0.2, residual_mode=mode)
    diag, rp, col, vals, rhs, dx = system(s)
    A = dense_system(diag, rp, col, vals)
    Cx = lambda x: s.contact_spmv(x.reshape(-1, 3)).ravel()
    lhs = A @ dx.ravel() + Cx(dx.ravel())
    want = rhs.ravel() + (Cx(x0.ravel()) if mode == 1 else 0.0)
    np.testing.assert_allclose(lhs, want, rtol=0, atol=1e-8 * np.abs(want).max())
