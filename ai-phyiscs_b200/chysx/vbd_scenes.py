"""Inputs of the cloth VBD step (the reference's ClothVBDSolver.step_cloth)
built from a chysx.scenes scene: per triangle Dm^-1 of its rest shape in a
2D frame, rest area and (mu, lambda, damping); per interior edge the four
vertices (o0, o1 opposite, v2 -> v3 the hinge), the rest hinge angle and
length and (stiffness, damping); inverse masses from the lumped area mass.
Plain NumPy; the arrays feed the CUDA solver, the oracle and the reference.
"""
from __future__ import annotations

import numpy as np


def rest_frames(pos, tris):
    """Dm^-1 (row-major 2x2) and area of every triangle, in the frame of its
    first edge."""
    x0, x1, x2 = (pos[tris[:, k]].astype(np.float64) for k in range(3))
    e1, e2 = x1 - x0, x2 - x0
    l1 = np.linalg.norm(e1, axis=1)
    t = e1 / l1[:, None]
    nrm = np.cross(e1, e2)
    area = 0.5 * np.linalg.norm(nrm, axis=1)
    b = np.cross(nrm / (2.0 * area)[:, None], t)
    dm = np.stack([np.stack([l1, np.einsum("ij,ij->i", e2, t)], 1),
                   np.stack([np.zeros_like(l1), np.einsum("ij,ij->i", e2, b)], 1)], 1)  # columns: e1, e2
    inv = np.linalg.inv(dm)
    return inv.reshape(-1, 4), area


def hinge_edges(tris):
    """Interior edges as (o0, o1, v2, v3): v2 -> v3 the shared edge as the
    first triangle walks it, o0 that triangle's third vertex, o1 the other's."""
    first = {}
    out = []
    for t, (a, b, c) in enumerate(np.asarray(tris)):
        for u, v, w in ((a, b, c), (b, c, a), (c, a, b)):
            key = (min(u, v), max(u, v))
            if key in first:
                u0, v0, w0 = first.pop(key)
                out.append((w0, w, u0, v0))
            else:
                first[key] = (u, v, w)
    return np.array(sorted(out, key=lambda e: (min(e[2], e[3]), max(e[2], e[3]))), np.int32).reshape(-1, 4)


def hinge_angle(x):
    x0, x1, x2, x3 = x
    n1 = np.cross(x2 - x0, x3 - x0)
    n2 = np.cross(x3 - x1, x2 - x1)
    e = x3 - x2
    n1 /= np.linalg.norm(n1)
    n2 /= np.linalg.norm(n2)
    e /= np.linalg.norm(e)
    return float(np.arctan2(np.dot(np.cross(n1, n2), e), np.dot(n1, n2)))


def lumped_inv_mass(pos, tris, density):
    _, area = rest_frames(pos, tris)
    m = np.zeros(pos.shape[0])
    np.add.at(m, tris.ravel(), np.repeat(area * density / 3.0, 3))
    return np.where(m > 0, 1.0 / np.maximum(m, 1e-30), 0.0)


def from_scene(sc, mu=2.0e3, lam=2.0e3, damping=1.0e-3, bend_k=5.0e-3, bend_damping=1.0e-3, pinned=()):
    """The VBD problem of a cloth scene; `pinned` particles get inverse mass 0."""
    pos = np.asarray(sc["pos"], np.float64)
    tris = np.asarray(sc["tris"], np.int32)
    poses, area = rest_frames(pos, tris)
    edges = hinge_edges(tris)
    rest_angle = np.array([hinge_angle(pos[e]) for e in edges])
    rest_length = np.linalg.norm(pos[edges[:, 3]] - pos[edges[:, 2]], axis=1) if len(edges) else np.zeros(0)
    inv_mass = lumped_inv_mass(pos, tris, sc["density"])
    inv_mass[np.asarray(pinned, np.int64)] = 0.0
    T, E = tris.shape[0], edges.shape[0]
    return dict(
        pos=pos.astype(np.float32), vel=np.asarray(sc["vel"], np.float32), inv_mass=inv_mass.astype(np.float32),
        tri_indices=tris, tri_poses=poses.astype(np.float32), tri_areas=area.astype(np.float32),
        tri_materials=np.tile(np.array([mu, lam, damping], np.float32), (T, 1)),
        edge_indices=edges, edge_rest_angle=rest_angle.astype(np.float32),
        edge_rest_length=rest_length.astype(np.float32),
        edge_bending_props=np.tile(np.array([bend_k, bend_damping], np.float32), (E, 1)),
        gravity=np.asarray(sc["gravity"], np.float32), dt=sc["dt"])
