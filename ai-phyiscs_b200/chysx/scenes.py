"""Seeded synthetic cloth scenes (the workloads the cloth step is measured on).

Every generator returns a plain dict of numpy arrays so the same inputs feed
the CUDA simulator, the CPU oracle and the compiled reference module:

    pos (N,3) f32, vel (N,3) f32, tris (T,3) i32, edges (E,2) i32,
    k_spring (scalar or (E,) f32), k_stretch (scalar or (T,) f32),
    pin_idx (P,) i32, pin_targets (P,3) f32, density, gravity, dt, steps,
    max_iter, rel_tol, det_eps, name

Grid layout follows the reference scene generator
(scenes/cloth_freefall.cu:38-61): vertex (i, j) has index j*w + i and each
quad is split into (v00, v10, v11) and (v00, v11, v01).  The cloth lies in
the XZ plane at y = 1 and gravity points along -y.
"""
from __future__ import annotations

import numpy as np

DT = 1.0 / 60.0
GRAVITY = (0.0, -9.81, 0.0)


def grid_mesh(w: int, h: int | None = None, size: float = 1.0, y: float = 1.0,
              spacing: float | None = None, origin=(-0.5, -0.5)):
    """Regular (w x h) vertex grid in the XZ plane; returns (pos, tris)."""
    h = w if h is None else h
    if spacing is None:
        dx = size / (w - 1)
        dz = size / (h - 1)
    else:
        dx = dz = spacing
    i, j = np.meshgrid(np.arange(w), np.arange(h), indexing="xy")
    pos = np.zeros((h * w, 3), np.float64)
    pos[:, 0] = origin[0] + (i.ravel() * dx)
    pos[:, 1] = y
    pos[:, 2] = origin[1] + (j.ravel() * dz)
    ii, jj = np.meshgrid(np.arange(w - 1), np.arange(h - 1), indexing="xy")
    v00 = (jj * w + ii).ravel()
    v10 = v00 + 1
    v01 = v00 + w
    v11 = v01 + 1
    tris = np.empty((2 * v00.size, 3), np.int32)
    tris[0::2] = np.stack([v00, v10, v11], 1)
    tris[1::2] = np.stack([v00, v11, v01], 1)
    return pos, tris


def unique_edges(tris: np.ndarray) -> np.ndarray:
    """Sorted unique undirected edges, the order ClothSimulator.set_mesh builds
    (src/cloth/cloth_simulator.cu:328-346)."""
    t = np.asarray(tris, np.int64)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]], 0)
    e = np.sort(e, axis=1)
    key = np.unique(e[:, 0] * (np.int64(1) << 32) + e[:, 1])
    return np.stack([key >> 32, key & 0xFFFFFFFF], 1).astype(np.int32)


def _log_uniform(rng, lo, hi, n):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)


def _finish(name, pos, tris, k_spring, k_stretch, pin_idx, steps, max_iter, rel_tol,
            density=0.1, det_eps=1.0e-6, **extra):
    pos = pos.astype(np.float32)
    pin_idx = np.asarray(pin_idx, np.int32)
    d = dict(name=name, pos=pos, vel=np.zeros_like(pos), tris=np.ascontiguousarray(tris, np.int32),
             edges=unique_edges(tris), k_spring=k_spring, k_stretch=k_stretch,
             pin_idx=pin_idx, pin_targets=pos[pin_idx].copy(), k_pin=1.0e6,
             density=density, damping=0.0, gravity=GRAVITY, dt=DT, steps=steps,
             max_iter=max_iter, rel_tol=rel_tol, det_eps=det_eps)
    d.update(extra)
    return d


def config_small(side: int = 10, steps: int = 200, max_iter: int = 100, rel_tol: float = 1.0e-6):
    """Plain method, small: 10x10 patch, springs k=1e3, BW k=1e4, vertex 0 pinned."""
    pos, tris = grid_mesh(side)
    return _finish(f"grid{side}", pos, tris, 1.0e3, 1.0e4, [0], steps, max_iter, rel_tol)


def config_contact(side: int = 10, steps: int = 60, max_iter: int = 2000, rel_tol: float = 1.0e-6,
                   friction: float = 0.3, height: float = 0.16):
    """Static-shape contact: a free side x side patch (1 m, springs k=1e3, BW
    k=1e4) dropped from `height` onto a table box (half extents 0.25 x 0.05 x
    0.25 around (0, 0.05, 0), axes rotated 0.3 rad about y) standing on the
    ground plane y = 0; thickness 0.01 m, contact k=1e4, Coulomb mu."""
    pos, tris = grid_mesh(side, y=height)
    c, s = np.cos(0.3), np.sin(0.3)
    box = ((0.0, 0.05, 0.0), (0.25, 0.05, 0.25), (c, 0.0, -s), (0.0, 1.0, 0.0), (s, 0.0, c))
    return _finish(f"grid{side}_contact", pos, tris, 1.0e3, 1.0e4, [], steps, max_iter, rel_tol,
                   planes=[((0.0, 1.0, 0.0), 0.0)], boxes=[box],
                   static_contact=(0.01, 1.0e4, friction, 1.0e-4))


def jittered_grid(side: int, seed: int, size: float = 1.0):
    rng = np.random.default_rng(seed)
    pos, tris = grid_mesh(side, size=size)
    h = size / (side - 1)
    pos = pos + rng.uniform(-0.01 * h, 0.01 * h, pos.shape)
    return pos, tris, rng


def config_large(side: int = 256, seed: int = 0, steps: int = 120, max_iter: int = 2000,
                 rel_tol: float = 1.0e-6):
    """Plain method, large: 256x256, +-1% jitter, per-edge spring k log-U[1e2,1e4],
    BW k=1e4, the two top corners pinned."""
    pos, tris, rng = jittered_grid(side, seed)
    E = unique_edges(tris).shape[0]
    k_spring = _log_uniform(rng, 1.0e2, 1.0e4, E)
    top = (side - 1) * side
    return _finish(f"grid{side}_jitter", pos, tris, k_spring, 1.0e4, [top, top + side - 1],
                   steps, max_iter, rel_tol)


def config_huge(side: int = 1024, seed: int = 3, steps: int = 60, max_iter: int = 4000,
                rel_tol: float = 1.0e-6, det_eps: float = 1.0e-12):
    """1024x1024, +-1% jitter, top edge pinned, materials of the small config.

    At this resolution every rest triangle has lab*v_c ~ 9.6e-7, below the
    reference's 1e-6 degenerate-shape threshold
    (src/constraint/cloth/triangle_stretch_constraint.cu:39,88-91), which would
    replace every Dm^-1 by the identity; the workload therefore uses a
    1e-12 threshold (same formula, scale-appropriate guard)."""
    pos, tris, _ = jittered_grid(side, seed)
    top = (side - 1) * side
    return _finish(f"grid{side}_jitter", pos, tris, 1.0e3, 1.0e4, np.arange(top, top + side),
                   steps, max_iter, rel_tol, det_eps=det_eps)


def batch_instances(count: int = 512, seed: int = 1, lo: int = 16, hi: int = 128,
                    steps: int = 60, max_iter: int = 2000, rel_tol: float = 1.0e-6):
    """Batched solve: `count` square grids, side U{lo..hi}, spacing 1/side,
    per-instance BW k log-U[1e3,1e5], per-edge spring k log-U[1e2,1e4],
    1-4 random corner pins.  Returns a list of scene dicts."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, count)
    out = []
    for b, s in enumerate(sides):
        s = int(s)
        pos, tris = grid_mesh(s, spacing=1.0 / s)
        E = unique_edges(tris).shape[0]
        k_stretch = float(_log_uniform(rng, 1.0e3, 1.0e5, 1)[0])
        k_spring = _log_uniform(rng, 1.0e2, 1.0e4, E)
        corners = np.array([0, s - 1, (s - 1) * s, s * s - 1])
        npins = int(rng.integers(1, 5))
        pins = np.sort(rng.choice(corners, npins, replace=False))
        out.append(_finish(f"inst{b}_s{s}", pos, tris, k_spring, k_stretch, pins, steps,
                           max_iter, rel_tol))
    return out


def concat(scenes):
    """Pack instances into one concatenated scene (disjoint vertex ranges) and
    return (scene, row_offsets) where row_offsets[b] is the first vertex of b."""
    offs = np.zeros(len(scenes) + 1, np.int64)
    for b, s in enumerate(scenes):
        offs[b + 1] = offs[b] + s["pos"].shape[0]
    pos = np.concatenate([s["pos"] for s in scenes])
    tris = np.concatenate([s["tris"] + offs[b] for b, s in enumerate(scenes)]).astype(np.int32)
    pins = np.concatenate([s["pin_idx"] + offs[b] for b, s in enumerate(scenes)]).astype(np.int32)
    # Vertex ranges are disjoint and increasing, so the per-instance sorted
    # edge lists, concatenated, are already the sorted edge list of the pack.
    k_spring = np.concatenate([np.broadcast_to(np.asarray(s["k_spring"], np.float32),
                                               (s["edges"].shape[0],)) for s in scenes])
    k_stretch = np.concatenate([np.broadcast_to(np.asarray(s["k_stretch"], np.float32),
                                                (s["tris"].shape[0],)) for s in scenes])
    sc = _finish("batch_concat", pos.astype(np.float64), tris, k_spring, k_stretch, pins,
                 scenes[0]["steps"], scenes[0]["max_iter"], scenes[0]["rel_tol"])
    return sc, offs
