"""Pins the cloth VBD restatement and the CUDA solver to the reference's own
ClothVBDSolver (fixture tests/golden/ref_grid10_vbd.npz, made by
tests/golden/make_golden.py on a B200): with the reference's colouring, one
step from each recorded state lands where the reference's did, and the
40-step trajectory stays with it."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import scenes, vbd_scenes
from golden_util import load

FIXTURE = "ref_grid10_vbd.npz"
PAIRS = [(0, 1), (9, 10), (29, 30)]


def problem(fx):
    vb = vbd_scenes.from_scene(scenes.config_small(), pinned=[90, 99])
    vb["colors"] = fx["colors"]
    return vb


def test_reference_colouring_is_valid():
    fx = load(FIXTURE)
    vb = problem(fx)
    col = fx["colors"]
    pairs = [(t[a], t[b]) for t in vb["tri_indices"] for a in range(3) for b in range(a + 1, 3)]
    pairs += [(e[a], e[b]) for e in vb["edge_indices"] for a in range(4) for b in range(a + 1, 4)]
    assert all(col[u] != col[v] for u, v in pairs)


@pytest.mark.parametrize("fp64", [True, False])
def test_oracle_step_matches_reference(fp64):
    fx = load(FIXTURE)
    vb = problem(fx)
    it = int(fx["iterations"])
    for a, b in PAIRS:
        p, v = O.vbd_step(vb, fx[f"s{a}_pos"], fx[f"s{a}_vel"], it, vb["dt"], fp64=fp64)
        assert np.abs(p - fx[f"s{b}_pos"]).max() < 2e-6
        assert np.abs(v - fx[f"s{b}_vel"]).max() < 2e-4


def test_oracle_trajectory_stays_with_reference():
    fx = load(FIXTURE)
    vb = problem(fx)
    it = int(fx["iterations"])
    p, v = vb["pos"].astype(float), vb["vel"].astype(float)
    for k in range(40):
        p, v = O.vbd_step(vb, p, v, it, vb["dt"], fp64=False)
        if f"s{k}_pos" in fx:
            assert np.abs(p - fx[f"s{k}_pos"]).max() < 5e-5 + 2e-5 * k
