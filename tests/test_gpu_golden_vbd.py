"""The CUDA cloth VBD solver against the reference's ClothVBDSolver
(fixture tests/golden/ref_grid10_vbd.npz), with the reference's colouring."""
import numpy as np
import pytest

from golden_util import load
from test_golden_vbd import FIXTURE, PAIRS, problem
from test_gpu_vbd import GpuVbd

pytestmark = pytest.mark.gpu


def test_cuda_vbd_step_and_trajectory_match_reference():
    import torch

    fx = load(FIXTURE)
    vb = problem(fx)
    it = int(fx["iterations"])
    g = GpuVbd(vb, colors=fx["colors"])
    for a, b in PAIRS:
        g.dev["pos"].copy_(torch.from_numpy(fx[f"s{a}_pos"]))
        g.dev["vel"].copy_(torch.from_numpy(fx[f"s{a}_vel"]))
        g.step(it)
        p, v = g.state()
        assert np.abs(p - fx[f"s{b}_pos"]).max() < 2e-6
        assert np.abs(v - fx[f"s{b}_vel"]).max() < 2e-4
    t = GpuVbd(vb, colors=fx["colors"])
    for k in range(40):
        t.step(it)
        if f"s{k}_pos" in fx:
            assert np.abs(t.state()[0] - fx[f"s{k}_pos"]).max() < 5e-5 + 2e-5 * k
