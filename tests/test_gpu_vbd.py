"""The cloth VBD solver on the GPU (include/chysx_vbd.h) against the CPU
restatement with the same colouring, and through the reference-named
pybind11 class."""
import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes, vbd_scenes

pytestmark = pytest.mark.gpu

KEYS = ("pos", "vel", "inv_mass", "tri_indices", "tri_poses", "tri_areas", "tri_materials", "edge_indices",
        "edge_rest_angle", "edge_rest_length", "edge_bending_props")


class GpuVbd:
    def __init__(self, vb, colors=None, api="capi"):
        import torch

        self.vb = vb
        self.n = vb["pos"].shape[0]
        self.dev = {k: torch.from_numpy(np.ascontiguousarray(vb[k])).cuda() for k in KEYS}
        if api == "capi":
            self.s = capi.Vbd()
        else:
            import chysx

            self.s = chysx.ClothVBDSolver()
        if colors is None:
            self.s.build_cloth_coloring(vb["tri_indices"], vb["edge_indices"], self.n)
        else:
            self.s.set_coloring(np.asarray(colors, np.int32))
        self.s.build_tri_adjacency(vb["tri_indices"], self.n)
        self.s.build_edge_adjacency(vb["edge_indices"], self.n)
        self.api = api

    def colors(self):
        return self.s.colors(self.n)

    def step(self, iterations, dt=None):
        d = self.dev
        dt = float(self.vb["dt"] if dt is None else dt)
        args = [d["pos"].data_ptr(), d["vel"].data_ptr(), d["inv_mass"].data_ptr(), self.n,
                d["tri_indices"].data_ptr(), d["tri_poses"].data_ptr(), d["tri_areas"].data_ptr(),
                d["tri_materials"].data_ptr(), self.vb["tri_indices"].shape[0], d["edge_indices"].data_ptr(),
                d["edge_rest_angle"].data_ptr(), d["edge_rest_length"].data_ptr(), d["edge_bending_props"].data_ptr(),
                self.vb["edge_indices"].shape[0]]
        g = [float(v) for v in self.vb["gravity"]]
        if self.api == "capi":
            self.s.step_cloth(*args, g, dt, iterations)
        else:
            self.s.step_cloth(*args, *g, dt, iterations)

    def state(self):
        import torch

        torch.cuda.synchronize()
        return self.dev["pos"].cpu().numpy().astype(np.float64), self.dev["vel"].cpu().numpy().astype(np.float64)


def problem(side=10):
    return vbd_scenes.from_scene(scenes.config_small(side=side), pinned=[side * (side - 1), side * side - 1])


@pytest.mark.parametrize("side", [10, 24])
def test_vbd_matches_oracle(side):
    vb = problem(side)
    g = GpuVbd(vb)
    vb["colors"] = g.colors()
    p, v = vb["pos"].astype(float), vb["vel"].astype(float)
    q, w = p.copy(), v.copy()
    for k in range(20):
        g.step(10)
        p, v = O.vbd_step(vb, p, v, 10, vb["dt"])               # FP64
        q, w = O.vbd_step(vb, q, w, 10, vb["dt"], fp64=False)   # FP32 port
        gp, gv = g.state()
        if k == 0:
            assert np.abs(gp - q).max() < 1e-6
        assert np.abs(gp - p).max() <= max(3 * np.abs(q - p).max(), 1e-6)
    assert np.abs(gp - p).max() < 5e-4
    assert np.abs(gv - v).max() < 5e-2


def test_vbd_pybind_facade_and_determinism():
    vb = problem(16)
    a = GpuVbd(vb)
    b = GpuVbd(vb, api="pybind")
    assert b.s.num_colors() == a.s.num_colors()
    np.testing.assert_array_equal(a.colors(), b.colors())
    for _ in range(5):
        a.step(8)
        b.step(8)
    np.testing.assert_array_equal(a.state()[0], b.state()[0])


def test_vbd_iteration_and_argument_changes_and_errors():
    vb = problem(10)
    g = GpuVbd(vb)
    vb["colors"] = g.colors()
    p, v = vb["pos"].astype(float), vb["vel"].astype(float)
    for it in (3, 0, 7):  # the step graph is rebuilt when the iteration count changes
        g.step(it)
        p, v = O.vbd_step(vb, p, v, it, vb["dt"], fp64=False)
        assert np.abs(g.state()[0] - p).max() < 1e-5
    with pytest.raises(ValueError):
        g.step(5, dt=0.0)
    h = capi.Vbd()
    h.set_coloring(np.zeros(g.n - 1, np.int32))  # a colouring of another particle count
    h.build_tri_adjacency(vb["tri_indices"], g.n)
    with pytest.raises(ValueError):
        d = g.dev
        h.step_cloth(d["pos"].data_ptr(), d["vel"].data_ptr(), d["inv_mass"].data_ptr(), g.n, 0, 0, 0, 0, 0, 0, 0,
                     0, 0, 0, vb["gravity"], vb["dt"], 3)
