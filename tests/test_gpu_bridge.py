"""The Newton bridge (chysx.newton_bridge.SolverChysX) and the double-buffered
step behind it (chysx_cloth_step_into), with torch tensors and Warp-like
arrays (objects exposing .ptr) standing in for Newton's state arrays."""
from types import SimpleNamespace

import numpy as np
import pytest

from chysx import capi, scenes
from chysx.newton_bridge import SolverChysX
from chysx.runner import GpuCloth

pytestmark = pytest.mark.gpu


class WarpLike:
    """A device array seen the way Warp exposes it: a .ptr address."""

    def __init__(self, t):
        self.t = t

    @property
    def ptr(self):
        return self.t.data_ptr()

    def numpy(self):
        return self.t.cpu().numpy()


def newton_objects(sc, wrap=lambda t: t):
    import torch

    n = sc["pos"].shape[0]
    q0 = torch.from_numpy(sc["pos"].copy()).cuda()
    model = SimpleNamespace(particle_count=n, particle_q=wrap(q0), particle_qd=wrap(torch.zeros_like(q0)),
                            particle_inv_mass=wrap(torch.ones(n, dtype=torch.float32, device="cuda")),
                            tri_indices=sc["tris"], gravity=np.asarray(sc["gravity"], np.float32))
    states = [SimpleNamespace(particle_q=wrap(q0.clone()), particle_qd=wrap(torch.zeros_like(q0)))
              for _ in range(2)]
    return model, states


def tensor(a):
    return a.t if isinstance(a, WarpLike) else a


@pytest.mark.parametrize("wrap", [lambda t: t, WarpLike], ids=["torch", "warp_like"])
def test_double_buffered_bridge_matches_in_place_stepping(wrap):
    sc = scenes.config_small(steps=30)
    ref = GpuCloth(sc, max_iter=100, rel_tol=0.0, warm_start="previous")
    model, (s0, s1) = newton_objects(sc, wrap)
    solver = SolverChysX(model, density=sc["density"], spring_stiffness=sc["k_spring"],
                         stretch_stiffness=sc["k_stretch"], pins=(sc["pin_idx"], sc["pin_targets"]),
                         redistribute_mass=True, pcg_iterations=100)
    np.testing.assert_array_equal(tensor(model.particle_inv_mass).cpu().numpy(), ref.inv_mass.cpu().numpy())
    for _ in range(30):
        before = tensor(s0.particle_q).clone()
        ref.step()
        solver.step(s0, s1, None, None, sc["dt"])
        assert tensor(s0.particle_q).equal(before)  # state_in is not written
        np.testing.assert_array_equal(tensor(s1.particle_q).cpu().numpy(), ref.positions().astype(np.float32))
        np.testing.assert_array_equal(tensor(s1.particle_qd).cpu().numpy(), ref.velocities().astype(np.float32))
        s0, s1 = s1, s0


def test_step_into_in_place_and_argument_checks():
    import torch

    sc = scenes.config_small(steps=5)
    a = GpuCloth(sc, max_iter=100, rel_tol=0.0)
    b = GpuCloth(sc, max_iter=100, rel_tol=0.0)
    for _ in range(5):
        a.step()
        b.sim.step_into(sc["dt"], b.pos.data_ptr(), b.vel.data_ptr(), b.pos.data_ptr(), b.vel.data_ptr())
    np.testing.assert_array_equal(a.positions(), b.positions())
    out = torch.empty_like(b.pos)
    with pytest.raises(ValueError):  # overlapping output
        b.sim.step_into(sc["dt"], b.pos.data_ptr(), b.vel.data_ptr(), b.pos.data_ptr() + 12, out.data_ptr())
    with pytest.raises(ValueError):  # only one of the two in place
        b.sim.step_into(sc["dt"], b.pos.data_ptr(), b.vel.data_ptr(), b.pos.data_ptr(), out.data_ptr())


def test_failed_solve_copies_the_input_state():
    import torch

    sc = scenes.config_small(steps=5)
    g = GpuCloth(sc, max_iter=100, rel_tol=0.0)
    g.step()
    g.pos[17, 1] = float("nan")
    pos_out = torch.full_like(g.pos, 3.0)
    vel_out = torch.full_like(g.vel, 3.0)
    g.sim.step_into(sc["dt"], g.pos.data_ptr(), g.vel.data_ptr(), pos_out.data_ptr(), vel_out.data_ptr())
    assert g.stats()[2] == capi.SOLVE_NONFINITE
    assert torch.equal(torch.nan_to_num(pos_out, 7.0), torch.nan_to_num(g.pos, 7.0))
    assert torch.equal(vel_out, g.vel)
