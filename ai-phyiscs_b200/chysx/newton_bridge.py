"""Newton bridge: ``SolverChysX``, the solver object a Newton simulation loop
steps (``solver.step(state_in, state_out, control, contacts, dt)``).

The reference's bridge lives in the Newton repository
(``newton/_src/solvers/chysx/solver_chysx.py``); its README describes it
(README.md:113-130): at construction it copies a ``ClothMaterial`` built from
the Newton model into a ``ClothSimulator``; every step copies ``state_in`` to
``state_out``, points the simulator at ``state_out``'s particle arrays and
steps them in place, so callers keep double-buffering.  This class keeps that
contract with one change of mechanism: the step reads ``state_in`` and writes
``state_out`` in the same kernels (``chysx_cloth_step_into``), so there is no
copy pass and ``state_in`` is left as it was.

Model and state are duck-typed, so the bridge runs with Newton's objects and
with stand-ins: a particle array may be a Warp array (``.ptr``), a torch CUDA
tensor (``data_ptr()``) or a raw device address.  The model provides
``particle_count``, ``particle_q`` (rest / initial positions, device),
``particle_inv_mass`` (device, may be None), ``tri_indices`` ((T, 3) ints,
host- or device-side) and ``gravity`` (3 floats); a state provides
``particle_q`` and ``particle_qd``.
"""
from __future__ import annotations

import numpy as np


def device_address(a) -> int:
    """Raw CUDA address of a Warp array, torch tensor or integer address."""
    if a is None:
        return 0
    if isinstance(a, (int, np.integer)):
        return int(a)
    if hasattr(a, "ptr"):
        return int(a.ptr)
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    raise TypeError(f"cannot take a device address of {type(a).__name__}")


def host_array(a, dtype):
    """A host NumPy copy of a Warp array, torch tensor or array-like."""
    if hasattr(a, "numpy"):
        try:
            return np.ascontiguousarray(a.numpy(), dtype)
        except TypeError:  # a torch CUDA tensor needs .cpu() first
            return np.ascontiguousarray(a.cpu().numpy(), dtype)
    if hasattr(a, "cpu"):
        return np.ascontiguousarray(a.cpu().numpy(), dtype)
    return np.ascontiguousarray(a, dtype)


class SolverChysX:
    """Implicit cloth step of a Newton model's particles and triangles.

    Keyword options select the constraint sets built from the model's
    initial positions (each None = not built) and the solver settings; the
    defaults are the reference simulator's (50 fixed PCG iterations, warm
    start from the previous dx).  Particles whose inverse mass is 0 are held
    by the reference's 1e8 mass rule; ``pins=(indices, targets)`` adds
    penalty pins.
    """

    def __init__(self, model, *, density=0.1, damping=0.0, spring_stiffness=None, stretch_stiffness=None,
                 shear_stiffness=None, bending_stiffness=None, pins=None, pin_stiffness=1.0e6,
                 redistribute_mass=False, pcg_iterations=50, rel_tol=0.0, warm_start="previous",
                 static_planes=(), static_boxes=(), static_contact=None, cuda_stream=0):
        import chysx

        self.model = model
        self.n = int(model.particle_count)
        self.stream = int(cuda_stream)
        g = [float(v) for v in host_array(model.gravity, np.float64).reshape(3)]
        mat = chysx.ClothMaterial()
        mat.density = float(density)
        mat.damping = float(damping)
        mat.gx, mat.gy, mat.gz = g
        sim = chysx.ClothSimulator()
        sim.set_material(mat)
        inv_mass = getattr(model, "particle_inv_mass", None)
        # the model's arrays are the "current positions" the rest shapes are
        # built from; stepping then points the simulator at the states
        sim.set_external_buffers(device_address(model.particle_q), device_address(getattr(model, "particle_qd", 0))
                                 or device_address(model.particle_q), self.n, device_address(inv_mass))
        sim.set_mesh(host_array(model.tri_indices, np.int32).reshape(-1, 3))
        if redistribute_mass:
            if inv_mass is None:
                raise ValueError("redistribute_mass needs model.particle_inv_mass to write into")
            sim.redistribute_mass_area_weighted(mat.density, device_address(inv_mass), self.n, self.stream)
        if spring_stiffness is not None:
            sim.build_springs_from_current_positions(_stiffness(spring_stiffness), self.stream)
        if stretch_stiffness is not None:
            sim.build_fem_stretch_from_current_positions(_stiffness(stretch_stiffness), self.stream)
        if shear_stiffness is not None:
            sim.build_fem_shear_from_current_positions(_stiffness(shear_stiffness), self.stream)
        if bending_stiffness is not None:
            sim.build_bending_from_current_positions(float(bending_stiffness), self.stream)
        if pins is not None:
            idx, tgt = pins
            sim.set_pins(np.asarray(idx, np.int32), np.asarray(tgt, np.float32).reshape(-1, 3), float(pin_stiffness))
        for n_, d_ in static_planes:
            sim.add_static_plane(np.asarray(n_, np.float32), float(d_))
        for box in static_boxes:
            sim.add_static_box(*[np.asarray(v, np.float32) for v in box])
        if static_contact is not None:
            t_, k_, mu_, eps_ = static_contact
            sim.set_static_contact_thickness(t_)
            sim.set_static_contact_stiffness(k_)
            sim.set_static_contact_friction(mu_)
            sim.set_static_contact_friction_epsilon(eps_)
        sim.set_solver(int(pcg_iterations), float(rel_tol), warm_start)
        self.sim = sim

    def step(self, state_in, state_out, control=None, contacts=None, dt=1.0 / 60.0):
        """Advance state_in by dt into state_out (the same object steps in place)."""
        self.sim.step_into(float(dt), device_address(state_in.particle_q), device_address(state_in.particle_qd),
                           device_address(state_out.particle_q), device_address(state_out.particle_qd),
                           self.stream)

    def last_stats(self):
        return self.sim.last_stats()


def _stiffness(k):
    return np.asarray(k, np.float32) if np.ndim(k) else float(k)
