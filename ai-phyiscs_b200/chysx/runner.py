"""Drive a seeded scene (chysx.scenes format) through the simulator on a GPU.

The caller-owned float3 buffers are torch CUDA tensors standing in for the
Warp arrays Newton passes to the reference (``data_ptr()`` is the same kind of
raw device address as ``wp.array.ptr``).  Two front ends reach the same C ABI:
``api="capi"`` (ctypes, include/chysx_cloth.h) and ``api="pybind"`` (the
``chysx.ClothSimulator`` facade).
"""
from __future__ import annotations

import numpy as np


class GpuCloth:
    def __init__(self, scene, *, max_iter=None, rel_tol=None, warm_start="zero", springs_in_step=True,
                 apply_force=False, api="capi", device="cuda", instances=None):
        import torch

        self.torch = torch
        self.scene = scene
        n = scene["pos"].shape[0]
        self.n = n
        self.pos = torch.from_numpy(np.ascontiguousarray(scene["pos"], np.float32)).to(device)
        self.vel = torch.from_numpy(np.ascontiguousarray(scene["vel"], np.float32)).to(device)
        self.inv_mass = torch.ones(n, dtype=torch.float32, device=device)
        force = scene.get("force")
        self.force = None if force is None else torch.from_numpy(np.ascontiguousarray(force, np.float32)).to(device)
        fptr = 0 if self.force is None else self.force.data_ptr()
        max_iter = scene["max_iter"] if max_iter is None else max_iter
        rel_tol = scene["rel_tol"] if rel_tol is None else rel_tol
        self.api = api
        if api == "capi":
            from . import capi

            s = capi.Cloth()
            s.set_material(density=scene["density"], damping=scene.get("damping", 0.0), gravity=scene["gravity"])
            s.set_external_buffers(self.pos.data_ptr(), self.vel.data_ptr(), n, self.inv_mass.data_ptr(), fptr)
            s.set_mesh(scene["tris"])
            if instances is not None:
                s.set_instances(instances)
            s.set_options(springs_in_step, apply_force, scene.get("det_eps", 1.0e-6))
            s.redistribute_mass(scene["density"], self.inv_mass.data_ptr(), n)
            if scene.get("k_spring") is not None:
                s.build_springs(scene["k_spring"])
            if scene.get("k_stretch") is not None:
                s.build_fem_stretch(scene["k_stretch"])
            if scene.get("k_shear") is not None:
                s.build_fem_shear(scene["k_shear"])
            if scene.get("k_bend") is not None:
                s.build_bending(scene["k_bend"])
            if len(scene["pin_idx"]):
                s.set_pins(scene["pin_idx"], scene["pin_targets"], scene.get("k_pin", 1.0e6))
            for n_, d_ in scene.get("planes", ()):
                s.add_static_plane(n_, d_)
            for box in scene.get("boxes", ()):
                s.add_static_box(*box)
            if scene.get("static_contact") is not None:
                s.set_static_contact(*scene["static_contact"])
            s.set_solver(max_iter, rel_tol, warm_start)
            self._step = s.step
            self._stats = s.last_stats
            self._dump = s.debug_dump
        else:
            import chysx

            s = chysx.ClothSimulator()
            m = chysx.ClothMaterial()
            m.density = scene["density"]
            m.damping = scene.get("damping", 0.0)
            m.gx, m.gy, m.gz = scene["gravity"]
            s.set_material(m)
            s.set_external_buffers(self.pos.data_ptr(), self.vel.data_ptr(), n, self.inv_mass.data_ptr(), fptr)
            s.set_mesh(np.ascontiguousarray(scene["tris"], np.int32))
            s.set_options(springs_in_step, apply_force, scene.get("det_eps", 1.0e-6))
            s.redistribute_mass_area_weighted(scene["density"], self.inv_mass.data_ptr(), n)
            if scene.get("k_spring") is not None:
                k = scene["k_spring"]
                s.build_springs_from_current_positions(np.asarray(k, np.float32) if np.ndim(k) else float(k))
            if scene.get("k_stretch") is not None:
                k = scene["k_stretch"]
                s.build_fem_stretch_from_current_positions(np.asarray(k, np.float32) if np.ndim(k) else float(k))
            if scene.get("k_shear") is not None:
                k = scene["k_shear"]
                s.build_fem_shear_from_current_positions(np.asarray(k, np.float32) if np.ndim(k) else float(k))
            if scene.get("k_bend") is not None:
                s.build_bending_from_current_positions(float(scene["k_bend"]))
            if len(scene["pin_idx"]):
                s.set_pins(np.asarray(scene["pin_idx"], np.int32), np.asarray(scene["pin_targets"], np.float32),
                           scene.get("k_pin", 1.0e6))
            for n_, d_ in scene.get("planes", ()):
                s.add_static_plane(np.asarray(n_, np.float32), float(d_))
            for box in scene.get("boxes", ()):
                s.add_static_box(*[np.asarray(v, np.float32) for v in box])
            if scene.get("static_contact") is not None:
                t_, k_, mu_, eps_ = scene["static_contact"]
                s.set_static_contact_thickness(t_)
                s.set_static_contact_stiffness(k_)
                s.set_static_contact_friction(mu_)
                s.set_static_contact_friction_epsilon(eps_)
            s.set_solver(max_iter, rel_tol, warm_start)
            self._step = s.step
            self._stats = s.last_stats
            self._dump = s.debug_dump_last_solve
        self.sim = s

    def step(self, dt=None, stream=0):
        self._step(self.scene["dt"] if dt is None else dt, stream)

    def stats(self):
        return self._stats()

    def dump(self):
        return self._dump()

    def positions(self):
        self.torch.cuda.synchronize()
        return self.pos.cpu().numpy().astype(np.float64)

    def velocities(self):
        self.torch.cuda.synchronize()
        return self.vel.cpu().numpy().astype(np.float64)

    def run(self, steps, record_iters=True):
        iters = []
        for _ in range(steps):
            self.step()
            if record_iters:
                iters.append(self.stats()[0])
        return np.array(iters)
