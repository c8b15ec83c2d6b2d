"""ctypes binding of the C ABI (include/chysx_cloth.h).

This is the binding a ctypes-based host (or a test) uses to drive the
library without the pybind11 facade; it loads the same in-tree
``libchysx_cloth.so`` the facade links.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchysx_cloth.so")

OK, ERR_INVALID_ARGUMENT, ERR_OUT_OF_RANGE, ERR_RUNTIME, ERR_CUDA = range(5)
SOLVE_CONVERGED, SOLVE_MAX_ITER, SOLVE_NONFINITE, SOLVE_KERNEL_ERROR = range(4)
WARM = {"zero": 0, "previous": 1, "learned": 2, "previous_scaled": 3}

u = ctypes.c_uint64
i32p = ctypes.POINTER(ctypes.c_int32)
f32p = ctypes.POINTER(ctypes.c_float)
ip = ctypes.POINTER(ctypes.c_int)
dp = ctypes.POINTER(ctypes.c_double)
H = ctypes.c_void_p


class Material(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in
                ("lame_mu", "lame_lambda", "bending", "density", "damping", "gx", "gy", "gz")]


class ContactOp(ctypes.Structure):
    """chysx_contact_op: a device-resident contact list (see the header)."""
    _fields_ = [("pairs", ctypes.c_uint64), ("weights", ctypes.c_uint64), ("count", ctypes.c_uint64),
                ("max_contacts", ctypes.c_int), ("stiffness", ctypes.c_float),
                ("stiffnesses", ctypes.c_uint64), ("slips", ctypes.c_uint64),
                ("friction_mu", ctypes.c_float), ("friction_epsilon", ctypes.c_float),
                ("residual_mode", ctypes.c_int)]


# name -> (restype, argtypes); every symbol include/chysx_cloth.h declares
SIGNATURES = {
    "chysx_last_error": (ctypes.c_char_p, []),
    "chysx_cloth_create": (ctypes.c_int, [ctypes.POINTER(H)]),
    "chysx_cloth_destroy": (ctypes.c_int, [H]),
    "chysx_cloth_set_material": (ctypes.c_int, [H, ctypes.POINTER(Material)]),
    "chysx_cloth_get_material": (ctypes.c_int, [H, ctypes.POINTER(Material)]),
    "chysx_cloth_set_external_buffers": (ctypes.c_int, [H, u, u, ctypes.c_int, u, u]),
    "chysx_cloth_set_mesh": (ctypes.c_int, [H, i32p, ctypes.c_int]),
    "chysx_cloth_num_edges": (ctypes.c_int, [H, ip]),
    "chysx_cloth_get_edges": (ctypes.c_int, [H, i32p]),
    "chysx_cloth_set_pins": (ctypes.c_int, [H, i32p, f32p, ctypes.c_int, ctypes.c_float]),
    "chysx_cloth_clear_pins": (ctypes.c_int, [H]),
    "chysx_cloth_num_pins": (ctypes.c_int, [H, ip]),
    "chysx_cloth_update_pin_targets": (ctypes.c_int, [H, f32p, ctypes.c_int, u]),
    "chysx_cloth_build_springs": (ctypes.c_int, [H, ctypes.c_float, f32p, u]),
    "chysx_cloth_num_springs": (ctypes.c_int, [H, ip]),
    "chysx_cloth_build_fem_stretch": (ctypes.c_int, [H, ctypes.c_float, f32p, u]),
    "chysx_cloth_build_fem_shear": (ctypes.c_int, [H, ctypes.c_float, f32p, u]),
    "chysx_cloth_build_bending": (ctypes.c_int, [H, ctypes.c_float, u]),
    "chysx_cloth_num_dihedrals": (ctypes.c_int, [H, ip]),
    "chysx_cloth_add_static_plane": (ctypes.c_int, [H, f32p, ctypes.c_float]),
    "chysx_cloth_add_static_box": (ctypes.c_int, [H, f32p, f32p, f32p, f32p, f32p]),
    "chysx_cloth_clear_static_shapes": (ctypes.c_int, [H]),
    "chysx_cloth_static_shape_counts": (ctypes.c_int, [H, ip, ip]),
    "chysx_cloth_set_static_contact_thickness": (ctypes.c_int, [H, ctypes.c_float]),
    "chysx_cloth_set_static_contact_stiffness": (ctypes.c_int, [H, ctypes.c_float]),
    "chysx_cloth_set_static_contact_friction": (ctypes.c_int, [H, ctypes.c_float]),
    "chysx_cloth_set_static_contact_friction_epsilon": (ctypes.c_int, [H, ctypes.c_float]),
    "chysx_cloth_get_static_contact": (ctypes.c_int, [H, f32p, f32p, f32p, f32p]),
    "chysx_cloth_set_contact_op": (ctypes.c_int, [H, ctypes.POINTER(ContactOp)]),
    "chysx_cloth_clear_contact_op": (ctypes.c_int, [H]),
    "chysx_cloth_contact_stats": (ctypes.c_int, [H, ip, ip, ip]),
    "chysx_cloth_redistribute_mass": (ctypes.c_int, [H, ctypes.c_float, u, ctypes.c_int, u]),
    "chysx_cloth_set_pcg_iterations": (ctypes.c_int, [H, ctypes.c_int]),
    "chysx_cloth_pcg_iterations": (ctypes.c_int, [H, ip]),
    "chysx_cloth_set_solver": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "chysx_cloth_set_options": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int, ctypes.c_float]),
    "chysx_cloth_step": (ctypes.c_int, [H, ctypes.c_float, u]),
    "chysx_cloth_step_into": (ctypes.c_int, [H, ctypes.c_float, u, u, u, u, u]),
    "chysx_cloth_last_stats": (ctypes.c_int, [H, ip, dp, ip]),
    "chysx_cloth_set_true_residual": (ctypes.c_int, [H, ctypes.c_int]),
    "chysx_cloth_true_residual": (ctypes.c_int, [H, ctypes.c_int, dp, dp]),
    "chysx_cloth_num_particles": (ctypes.c_int, [H, ip]),
    "chysx_cloth_num_off_diag_blocks": (ctypes.c_int, [H, ip]),
    "chysx_cloth_debug_dump": (ctypes.c_int, [H, f32p, i32p, i32p, f32p, f32p, f32p]),
    "chysx_cloth_debug_coarse": (ctypes.c_int, [H, i32p, f32p, f32p, ctypes.c_int]),
    "chysx_cloth_debug_coarse_rows": (ctypes.c_int, [H, i32p, ctypes.c_int, i32p]),
    "chysx_cloth_set_network": (ctypes.c_int, [H, f32p, ctypes.c_int]),
    "chysx_cloth_set_feature_output": (ctypes.c_int, [H, u, u]),
    "chysx_cloth_guess_kept": (ctypes.c_int, [H, ip]),
    "chysx_mlp_num_params": (ctypes.c_int, []),
    "chysx_mlp_num_features": (ctypes.c_int, []),
    "chysx_mlp_workspace_bytes": (ctypes.c_uint64, [ctypes.c_int]),
    "chysx_mlp_gradients": (ctypes.c_int, [u, u, u, ctypes.c_int, u, dp, u, ctypes.c_uint64, u]),
    "chysx_mlp_predict": (ctypes.c_int, [u, u, ctypes.c_int, u, u, ctypes.c_uint64, u]),
    "chysx_mlp_train_step": (ctypes.c_int, [u, u, u, u, u, u, ctypes.c_int, ctypes.c_float, ctypes.c_int, u,
                                            ctypes.c_uint64, dp, u]),
    "chysx_mlp_gradients_noalloc": (ctypes.c_int, [u, u, u, ctypes.c_int, u, dp, u]),
    "chysx_mlp_noalloc_max_rows": (ctypes.c_int, []),
    "chysx_cloth_set_instances": (ctypes.c_int, [H, i32p, ctypes.c_int]),
    "chysx_cloth_num_instances": (ctypes.c_int, [H, ip]),
    "chysx_cloth_instance_stats": (ctypes.c_int, [H, ctypes.c_int, ip, dp, ip]),
    "chysx_cloth_set_sync_mode": (ctypes.c_int, [H, ctypes.c_int]),
    "chysx_cloth_autotune": (ctypes.c_int, [H, ctypes.c_float, ctypes.c_int, u]),
    "chysx_cloth_autotune_results": (ctypes.c_int, [H, ctypes.c_int, ctypes.POINTER(ctypes.c_int), i32p,
                                                    ctypes.POINTER(ctypes.c_float)]),
    "chysx_cloth_sync_mode": (ctypes.c_int, [H, ctypes.POINTER(ctypes.c_int)]),
    "chysx_cloth_set_tuning": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "chysx_cloth_solver_info": (ctypes.c_int, [H, ip, ip, ip]),
    "chysx_cloth_set_preconditioner": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int, ctypes.c_float]),
    "chysx_cloth_set_row_order": (ctypes.c_int, [H, ctypes.c_int]),
    "chysx_cloth_row_of_particles": (ctypes.c_int, [H, ctypes.c_int, i32p]),
    "chysx_cloth_preconditioner": (ctypes.c_int, [H, ip, ip, f32p, ip]),
    "chysx_cloth_enable_timing": (ctypes.c_int, [H, ctypes.c_int]),
    "chysx_cloth_last_timing": (ctypes.c_int, [H, f32p, f32p, f32p]),
    "chysx_vbd_create": (ctypes.c_int, [ctypes.POINTER(H)]),
    "chysx_vbd_destroy": (ctypes.c_int, [H]),
    "chysx_vbd_build_cloth_coloring": (ctypes.c_int, [H, i32p, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int]),
    "chysx_vbd_set_coloring": (ctypes.c_int, [H, i32p, ctypes.c_int]),
    "chysx_vbd_build_tri_adjacency": (ctypes.c_int, [H, i32p, ctypes.c_int, ctypes.c_int]),
    "chysx_vbd_build_edge_adjacency": (ctypes.c_int, [H, i32p, ctypes.c_int, ctypes.c_int]),
    "chysx_vbd_num_colors": (ctypes.c_int, [H, ip]),
    "chysx_vbd_colors": (ctypes.c_int, [H, i32p, ctypes.c_int]),
    "chysx_vbd_step_cloth": (ctypes.c_int, [H, u, u, u, ctypes.c_int, u, u, u, u, ctypes.c_int, u, u, u, u,
                                            ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_float, ctypes.c_int, u]),
    "chysx_topology_pattern": (ctypes.c_int, [ctypes.c_int, i32p, ctypes.c_int, i32p, ctypes.c_int,
                                              i32p, i32p, ctypes.c_int, ip, ip, ip]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with ai-phyiscs_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class ChysxError(RuntimeError):
    pass


def check(rc: int) -> None:
    if rc == OK:
        return
    msg = lib().chysx_last_error().decode()
    if rc == ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if rc == ERR_OUT_OF_RANGE:
        raise IndexError(msg)
    raise ChysxError(msg)


def _p(a, t):
    return ctypes.cast(None, t) if a is None else a.ctypes.data_as(t)


class Cloth:
    """Thin object wrapper over the C ABI handle."""

    def __init__(self):
        self._L = lib()
        h = H()
        check(self._L.chysx_cloth_create(ctypes.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self._L.chysx_cloth_destroy(self.h)
            self.h = None

    def set_material(self, density=0.05, damping=0.0, gravity=(0.0, 0.0, -9.81)):
        m = Material(0.0, 0.0, 0.0, density, damping, *gravity)
        check(self._L.chysx_cloth_set_material(self.h, ctypes.byref(m)))

    def set_external_buffers(self, pos, vel, n, inv_mass=0, force=0):
        check(self._L.chysx_cloth_set_external_buffers(self.h, pos, vel, n, inv_mass, force))

    def set_mesh(self, tris):
        t = np.ascontiguousarray(tris, np.int32)
        check(self._L.chysx_cloth_set_mesh(self.h, _p(t, i32p), t.shape[0]))

    def edges(self):
        n = ctypes.c_int()
        check(self._L.chysx_cloth_num_edges(self.h, ctypes.byref(n)))
        out = np.zeros((n.value, 2), np.int32)
        check(self._L.chysx_cloth_get_edges(self.h, _p(out, i32p)))
        return out

    def set_pins(self, idx, targets, k=1.0e6):
        i = np.ascontiguousarray(idx, np.int32)
        t = np.ascontiguousarray(targets, np.float32)
        check(self._L.chysx_cloth_set_pins(self.h, _p(i, i32p), _p(t, f32p), i.shape[0], k))

    def num_pins(self):
        n = ctypes.c_int()
        check(self._L.chysx_cloth_num_pins(self.h, ctypes.byref(n)))
        return n.value

    def update_pin_targets(self, targets, stream=0):
        t = np.ascontiguousarray(targets, np.float32)
        check(self._L.chysx_cloth_update_pin_targets(self.h, _p(t, f32p), t.shape[0], stream))

    def build_springs(self, k, stream=0):
        if np.ndim(k):
            ke = np.ascontiguousarray(k, np.float32)
            check(self._L.chysx_cloth_build_springs(self.h, 0.0, _p(ke, f32p), stream))
        else:
            check(self._L.chysx_cloth_build_springs(self.h, float(k), _p(None, f32p), stream))

    def build_fem_stretch(self, k, stream=0):
        if np.ndim(k):
            kt = np.ascontiguousarray(k, np.float32)
            check(self._L.chysx_cloth_build_fem_stretch(self.h, 0.0, _p(kt, f32p), stream))
        else:
            check(self._L.chysx_cloth_build_fem_stretch(self.h, float(k), _p(None, f32p), stream))

    def build_fem_shear(self, k, stream=0):
        if np.ndim(k):
            kt = np.ascontiguousarray(k, np.float32)
            check(self._L.chysx_cloth_build_fem_shear(self.h, 0.0, _p(kt, f32p), stream))
        else:
            check(self._L.chysx_cloth_build_fem_shear(self.h, float(k), _p(None, f32p), stream))

    def build_bending(self, k, stream=0):
        check(self._L.chysx_cloth_build_bending(self.h, float(k), stream))

    def num_dihedrals(self):
        v = ctypes.c_int()
        check(self._L.chysx_cloth_num_dihedrals(self.h, ctypes.byref(v)))
        return v.value

    def add_static_plane(self, n, d):
        n = np.ascontiguousarray(n, np.float32).reshape(3)
        check(self._L.chysx_cloth_add_static_plane(self.h, _p(n, f32p), float(d)))

    def add_static_box(self, center, half_ext, ex=(1, 0, 0), ey=(0, 1, 0), ez=(0, 0, 1)):
        a = [np.ascontiguousarray(v, np.float32).reshape(3) for v in (center, half_ext, ex, ey, ez)]
        check(self._L.chysx_cloth_add_static_box(self.h, *[_p(v, f32p) for v in a]))

    def clear_static_shapes(self):
        check(self._L.chysx_cloth_clear_static_shapes(self.h))

    def set_static_contact(self, thickness, stiffness, friction=0.0, friction_epsilon=1.0e-4):
        check(self._L.chysx_cloth_set_static_contact_thickness(self.h, float(thickness)))
        check(self._L.chysx_cloth_set_static_contact_stiffness(self.h, float(stiffness)))
        check(self._L.chysx_cloth_set_static_contact_friction(self.h, float(friction)))
        check(self._L.chysx_cloth_set_static_contact_friction_epsilon(self.h, float(friction_epsilon)))

    def static_contact(self):
        v = [ctypes.c_float() for _ in range(4)]
        check(self._L.chysx_cloth_get_static_contact(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def static_shape_counts(self):
        p, b = ctypes.c_int(), ctypes.c_int()
        check(self._L.chysx_cloth_static_shape_counts(self.h, ctypes.byref(p), ctypes.byref(b)))
        return p.value, b.value

    def set_contact_op(self, pairs, weights, count, max_contacts, stiffness, stiffnesses=0, slips=0,
                       friction_mu=0.0, friction_epsilon=1.0e-4, residual_mode=0):
        """Device addresses of int32 pairs (M, 4), float32 weights (M, 8),
        the int32 count and the optional per-contact stiffness / slips."""
        op = ContactOp(pairs, weights, count, max_contacts, stiffness, stiffnesses, slips, friction_mu,
                       friction_epsilon, residual_mode)
        check(self._L.chysx_cloth_set_contact_op(self.h, ctypes.byref(op)))

    def clear_contact_op(self):
        check(self._L.chysx_cloth_clear_contact_op(self.h))

    def contact_stats(self):
        v = [ctypes.c_int() for _ in range(3)]
        check(self._L.chysx_cloth_contact_stats(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def redistribute_mass(self, density, inv_mass_ptr, n, stream=0):
        check(self._L.chysx_cloth_redistribute_mass(self.h, density, inv_mass_ptr, n, stream))

    def set_solver(self, max_iter=50, rel_tol=0.0, warm_start="previous"):
        check(self._L.chysx_cloth_set_solver(self.h, max_iter, rel_tol, WARM[warm_start]))

    def set_pcg_iterations(self, m):
        check(self._L.chysx_cloth_set_pcg_iterations(self.h, m))

    def set_options(self, springs_in_step=True, apply_external_force=False, fem_det_eps=1.0e-6):
        check(self._L.chysx_cloth_set_options(self.h, int(springs_in_step), int(apply_external_force),
                                              fem_det_eps))

    def set_network(self, params):
        p = np.ascontiguousarray(params, np.float32)
        check(self._L.chysx_cloth_set_network(self.h, _p(p, f32p), p.shape[0]))

    def set_feature_output(self, features_ptr, predictions_ptr=0):
        check(self._L.chysx_cloth_set_feature_output(self.h, features_ptr, predictions_ptr))

    def guess_kept(self):
        v = ctypes.c_int()
        check(self._L.chysx_cloth_guess_kept(self.h, ctypes.byref(v)))
        return v.value

    def set_instances(self, offsets):
        o = None if offsets is None else np.ascontiguousarray(offsets, np.int32)
        n = 0 if o is None else o.shape[0] - 1
        check(self._L.chysx_cloth_set_instances(self.h, _p(o, i32p), n))

    def num_instances(self):
        v = ctypes.c_int()
        check(self._L.chysx_cloth_num_instances(self.h, ctypes.byref(v)))
        return v.value

    def instance_stats(self):
        n = self.num_instances()
        it = np.zeros(n, np.int32)
        rr = np.zeros(n, np.float64)
        st = np.zeros(n, np.int32)
        check(self._L.chysx_cloth_instance_stats(self.h, n, it.ctypes.data_as(ip), rr.ctypes.data_as(dp),
                                                  st.ctypes.data_as(ip)))
        return it, rr, st

    def set_tuning(self, solver_path=0, block=0, grid=0):
        check(self._L.chysx_cloth_set_tuning(self.h, solver_path, block, grid))

    def set_row_order(self, mode):
        """0: the caller's particle order; 1 or "spatial": compact blocks."""
        check(self._L.chysx_cloth_set_row_order(self.h, 1 if mode in (1, "spatial") else 0))

    def row_of_particles(self, n):
        rows = np.zeros(n, np.int32)
        check(self._L.chysx_cloth_row_of_particles(self.h, n, rows.ctypes.data_as(i32p)))
        return rows

    def set_preconditioner(self, kind="block_jacobi", degree=0, ratio=30.0):
        """"block_jacobi" (reference), "chebyshev" (CTA-local, odd degree) or
        "chebyshev_coarse" (CTA-local plus a coarse level of one translation
        per CTA block)."""
        k = {"block_jacobi": 0, "chebyshev": 1, "chebyshev_coarse": 2}[kind]
        check(self._L.chysx_cloth_set_preconditioner(self.h, k, int(degree), float(ratio)))

    def preconditioner(self):
        k, d, u = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        r = ctypes.c_float()
        check(self._L.chysx_cloth_preconditioner(self.h, ctypes.byref(k), ctypes.byref(d), ctypes.byref(r),
                                                 ctypes.byref(u)))
        # in_use: 0 block-Jacobi, 1 local, 2 two-level (translations), 3 two-level (translations + linear fields)
        return ("block_jacobi", "chebyshev", "chebyshev_coarse")[k.value], d.value, r.value, u.value

    def solver_info(self):
        """(kernel, grid, block) of the last graph build; kernel is
        'resident', 'loop' or 'streamed'."""
        p, g, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._L.chysx_cloth_solver_info(self.h, ctypes.byref(p), ctypes.byref(g), ctypes.byref(b)))
        return ("resident", "loop", "streamed")[p.value], g.value, b.value

    def autotune(self, dt, repetitions=2, stream=0):
        """Times the applicable solver configurations on the current state
        (which is restored) and keeps the fastest; returns the table as a
        list of dicts."""
        check(self._L.chysx_cloth_autotune(self.h, float(dt), int(repetitions), stream))
        cnt = ctypes.c_int()
        check(self._L.chysx_cloth_autotune_results(self.h, 0, ctypes.byref(cnt), None, None))
        cfg = np.zeros((max(cnt.value, 1), 8), np.int32)
        ms = np.zeros(max(cnt.value, 1), np.float32)
        check(self._L.chysx_cloth_autotune_results(self.h, cnt.value, ctypes.byref(cnt),
                                                   cfg.ctypes.data_as(i32p), ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        keys = ("path", "block", "sync", "kernel", "grid", "threads", "iters", "status")
        kernels = ("resident", "loop", "streamed")
        out = []
        for k in range(cnt.value):
            d = dict(zip(keys, (int(x) for x in cfg[k])))
            d["kernel"] = kernels[d["kernel"]]
            d["solve_ms"] = float(ms[k])
            out.append(d)
        return out

    def set_sync_mode(self, mode):
        check(self._L.chysx_cloth_set_sync_mode(self.h, int(mode)))

    def sync_mode(self):
        m = ctypes.c_int()
        check(self._L.chysx_cloth_sync_mode(self.h, ctypes.byref(m)))
        return m.value

    def num_off_diag_blocks(self):
        v = ctypes.c_int()
        check(self._L.chysx_cloth_num_off_diag_blocks(self.h, ctypes.byref(v)))
        return v.value

    def enable_timing(self, on=True):
        check(self._L.chysx_cloth_enable_timing(self.h, int(on)))

    def last_timing(self):
        a, b, f = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(self._L.chysx_cloth_last_timing(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(f)))
        return a.value, b.value, f.value

    def step_into(self, dt, pos_in, vel_in, pos_out, vel_out, stream=0):
        check(self._L.chysx_cloth_step_into(self.h, dt, pos_in, vel_in, pos_out, vel_out, stream))

    def step(self, dt, stream=0):
        check(self._L.chysx_cloth_step(self.h, dt, stream))

    def last_stats(self):
        it, st = ctypes.c_int(), ctypes.c_int()
        rr = ctypes.c_double()
        check(self._L.chysx_cloth_last_stats(self.h, ctypes.byref(it), ctypes.byref(rr), ctypes.byref(st)))
        return it.value, rr.value, st.value

    def set_true_residual(self, on=True):
        check(self._L.chysx_cloth_set_true_residual(self.h, int(bool(on))))

    def true_residual(self):
        """(per-instance ||b - A dx|| / ||b|| of the last step, the largest)."""
        n = self.num_instances()
        rel = np.zeros(n, np.float64)
        worst = ctypes.c_double()
        check(self._L.chysx_cloth_true_residual(self.h, n, rel.ctypes.data_as(dp), ctypes.byref(worst)))
        return rel, worst.value

    def debug_dump(self):
        n, nnz = ctypes.c_int(), ctypes.c_int()
        check(self._L.chysx_cloth_num_particles(self.h, ctypes.byref(n)))
        check(self._L.chysx_cloth_num_off_diag_blocks(self.h, ctypes.byref(nnz)))
        n, nnz = n.value, nnz.value
        diag = np.zeros((n, 3, 3), np.float32)
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(max(nnz, 1), np.int32)
        vals = np.zeros((max(nnz, 1), 3, 3), np.float32)
        rhs = np.zeros((n, 3), np.float32)
        dx = np.zeros((n, 3), np.float32)
        check(self._L.chysx_cloth_debug_dump(self.h, _p(diag, f32p), _p(rp, i32p), _p(col, i32p),
                                             _p(vals, f32p), _p(rhs, f32p), _p(dx, f32p)))
        return diag, rp, col[:nnz], vals[:nnz], rhs, dx

    def debug_coarse(self):
        """(info dict, A_c dense, rows of A_c^-1) of the last step's coarse
        level, or (info, None, None) when it is off."""
        info = np.zeros(6, np.int32)
        check(self._L.chysx_cloth_debug_coarse(self.h, _p(info, i32p), None, None, 0))
        keys = ("on", "blocks", "ctas_per_block", "fields", "m", "unused")
        d = dict(zip(keys, (int(v) for v in info)))
        if not d["on"]:
            return d, None, None
        m = d["m"]
        ac = np.zeros((m, m), np.float32)
        ainv = np.zeros((m, m), np.float32)
        check(self._L.chysx_cloth_debug_coarse(self.h, _p(info, i32p), _p(ac, f32p), _p(ainv, f32p), m * m))
        return d, ac, ainv

    def debug_coarse_rows(self):
        """First internal row of every coarse block of the last graph build
        (blocks + 1 entries; empty without a coarse level)."""
        n = np.zeros(1, np.int32)
        check(self._L.chysx_cloth_debug_coarse_rows(self.h, None, 0, _p(n, i32p)))
        rows = np.zeros(max(1, int(n[0])), np.int32)
        if n[0]:
            check(self._L.chysx_cloth_debug_coarse_rows(self.h, _p(rows, i32p), int(n[0]), _p(n, i32p)))
        return rows[:int(n[0])]


class Vbd:
    """The cloth VBD solver through the C ABI (include/chysx_vbd.h)."""

    def __init__(self):
        self._L = lib()
        h = H()
        check(self._L.chysx_vbd_create(ctypes.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self._L.chysx_vbd_destroy(h)

    def build_cloth_coloring(self, tris, edges, n):
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        e = np.ascontiguousarray(edges, np.int32).reshape(-1, 4)
        check(self._L.chysx_vbd_build_cloth_coloring(self.h, _p(t, i32p), t.shape[0], _p(e, i32p), e.shape[0], n))

    def set_coloring(self, colors):
        c = np.ascontiguousarray(colors, np.int32)
        check(self._L.chysx_vbd_set_coloring(self.h, _p(c, i32p), c.shape[0]))

    def build_tri_adjacency(self, tris, n):
        t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        check(self._L.chysx_vbd_build_tri_adjacency(self.h, _p(t, i32p), t.shape[0], n))

    def build_edge_adjacency(self, edges, n):
        e = np.ascontiguousarray(edges, np.int32).reshape(-1, 4)
        check(self._L.chysx_vbd_build_edge_adjacency(self.h, _p(e, i32p), e.shape[0], n))

    def num_colors(self):
        v = ctypes.c_int()
        check(self._L.chysx_vbd_num_colors(self.h, ctypes.byref(v)))
        return v.value

    def colors(self, n):
        out = np.zeros(n, np.int32)
        check(self._L.chysx_vbd_colors(self.h, _p(out, i32p), n))
        return out

    def step_cloth(self, pos, vel, inv_mass, n, tris, poses, areas, mats, n_tris, edges, rest_angle, rest_length,
                   props, n_edges, gravity, dt, iterations, stream=0):
        """Device addresses of the step's arrays (see the header)."""
        check(self._L.chysx_vbd_step_cloth(self.h, pos, vel, inv_mass, n, tris, poses, areas, mats, n_tris, edges,
                                           rest_angle, rest_length, props, n_edges, *[float(g) for g in gravity],
                                           float(dt), int(iterations), stream))


def topology_pattern(n, tris, edges=None):
    """Host-only: (row_offsets, col_indices, ell_entries, max_width) of the
    off-diagonal block pattern for a mesh (+ spring edges)."""
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    e = np.zeros((0, 2), np.int32) if edges is None else np.ascontiguousarray(edges, np.int32).reshape(-1, 2)
    rp = np.zeros(n + 1, np.int32)
    cap = 6 * t.shape[0] + 2 * e.shape[0] + 1
    col = np.zeros(cap, np.int32)
    nnz, ell, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().chysx_topology_pattern(n, _p(t, i32p), t.shape[0], _p(e, i32p), e.shape[0], _p(rp, i32p),
                                       _p(col, i32p), cap, ctypes.byref(nnz), ctypes.byref(ell), ctypes.byref(w)))
    return rp, col[:nnz.value], ell.value, w.value
