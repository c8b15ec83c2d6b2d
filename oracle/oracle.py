"""Test infrastructure only: ctypes wrapper of the CPU cloth oracle.

`OracleCloth(fp64=True)` is the FP64 restatement of ChysX's
``ClothSimulator::step`` (src/cloth/cloth_simulator.cu:814-1261);
`OracleCloth(fp64=False)` is the single-threaded FP32 CPU baseline of the
same assembly + PCG.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU legs may use this module, and only as the checker / baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libchysx_oracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle shared library in place (g++ -fopenmp)."""
    srcs = [os.path.join(_HERE, f) for f in ("cloth_oracle.cpp", "vbd_oracle.cpp")]
    if force or not os.path.exists(_LIB_PATH) or any(os.path.getmtime(_LIB_PATH) < os.path.getmtime(f) for f in srcs):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libchysx_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_threads.argtypes = [ctypes.c_int]
        vp = ctypes.c_void_p
        L.orc_set_material.argtypes = [vp] + [ctypes.c_float] * 5
        L.orc_set_state.argtypes = [vp, ctypes.c_int, _f32p, _f32p, _f32p, _f32p]
        L.orc_get_state.argtypes = [vp, _f64p, _f64p]
        L.orc_set_mesh.argtypes = [vp, _i32p, ctypes.c_int]
        L.orc_num_edges.argtypes = [vp]
        L.orc_get_edges.argtypes = [vp, _i32p]
        L.orc_build_springs.argtypes = [vp, ctypes.c_float, _f32p]
        L.orc_build_stretch.argtypes = [vp, ctypes.c_float, _f32p, ctypes.c_float]
        L.orc_build_shear.argtypes = [vp, ctypes.c_float, _f32p]
        L.orc_build_bending.argtypes = [vp, ctypes.c_float]
        L.orc_num_dihedrals.argtypes = [vp]
        L.orc_bending_eval.argtypes = [_f64p, ctypes.c_double, ctypes.c_double, _f64p, _f64p, _f64p]
        L.orc_bending_angle.argtypes = [_f64p]
        L.orc_bending_angle.restype = ctypes.c_double
        L.orc_redistribute_mass.argtypes = [vp, ctypes.c_float, _f32p]
        L.orc_set_pins.argtypes = [vp, _i32p, _f32p, ctypes.c_int, ctypes.c_float]
        L.orc_set_options.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_set_solver.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_set_warm_guess.argtypes = [vp, _f64p]
        L.orc_step.argtypes = [vp, ctypes.c_float]
        L.orc_last_stats.argtypes = [vp, _i32p, _f64p, _i32p]
        L.orc_nnz.argtypes = [vp]
        L.orc_num_particles.argtypes = [vp]
        L.orc_dump_system.argtypes = [vp, _f64p, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.orc_spmv.argtypes = [vp, _f64p, _f64p]
        L.orc_contact_spmv.argtypes = [vp, _f64p, _f64p]
        L.orc_vbd_step.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p, _i32p, _f64p, _f64p, _f64p, ctypes.c_int,
                                   _i32p, _f64p, _f64p, _f64p, ctypes.c_int, _i32p, _f64p, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int]
        L.orc_vbd_membrane.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p] + [ctypes.c_double] * 5 + [_f64p, _f64p]
        L.orc_vbd_membrane_energy.argtypes = [_f64p, _f64p] + [ctypes.c_double] * 3
        L.orc_vbd_membrane_energy.restype = ctypes.c_double
        L.orc_vbd_bending.argtypes = [ctypes.c_int, _f64p, _f64p] + [ctypes.c_double] * 5 + [_f64p, _f64p]
        L.orc_vbd_hinge_angle.argtypes = [_f64p]
        L.orc_vbd_hinge_angle.restype = ctypes.c_double
        L.orc_set_preconditioner.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_set_coarse_bounds.argtypes = [vp, ctypes.c_void_p, ctypes.c_int]
        L.orc_add_static_plane.argtypes = [vp, _f32p, ctypes.c_float]
        L.orc_coarse_system.argtypes = [vp, ctypes.c_void_p]
        L.orc_add_static_box.argtypes = [vp, _f32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_clear_static_shapes.argtypes = [vp]
        L.orc_set_static_contact.argtypes = [vp] + [ctypes.c_float] * 4
        L.orc_set_contacts.argtypes = [vp, _i32p, _f32p, ctypes.c_int, ctypes.c_float, _f32p, _f32p,
                                       ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.orc_rest_shape.argtypes = [_f64p, ctypes.c_double, ctypes.c_double, _f64p, _f64p]
        L.orc_triangle_eval.argtypes = [_f64p, _f64p, ctypes.c_double, ctypes.c_double, _f64p, _f64p, _f64p]
        L.orc_spring_eval.argtypes = [_f64p, ctypes.c_double, ctypes.c_double, _f64p, _f64p, _f64p]
        _lib = L
    return _lib


def _p(a, t):
    if a is None:
        return ctypes.cast(None, t)
    return a.ctypes.data_as(t)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class OracleError(RuntimeError):
    pass


def _check(rc: int) -> None:
    if rc != 0:
        msg = lib().orc_last_error().decode()
        if rc == 1:
            raise ValueError(msg)
        raise OracleError(msg)


class OracleCloth:
    """Host restatement of ClothSimulator with the same call sequence."""

    def __init__(self, fp64: bool = True):
        self._L = lib()
        self._h = self._L.orc_create(1 if fp64 else 0)
        self.n = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.orc_destroy(h)
            self._h = None

    def set_material(self, density, damping, g):
        _check(self._L.orc_set_material(self._h, density, damping, *[float(v) for v in g]))

    def set_state(self, pos, vel, inv_mass=None, force=None):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        self.n = pos.shape[0]
        im = None if inv_mass is None else np.ascontiguousarray(inv_mass, np.float32)
        fo = None if force is None else np.ascontiguousarray(force, np.float32)
        _check(self._L.orc_set_state(self._h, self.n, _p(pos, _f32p), _p(vel, _f32p), _p(im, _f32p), _p(fo, _f32p)))

    def state(self):
        p = np.zeros((self.n, 3), np.float64)
        v = np.zeros((self.n, 3), np.float64)
        _check(self._L.orc_get_state(self._h, _p(p, _f64p), _p(v, _f64p)))
        return p, v

    def set_mesh(self, tris):
        tris = np.ascontiguousarray(tris, np.int32)
        _check(self._L.orc_set_mesh(self._h, _p(tris, _i32p), tris.shape[0]))

    def edges(self):
        e = np.zeros((self._L.orc_num_edges(self._h), 2), np.int32)
        _check(self._L.orc_get_edges(self._h, _p(e, _i32p)))
        return e

    def build_springs(self, k):
        ke = None
        if np.ndim(k) > 0:
            ke = np.ascontiguousarray(k, np.float32)
            k = 0.0
        _check(self._L.orc_build_springs(self._h, float(k), _p(ke, _f32p)))

    def build_bending(self, k):
        _check(self._L.orc_build_bending(self._h, float(k)))

    def num_dihedrals(self):
        return int(self._L.orc_num_dihedrals(self._h))

    def build_shear(self, k):
        kt = np.ascontiguousarray(k, np.float32) if np.ndim(k) else None
        _check(self._L.orc_build_shear(self._h, 0.0 if np.ndim(k) else float(k), _p(kt, _f32p)))

    def build_stretch(self, k, theta=0.0):
        kt = None
        if np.ndim(k) > 0:
            kt = np.ascontiguousarray(k, np.float32)
            k = 0.0
        _check(self._L.orc_build_stretch(self._h, float(k), _p(kt, _f32p), float(theta)))

    def redistribute_mass(self, density):
        out = np.zeros(self.n, np.float32)
        _check(self._L.orc_redistribute_mass(self._h, float(density), _p(out, _f32p)))
        return out

    def set_pins(self, idx, targets, k=1.0e6):
        idx = np.ascontiguousarray(idx, np.int32)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 3)
        _check(self._L.orc_set_pins(self._h, _p(idx, _i32p), _p(t, _f32p), idx.shape[0], float(k)))

    def set_options(self, springs_in_step=True, apply_force=False, det_eps=1.0e-6):
        _check(self._L.orc_set_options(self._h, int(springs_in_step), int(apply_force), float(det_eps)))

    def set_solver(self, max_iter=50, rel_tol=0.0, warm_start="previous"):
        wm = {"zero": 0, "previous": 1, "user": 2, "previous_scaled": 3, "user_scaled": 4}[warm_start]
        _check(self._L.orc_set_solver(self._h, int(max_iter), float(rel_tol), wm))

    def set_warm_guess(self, dx0):
        d = np.ascontiguousarray(dx0, np.float64)
        _check(self._L.orc_set_warm_guess(self._h, _p(d, _f64p)))

    def step(self, dt):
        _check(self._L.orc_step(self._h, float(dt)))

    def stats(self):
        it = ctypes.c_int()
        rr = ctypes.c_double()
        st = ctypes.c_int()
        _check(self._L.orc_last_stats(self._h, ctypes.byref(it), ctypes.byref(rr), ctypes.byref(st)))
        return it.value, rr.value, st.value

    def dump_system(self):
        n = self.n
        nnz = self._L.orc_nnz(self._h)
        diag = np.zeros((n, 3, 3))
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        vals = np.zeros((nnz, 3, 3))
        rhs = np.zeros((n, 3))
        dx = np.zeros((n, 3))
        _check(self._L.orc_dump_system(self._h, _p(diag, _f64p), _p(rp, _i32p), _p(col, _i32p),
                                       _p(vals, _f64p), _p(rhs, _f64p), _p(dx, _f64p)))
        return diag, rp, col, vals, rhs, dx

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        y = np.zeros_like(x)
        _check(self._L.orc_spmv(self._h, _p(x, _f64p), _p(y, _f64p)))
        return y

    def contact_spmv(self, x):
        """The contact operator's off-diagonal part C_off x."""
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        y = np.zeros_like(x)
        _check(self._L.orc_contact_spmv(self._h, _p(x, _f64p), _p(y, _f64p)))
        return y

    def set_preconditioner(self, degree=0, ratio=30.0, block_rows=512, coarse=False, coarse_rows=0):
        """0: block-Jacobi (the reference's); odd degree: the product's
        block-local Chebyshev preconditioner on blocks of block_rows rows;
        coarse: plus the coarse level of one translation per coarse block
        (True or "translation"), or of the translation and the linear fields
        along the block's principal axes ("linear"); coarse blocks of
        coarse_rows rows (0: block_rows)."""
        c = {False: 0, True: 1, "translation": 1, "linear": 2}[coarse]
        _check(self._L.orc_set_preconditioner(self._h, int(degree), float(ratio), int(block_rows), c,
                                              int(coarse_rows)))

    def set_coarse_bounds(self, bounds=None):
        """Explicit coarse blocks: their first rows (increasing from 0, the
        last entry n or more) instead of blocks of coarse_rows rows; None
        goes back to those."""
        if bounds is None:
            _check(self._L.orc_set_coarse_bounds(self._h, None, 0))
            return
        b = np.ascontiguousarray(bounds, np.int32)
        _check(self._L.orc_set_coarse_bounds(self._h, b.ctypes.data_as(ctypes.c_void_p), int(b.size)))

    def coarse_system(self):
        """A_c of the last solve with the coarse level (dense, float64)."""
        m = self._L.orc_coarse_system(self._h, None)
        out = np.zeros((m, m), np.float64)
        self._L.orc_coarse_system(self._h, out.ctypes.data_as(ctypes.c_void_p))
        return out

    def add_static_plane(self, n, d):
        n = np.ascontiguousarray(n, np.float32).reshape(3)
        _check(self._L.orc_add_static_plane(self._h, _p(n, _f32p), float(d)))

    def add_static_box(self, center, half_ext, ex=(1, 0, 0), ey=(0, 1, 0), ez=(0, 0, 1)):
        a = [np.ascontiguousarray(v, np.float32).reshape(3) for v in (center, half_ext, ex, ey, ez)]
        _check(self._L.orc_add_static_box(self._h, *[_p(v, _f32p) for v in a]))

    def clear_static_shapes(self):
        _check(self._L.orc_clear_static_shapes(self._h))

    def set_static_contact(self, thickness, stiffness, friction=0.0, friction_epsilon=1.0e-4):
        _check(self._L.orc_set_static_contact(self._h, float(thickness), float(stiffness), float(friction),
                                              float(friction_epsilon)))

    def set_contacts(self, pairs, weights, stiffness, stiffnesses=None, slips=None, friction=0.0,
                     friction_epsilon=1.0e-4, residual_mode=0):
        """Contact operator: pairs (M, 4) int32, weights (M, 8) float32
        (w0..w3, normal, depth), optional per-contact stiffness (M,) and
        lagged slips (M, 4); residual_mode 1 reproduces the reference's
        warm-start residual without the off-diagonal contact part."""
        pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 4)
        weights = np.ascontiguousarray(weights, np.float32).reshape(-1, 8)
        ks = None if stiffnesses is None else np.ascontiguousarray(stiffnesses, np.float32).reshape(-1)
        sl = None if slips is None else np.ascontiguousarray(slips, np.float32).reshape(-1, 4)
        self._contact_keep = (pairs, weights, ks, sl)
        _check(self._L.orc_set_contacts(self._h, _p(pairs, _i32p), _p(weights, _f32p), pairs.shape[0],
                                        float(stiffness), _p(ks, _f32p), _p(sl, _f32p), float(friction),
                                        float(friction_epsilon), int(residual_mode)))


def rest_shape(x9, det_eps=1.0e-6, theta=0.0):
    x9 = np.ascontiguousarray(x9, np.float64).reshape(9)
    dm = np.zeros(4)
    ar = np.zeros(1)
    lib().orc_rest_shape(_p(x9, _f64p), det_eps, theta, _p(dm, _f64p), _p(ar, _f64p))
    return dm, float(ar[0])


def triangle_eval(x9, dm_inv, area, k):
    x9 = np.ascontiguousarray(x9, np.float64).reshape(9)
    dm = np.ascontiguousarray(dm_inv, np.float64).reshape(4)
    e = np.zeros(1)
    g = np.zeros(9)
    h = np.zeros((9, 9))
    lib().orc_triangle_eval(_p(x9, _f64p), _p(dm, _f64p), float(area), float(k), _p(e, _f64p), _p(g, _f64p), _p(h, _f64p))
    return float(e[0]), g, h


def bending_eval(x12, k, theta0):
    """Energy, gradient (12) and Gauss-Newton Hessian (12 x 12) of one
    dihedral (v0, v1 hinge; v2, v3 wings), or None when degenerate."""
    x12 = np.ascontiguousarray(x12, np.float64).reshape(12)
    e = np.zeros(1)
    g = np.zeros(12)
    h = np.zeros((12, 12))
    ok = lib().orc_bending_eval(_p(x12, _f64p), float(k), float(theta0), _p(e, _f64p), _p(g, _f64p), _p(h, _f64p))
    return (float(e[0]), g, h) if ok else None


def bending_angle(x12):
    x12 = np.ascontiguousarray(x12, np.float64).reshape(12)
    return float(lib().orc_bending_angle(_p(x12, _f64p)))


def spring_eval(x6, L, k):
    x6 = np.ascontiguousarray(x6, np.float64).reshape(6)
    e = np.zeros(1)
    g = np.zeros(6)
    h = np.zeros((6, 6))
    lib().orc_spring_eval(_p(x6, _f64p), float(L), float(k), _p(e, _f64p), _p(g, _f64p), _p(h, _f64p))
    return float(e[0]), g, h


def add_static_shapes(sim, scene):
    """Static planes / boxes and contact parameters of a scene dict."""
    for n_, d_ in scene.get("planes", ()):
        sim.add_static_plane(n_, d_)
    for box in scene.get("boxes", ()):
        sim.add_static_box(*box)
    if scene.get("static_contact") is not None:
        sim.set_static_contact(*scene["static_contact"])


def run_scene(scene, steps=None, fp64=True, rel_tol=None, max_iter=None, warm_start="zero",
              springs_in_step=True, apply_force=False, record=False):
    """Run a scene dict (chysx.scenes format) through the oracle.

    Returns (pos, vel, iters_per_step[, trajectory]).
    """
    sim = OracleCloth(fp64=fp64)
    sim.set_material(scene["density"], scene.get("damping", 0.0), scene["gravity"])
    n = scene["pos"].shape[0]
    sim.set_state(scene["pos"], scene["vel"], np.ones(n, np.float32), scene.get("force"))
    sim.set_mesh(scene["tris"])
    sim.set_options(springs_in_step=springs_in_step, apply_force=apply_force,
                    det_eps=scene.get("det_eps", 1.0e-6))
    inv_mass = sim.redistribute_mass(scene["density"])
    sim.set_state(scene["pos"], scene["vel"], inv_mass, scene.get("force"))
    if scene.get("k_spring") is not None:
        sim.build_springs(scene["k_spring"])
    if scene.get("k_stretch") is not None:
        sim.build_stretch(scene["k_stretch"])
    if scene.get("k_shear") is not None:
        sim.build_shear(scene["k_shear"])
    if scene.get("k_bend") is not None:
        sim.build_bending(scene["k_bend"])
    if len(scene["pin_idx"]):
        sim.set_pins(scene["pin_idx"], scene["pin_targets"], scene.get("k_pin", 1.0e6))
    add_static_shapes(sim, scene)
    sim.set_solver(max_iter=max_iter if max_iter is not None else scene["max_iter"],
                   rel_tol=rel_tol if rel_tol is not None else scene["rel_tol"],
                   warm_start=warm_start)
    iters = []
    traj = []
    for _ in range(steps if steps is not None else scene["steps"]):
        sim.step(scene["dt"])
        iters.append(sim.stats()[0])
        if record:
            traj.append(sim.state()[0].copy())
    p, v = sim.state()
    if record:
        return p, v, np.array(iters), np.array(traj)
    return p, v, np.array(iters)


# ---------------------------------------------------------------------------
# Cloth VBD (restatement of the reference's ClothVBDSolver.step_cloth)
# ---------------------------------------------------------------------------

def _d(a, shape=None):
    a = np.ascontiguousarray(a, np.float64)
    return a if shape is None else a.reshape(shape)


def vbd_step(vb, pos, vel, iterations, dt, fp64=True):
    """One VBD step of the problem dict `vb` (chysx.vbd_scenes format) from
    (pos, vel); returns the new (pos, vel) as float64 arrays."""
    n = pos.shape[0]
    p = _d(pos, (n, 3)).copy()
    v = _d(vel, (n, 3)).copy()
    tris = np.ascontiguousarray(vb["tri_indices"], np.int32)
    edges = np.ascontiguousarray(vb["edge_indices"], np.int32)
    colors = np.ascontiguousarray(vb["colors"], np.int32)
    args = [_d(vb["inv_mass"]), tris, _d(vb["tri_poses"]), _d(vb["tri_areas"]), _d(vb["tri_materials"])]
    eargs = [edges, _d(vb["edge_rest_angle"]), _d(vb["edge_rest_length"]), _d(vb["edge_bending_props"])]
    g = _d(vb["gravity"])
    rc = lib().orc_vbd_step(n, _p(p, _f64p), _p(v, _f64p), _p(args[0], _f64p), _p(tris, _i32p),
                            _p(args[2], _f64p), _p(args[3], _f64p), _p(args[4], _f64p), tris.shape[0],
                            _p(edges, _i32p), _p(eargs[1], _f64p), _p(eargs[2], _f64p), _p(eargs[3], _f64p),
                            edges.shape[0], _p(colors, _i32p), _p(g, _f64p), float(dt), int(iterations),
                            1 if fp64 else 0)
    assert rc == 0
    return p, v


def vbd_membrane(which, x9, p9, dmi, area, mu, lam, damping=0.0, dt=1.0 / 60.0):
    x9, p9, dmi = _d(x9, 9), _d(p9, 9), _d(dmi, 4)
    f, h = np.zeros(3), np.zeros(9)
    lib().orc_vbd_membrane(int(which), _p(x9, _f64p), _p(p9, _f64p), _p(dmi, _f64p), float(area), float(mu),
                           float(lam), float(damping), float(dt), _p(f, _f64p), _p(h, _f64p))
    return f, h.reshape(3, 3)


def vbd_membrane_energy(x9, dmi, area, mu, lam):
    x9, dmi = _d(x9, 9), _d(dmi, 4)
    return float(lib().orc_vbd_membrane_energy(_p(x9, _f64p), _p(dmi, _f64p), float(area), float(mu), float(lam)))


def vbd_bending(which, x12, p12, rest_angle, rest_length, k, damping=0.0, dt=1.0 / 60.0):
    x12, p12 = _d(x12, 12), _d(p12, 12)
    f, h = np.zeros(3), np.zeros(9)
    lib().orc_vbd_bending(int(which), _p(x12, _f64p), _p(p12, _f64p), float(rest_angle), float(rest_length),
                          float(k), float(damping), float(dt), _p(f, _f64p), _p(h, _f64p))
    return f, h.reshape(3, 3)


def vbd_hinge_angle(x12):
    x12 = _d(x12, 12)
    return float(lib().orc_vbd_hinge_angle(_p(x12, _f64p)))
