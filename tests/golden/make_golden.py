"""Generate the reference golden fixtures in tests/golden/ (run on a B200).

The reference has no CPU implementation and no golden vectors for this path,
so the fixtures are produced by running the reference's own ClothSimulator,
compiled from its sources by ``oracle/build_ref.sh`` into ``oracle/_ref/``:

    bash oracle/build_ref.sh                       # here (needs the sources)
    python tests/golden/make_golden.py             # on a GPU box

Each fixture records, for one seeded scene, the reference's assembled system
(``debug_dump_last_solve``: diag, row_offsets, col_indices, values, rhs, dx),
the particle state it was assembled from, and final trajectories.  Two builds
are used: ``_chysx_ref`` (unmodified: springs are built but skipped by
step(), src/cloth/cloth_simulator.cu:921) and ``_chysx_ref_springs`` (the
three spring call sites enabled).  The fixtures are small (<= 16x16 grids).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
sys.path.insert(0, os.path.join(ROOT, "ai-phyiscs_b200"))

import torch  # noqa: E402

from chysx import scenes  # noqa: E402


def run_reference(mod, sc, pcg_iters, steps, dump_at=()):
    """Run `steps` reference steps; for each step in dump_at record the state
    before the step and the system dumped after it."""
    n = sc["pos"].shape[0]
    pos = torch.from_numpy(sc["pos"].copy()).cuda()
    vel = torch.from_numpy(sc["vel"].copy()).cuda()
    inv = torch.ones(n, dtype=torch.float32, device="cuda")
    s = mod.ClothSimulator()
    s.set_material(sc["density"], sc.get("damping", 0.0), *sc["gravity"])
    s.set_external_buffers(pos.data_ptr(), vel.data_ptr(), n, inv.data_ptr())
    s.set_mesh(sc["tris"])
    s.redistribute_mass_area_weighted(sc["density"], inv.data_ptr(), n)
    s.build_springs_from_current_positions(float(sc["k_spring"]))
    s.build_fem_stretch_from_current_positions(float(sc["k_stretch"]))
    if sc.get("k_shear") is not None:
        s.build_fem_shear_from_current_positions(float(sc["k_shear"]))
    if sc.get("k_bend") is not None:
        s.build_bending_from_current_positions(float(sc["k_bend"]))
    if len(sc["pin_idx"]):
        s.set_pins(sc["pin_idx"].astype(np.int32), sc["pin_targets"].astype(np.float32), float(sc["k_pin"]))
    for n_, d_ in sc.get("planes", ()):
        s.add_static_plane(*[float(v) for v in n_], float(d_))
    for box in sc.get("boxes", ()):
        s.add_static_box(np.concatenate([np.asarray(v, np.float32) for v in box]))
    if sc.get("static_contact") is not None:
        s.set_static_contact(*[float(v) for v in sc["static_contact"]])
    if sc.get("self_collision") is not None:
        s.set_self_collision(*sc["self_collision"])
    s.set_pcg_iterations(pcg_iters)
    torch.cuda.synchronize()
    out = {"inv_mass": inv.cpu().numpy()}
    for k in range(steps):
        if k in dump_at:
            torch.cuda.synchronize()
            out[f"s{k}_pos"] = pos.cpu().numpy()
            out[f"s{k}_vel"] = vel.cpu().numpy()
        s.step(sc["dt"])
        if not bool(torch.isfinite(pos).all()):
            out["stopped_at"] = np.array(k)
            break
        if k in dump_at:
            torch.cuda.synchronize()
            diag, rp, col, vals, rhs, dx = s.debug_dump_last_solve()
            for name, a in zip(("diag", "row_offsets", "col_indices", "values", "rhs", "dx"),
                               (diag, rp, col, vals, rhs, dx)):
                out[f"s{k}_{name}"] = np.array(a)
            if sc.get("self_collision") is not None:
                cp, cw, cs = s.self_collision_contacts()
                out[f"s{k}_cpairs"] = np.array(cp)
                out[f"s{k}_cweights"] = np.array(cw)
                out[f"s{k}_cslips"] = np.array(cs)
    torch.cuda.synchronize()
    out["final_pos"] = pos.cpu().numpy()
    out["final_vel"] = vel.cpu().numpy()
    return out


def scene_grid16():
    pos, tris, _ = scenes.jittered_grid(16, seed=5)
    sc = scenes._finish("grid16_jitter", pos, tris, 500.0, 5.0e3, [240, 255], 40, 2000, 0.0)
    return sc


def scene_grid10_shear():
    """Config 1 with a Baraff-Witkin shear set (k = 5e3) beside the stretch set."""
    sc = scenes.config_small(steps=60)
    sc["k_shear"] = 5.0e3
    return sc


def scene_grid10_bending():
    """Config 1 with discrete bending (k = 5e-3) beside springs and stretch."""
    sc = scenes.config_small(steps=60)
    sc["k_bend"] = 5.0e-3
    return sc


def scene_grid10_contact():
    """Static-shape contact: config 1's patch, free, dropped onto a rotated
    table box on the ground plane, Coulomb mu = 0.3 (chysx.scenes.config_contact)."""
    return scenes.config_contact(friction=0.3, steps=30)


def scene_two_sheets():
    """Self-collision: two 10x10 sheets (0.5 m) in one mesh, the lower one
    pinned at its corners at y = 0.1, the upper one 7 mm above it, shifted by
    half a cell; thickness 10 mm, k = 1e3, mu = 0.2, so contacts exist from
    the first step."""
    h = 0.5 / 9
    pa, ta = scenes.grid_mesh(10, size=0.5, y=0.10, origin=(-0.25, -0.25))
    pb, tb = scenes.grid_mesh(10, size=0.5, y=0.107, origin=(-0.25 + 0.5 * h, -0.25 + 0.5 * h))
    pos = np.concatenate([pa, pb], 0)
    tris = np.concatenate([ta, tb + pa.shape[0]], 0)
    return scenes._finish("two_sheets", pos, tris, 1.0e3, 1.0e4, [0, 9, 90, 99], 3, 1000, 0.0,
                          self_collision=(0.01, 1.0e3, 0.2, 1.0e-4, 8192))


def make_contact(out_dir=HERE):
    import _chysx_ref_springs as mod

    a = run_reference(mod, scene_grid10_contact(), 1000, 30, dump_at=(0, 8, 14, 22, 29))
    np.savez_compressed(os.path.join(out_dir, "ref_grid10_contact.npz"), **a)
    print("grid10 contact done", flush=True)
    b = run_reference(mod, scene_two_sheets(), 1000, 3, dump_at=(0, 1, 2))
    np.savez_compressed(os.path.join(out_dir, "ref_two_sheets_selfcontact.npz"), **b)
    print("two sheets done", flush=True)


def scene_vbd():
    """Config 1's patch as a VBD problem (chysx.vbd_scenes.from_scene): the
    two far corners held (inverse mass 0), membrane mu = lambda = 2e3,
    bending k = 5e-3, damping 1e-3 on both."""
    from chysx import vbd_scenes

    return vbd_scenes.from_scene(scenes.config_small(), pinned=[90, 99])


def make_vbd(out_dir=HERE, steps=40, iterations=10, record=(0, 1, 9, 10, 29, 30, 39)):
    import _chysx_ref_springs as mod

    vb = scene_vbd()
    n = vb["pos"].shape[0]
    s = mod.ClothVBDSolver()
    s.build_cloth_coloring(vb["tri_indices"], vb["edge_indices"], n)
    s.build_tri_adjacency(vb["tri_indices"], n)
    s.build_edge_adjacency(vb["edge_indices"], n)
    dev = {k: torch.from_numpy(np.ascontiguousarray(vb[k])).cuda() for k in
           ("pos", "vel", "inv_mass", "tri_indices", "tri_poses", "tri_areas", "tri_materials", "edge_indices",
            "edge_rest_angle", "edge_rest_length", "edge_bending_props")}
    out = {"colors": np.array(s.colors()), "iterations": np.array(iterations)}
    g = [float(v) for v in vb["gravity"]]
    for k in range(steps):
        s.step_cloth(dev["pos"].data_ptr(), dev["vel"].data_ptr(), dev["inv_mass"].data_ptr(), n,
                     dev["tri_indices"].data_ptr(), dev["tri_poses"].data_ptr(), dev["tri_areas"].data_ptr(),
                     dev["tri_materials"].data_ptr(), vb["tri_indices"].shape[0], dev["edge_indices"].data_ptr(),
                     dev["edge_rest_angle"].data_ptr(), dev["edge_rest_length"].data_ptr(),
                     dev["edge_bending_props"].data_ptr(), vb["edge_indices"].shape[0], *g, float(vb["dt"]),
                     iterations)
        if k in record:
            torch.cuda.synchronize()
            out[f"s{k}_pos"] = dev["pos"].cpu().numpy()
            out[f"s{k}_vel"] = dev["vel"].cpu().numpy()
    np.savez_compressed(os.path.join(out_dir, "ref_grid10_vbd.npz"), **out)
    print("grid10 vbd done", flush=True)


def make_bending(out_dir=HERE):
    import _chysx_ref_springs as mod

    a = run_reference(mod, scene_grid10_bending(), 1000, 60, dump_at=(0, 30))
    np.savez_compressed(os.path.join(out_dir, "ref_grid10_bending.npz"), **a)
    print("grid10 bending done", flush=True)


def make_shear(out_dir=HERE):
    import _chysx_ref_springs as mod

    a = run_reference(mod, scene_grid10_shear(), 1000, 60, dump_at=(0, 30))
    np.savez_compressed(os.path.join(out_dir, "ref_grid10_shear.npz"), **a)
    print("grid10 shear done", flush=True)


def main(out_dir=HERE):
    os.makedirs(out_dir, exist_ok=True)
    import _chysx_ref  # noqa: F401
    import _chysx_ref_springs  # noqa: F401

    mods = {"nosprings": sys.modules["_chysx_ref"], "springs": sys.modules["_chysx_ref_springs"]}
    c1 = scenes.config_small()
    for tag, mod in mods.items():
        out = {}
        a = run_reference(mod, c1, 100, 200, dump_at=(0, 50, 199))
        out.update({f"it100_{k}": v for k, v in a.items()})
        b = run_reference(mod, c1, 1000, 200, dump_at=(0, 50))
        out.update({f"it1000_{k}": v for k, v in b.items()})
        np.savez_compressed(os.path.join(out_dir, f"ref_grid10_{tag}.npz"), **out)
        print(tag, "grid10 done", flush=True)
    g = scene_grid16()
    a = run_reference(mods["springs"], g, 2000, 40, dump_at=(0, 20, 39))
    np.savez_compressed(os.path.join(out_dir, "ref_grid16_springs.npz"), **a)
    print("grid16 done", flush=True)
    make_shear(out_dir)
    make_bending(out_dir)
    make_contact(out_dir)
    make_vbd(out_dir)


if __name__ == "__main__":
    # python make_golden.py [out_dir] [shear|bending|contact|vbd]   (only that fixture)
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    if len(sys.argv) > 2 and sys.argv[2] == "shear":
        make_shear(out)
    elif len(sys.argv) > 2 and sys.argv[2] == "bending":
        make_bending(out)
    elif len(sys.argv) > 2 and sys.argv[2] == "contact":
        make_contact(out)
    elif len(sys.argv) > 2 and sys.argv[2] == "vbd":
        make_vbd(out)
    else:
        main(out)
