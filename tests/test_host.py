"""CPU tests of the C-ABI library's host logic (no GPU needed): the library
loads, exports every symbol include/chysx_cloth.h declares, and its host-side
mesh / topology / argument handling matches the oracle and the reference's
error behaviour."""
import os
import re

import numpy as np
import pytest

import oracle.oracle as O
from chysx import capi, scenes

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
HEADERS = [os.path.join(INCLUDE, f) for f in sorted(os.listdir(INCLUDE)) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(chysx_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("chysx_cloth_create", "chysx_cloth_step", "chysx_cloth_set_external_buffers",
                 "chysx_cloth_set_mesh", "chysx_cloth_set_pins", "chysx_cloth_build_springs",
                 "chysx_cloth_build_fem_stretch", "chysx_cloth_redistribute_mass",
                 "chysx_cloth_set_pcg_iterations", "chysx_cloth_debug_dump", "chysx_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the ctypes table covers the header exactly
    assert sorted(capi.SIGNATURES) == declared_functions()


def test_set_mesh_builds_reference_edge_list():
    sc = scenes.config_small()
    c = capi.Cloth()
    c.set_mesh(sc["tris"])
    np.testing.assert_array_equal(c.edges(), sc["edges"])
    assert c.edges().shape == (261, 2)


def test_edge_list_with_duplicates_and_degenerate_triangles():
    tris = np.array([[0, 1, 2], [2, 1, 0], [0, 0, 3], [3, 2, 1]], np.int32)
    c = capi.Cloth()
    c.set_mesh(tris)
    o = O.OracleCloth(True)
    o.set_state(np.zeros((4, 3), np.float32), np.zeros((4, 3), np.float32))
    o.set_mesh(tris)
    np.testing.assert_array_equal(c.edges(), o.edges())
    np.testing.assert_array_equal(c.edges(), scenes.unique_edges(tris))


def test_empty_mesh():
    c = capi.Cloth()
    c.set_mesh(np.zeros((0, 3), np.int32))
    assert c.edges().shape == (0, 2)


def _oracle_pattern(sc):
    n = sc["pos"].shape[0]
    o = O.OracleCloth(True)
    o.set_material(sc["density"], 0.0, sc["gravity"])
    o.set_state(sc["pos"], sc["vel"], np.ones(n, np.float32))
    o.set_mesh(sc["tris"])
    o.build_springs(sc["k_spring"])
    o.build_stretch(sc["k_stretch"])
    o.set_solver(1, 0.0, "zero")
    o.step(sc["dt"])
    _, rp, col, _, _, _ = o.dump_system()
    return rp, col


@pytest.mark.parametrize("side", [3, 10, 33])
def test_topology_pattern_matches_oracle(side):
    sc = scenes.config_small(side=side)
    n = sc["pos"].shape[0]
    rp, col, ell, w = capi.topology_pattern(n, sc["tris"], sc["edges"])
    orp, ocol = _oracle_pattern(sc)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert w == 6 if side > 3 else w <= 6
    assert ell >= len(col) and ell % 32 == 0


def test_topology_pattern_random_mesh():
    rng = np.random.default_rng(7)
    n = 200
    tris = rng.integers(0, n, size=(500, 3)).astype(np.int32)
    edges = scenes.unique_edges(tris)
    rp, col, ell, w = capi.topology_pattern(n, tris, edges)
    # reference construction: all (a,b) pairs a != b per triangle, sort+unique
    pairs = set()
    for t in tris:
        for a in range(3):
            for b in range(3):
                if a != b and t[a] != t[b]:
                    pairs.add((int(t[a]), int(t[b])))
    pairs = sorted(pairs)
    ref_rp = np.zeros(n + 1, np.int64)
    for r, _ in pairs:
        ref_rp[r + 1] += 1
    np.testing.assert_array_equal(rp, np.cumsum(ref_rp))
    np.testing.assert_array_equal(col, [c for _, c in pairs])
    assert w == max(np.diff(rp))


def test_topology_rejects_out_of_range_vertex():
    with pytest.raises(IndexError):
        capi.topology_pattern(3, np.array([[0, 1, 5]], np.int32))


def test_topology_rejects_too_wide_rows():
    # a fan of 300 triangles around vertex 0 -> 301 neighbours
    n = 302
    tris = np.array([[0, k, k + 1] for k in range(1, 301)], np.int32)
    with pytest.raises(RuntimeError):
        capi.topology_pattern(n, tris)


def test_argument_errors_map_like_the_reference():
    c = capi.Cloth()
    with pytest.raises(ValueError):
        c.set_mesh(np.zeros((0, 3), np.int32).reshape(0, 3)[:0]) or c.set_solver(max_iter=-1)
    with pytest.raises(ValueError):
        c.set_solver(50, -1.0, "zero")
    with pytest.raises(ValueError):
        c.set_pcg_iterations(-3)
    with pytest.raises(RuntimeError):
        c.set_solver(50, 1e-6, "learned")  # no network loaded
    c.set_pins([0, 1], [[0, 0, 0], [1, 1, 1]])
    assert c.num_pins() == 2
    with pytest.raises(ValueError):
        c.update_pin_targets(np.zeros((3, 3), np.float32))
    # step with missing buffers: RuntimeError (reference: runtime_error)
    c.set_external_buffers(0, 0, 4)
    with pytest.raises(RuntimeError):
        c.step(0.01)
    # build_springs before positions: RuntimeError
    c.set_mesh(np.array([[0, 1, 2]], np.int32))
    with pytest.raises(RuntimeError):
        c.build_springs(10.0)
    # redistribute_mass argument checks: invalid_argument before any device work
    with pytest.raises(ValueError):
        c.redistribute_mass(0.1, 0, 4)
    with pytest.raises(ValueError):
        c.redistribute_mass(-1.0, 1234, 4)
    # zero particles: step is a no-op
    c.set_external_buffers(0, 0, 0)
    c.step(0.01)


def test_no_alloc_gradients_reject_sizes_before_any_device_work():
    # the limit comes from the library; sizes are checked before any CUDA call
    L = capi.lib()
    limit = int(L.chysx_mlp_noalloc_max_rows())
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "chysx_cloth.h")).read()
    assert limit == int(re.search(r"#define CHYSX_MLP_NOALLOC_MAX_ROWS (\d+)", header).group(1))
    for rows in (limit + 1, 1 << 20, 0, -5):
        assert L.chysx_mlp_gradients_noalloc(16, 16, 16, rows, 16, None, 0) == capi.ERR_INVALID_ARGUMENT
    assert L.chysx_mlp_gradients_noalloc(16, 16, 16, limit + 1, 16, None, 0) == capi.ERR_INVALID_ARGUMENT
    msg = L.chysx_last_error().decode()
    assert "CHYSX_MLP_NOALLOC_MAX_ROWS" in msg and str(limit) in msg
    # the static scratch is the workspace layout at the limit (activations,
    # loss partials and the per-chunk weight-gradient partials)
    assert L.chysx_mlp_workspace_bytes(limit) == 5308672


def test_material_round_trip():
    c = capi.Cloth()
    c.set_material(density=0.3, damping=0.5, gravity=(1.0, 2.0, 3.0))
    m = capi.Material()
    capi.check(capi.lib().chysx_cloth_get_material(c.h, m))
    assert (m.density, m.damping, m.gx, m.gy, m.gz) == pytest.approx((0.3, 0.5, 1.0, 2.0, 3.0))
    assert m.lame_mu == 0.0


def test_pybind_facade_mirrors_reference_api():
    import chysx

    mat = chysx.ClothMaterial()
    # reference defaults (src/cloth/cloth_material.h:20-43)
    assert (mat.density, mat.damping, mat.gx, mat.gy, mat.gz) == pytest.approx((0.05, 0.0, 0.0, 0.0, -9.81))
    for field in ("lame_mu", "lame_lambda", "bending"):
        assert getattr(mat, field) == 0.0
    sim = chysx.ClothSimulator()
    for name in ("set_material", "set_external_buffers", "step", "set_pins", "clear_pins", "num_pins",
                 "update_pin_targets", "set_mesh", "build_springs_from_current_positions", "num_springs",
                 "redistribute_mass_area_weighted", "build_fem_stretch_from_current_positions",
                 "set_pcg_iterations", "pcg_iterations", "debug_dump_last_solve"):
        assert callable(getattr(sim, name)), name
    assert sim.pcg_iterations() == 50  # reference default (cloth_simulator.h:713)
    sim.set_pcg_iterations(100)
    assert sim.pcg_iterations() == 100
    with pytest.raises(ValueError):
        sim.set_mesh(np.zeros((4, 2), np.int32))
    with pytest.raises(ValueError):
        sim.set_pins(np.array([0, 1], np.int32), np.zeros((3, 3), np.float32))
    sim.set_mesh(np.array([[0, 1, 2], [0, 2, 3]], np.int32))
    assert sim.edges().shape == (5, 2)
    sim.set_external_buffers(0, 0, 4)
    with pytest.raises(RuntimeError):
        sim.step(1.0 / 60.0)
    sim.set_external_buffers(1, 1, 4)
    with pytest.raises(ValueError):
        sim.step(0.0)


def test_bridge_device_addresses_and_host_arrays():
    """The Newton bridge's duck typing needs no GPU: Warp arrays (.ptr),
    tensors (data_ptr()), raw addresses; host copies of array-likes."""
    from chysx.newton_bridge import device_address, host_array

    class W:
        ptr = 0x7000

    class T:
        def data_ptr(self):
            return 0x9000

    assert device_address(W()) == 0x7000
    assert device_address(T()) == 0x9000
    assert device_address(0x1234) == 0x1234
    assert device_address(None) == 0
    with pytest.raises(TypeError):
        device_address("x")
    a = host_array([[0, 1, 2], [2, 1, 3]], np.int32)
    assert a.dtype == np.int32 and a.shape == (2, 3)
