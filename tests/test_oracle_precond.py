"""CPU tests of the oracle's restatement of the product's preconditioners
(block-Jacobi, CTA-local Chebyshev, and the two-level operator with one
rigid translation per block): every variant converges to the block-Jacobi
solution, and each level removes iterations."""
import numpy as np
import pytest

from chysx import scenes
from test_gpu_precond import oracle_sim


def solve(sc, degree, coarse, block_rows=256, tol=1e-9, coarse_rows=0):
    s = oracle_sim(sc, tol, degree=degree, block_rows=block_rows)
    if coarse:
        s.set_preconditioner(degree, 30.0, block_rows, coarse=coarse, coarse_rows=coarse_rows)
    s.step(sc["dt"])
    its, _, status = s.stats()
    assert status == 0
    return its, s.dump_system()[5]


def test_two_level_converges_to_the_block_jacobi_solution_in_fewer_iterations():
    # the stiff benchmark material on 40 x 40 particles: 1600 rows, 6 blocks
    # of 256 (the last one ragged); about 950 block-Jacobi iterations
    sc = scenes.config_large(side=40, max_iter=20000)
    bj, x_bj = solve(sc, 0, False)
    loc, x_loc = solve(sc, 5, False)
    two, x_two = solve(sc, 5, True)
    scale = np.abs(x_bj).max()
    for x in (x_loc, x_two):
        assert np.abs(x - x_bj).max() <= 1e-6 * scale
    assert two < loc < bj


def test_linear_coarse_fields_converge_and_cut_iterations():
    """Translation plus linear fields on 2-block coarse blocks: the same
    solution, fewer iterations than translations on 1-block blocks, and a
    symmetric positive-definite coarse system of 12 unknowns per block (9
    where an axis is dropped)."""
    sc = scenes.config_large(side=40, max_iter=20000)
    _, x_bj = solve(sc, 0, False)
    tr, _ = solve(sc, 5, True)
    s = oracle_sim(sc, 1e-9, degree=5, block_rows=256)
    s.set_preconditioner(5, 30.0, 256, coarse="linear", coarse_rows=512)
    s.step(sc["dt"])
    lin, _, status = s.stats()
    assert status == 0
    assert np.abs(s.dump_system()[5] - x_bj).max() <= 1e-6 * np.abs(x_bj).max()
    assert lin < tr
    A = s.coarse_system()
    assert 36 <= A.shape[0] <= 48 and A.shape[0] % 3 == 0  # 4 coarse blocks, 3 to 4 fields each
    np.testing.assert_allclose(A, A.T, rtol=1e-10, atol=1e-9 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0


def test_block_jacobi_with_the_coarse_level():
    # the streamed device kernel's preconditioner: block-Jacobi plus the
    # coarse level (degree 0 with coarse); same solution, fewer iterations
    sc = scenes.config_large(side=48, steps=2)
    a, b = oracle_sim(sc, 1e-10), oracle_sim(sc, 1e-10)
    b.set_preconditioner(0, 30.0, 512, coarse="linear", coarse_rows=512)
    for _ in range(2):
        a.step(sc["dt"])
        b.step(sc["dt"])
    assert np.abs(a.state()[0] - b.state()[0]).max() < 1e-9
    assert b.stats()[0] < 0.75 * a.stats()[0]  # 638 against 1140 here (strips of the caller order)
    with pytest.raises(ValueError):
        b.set_preconditioner(4, 30.0, 256)  # even degree


def test_explicit_coarse_bounds_restate_fixed_blocks_and_accept_ragged_ones():
    """Explicit coarse block starts (the device's batched blocks, one per CTA
    segment of an instance): bounds equal to fixed 512-row blocks give the
    same coarse system and iterations; ragged bounds converge to the same
    solution; bad bounds are rejected."""
    sc = scenes.config_large(side=40, steps=2)
    n = sc["pos"].shape[0]
    a, b, c = oracle_sim(sc, 1e-10), oracle_sim(sc, 1e-10), oracle_sim(sc, 1e-10)
    a.set_preconditioner(0, 60.0, 512, coarse="linear", coarse_rows=512)
    b.set_preconditioner(0, 60.0, 512, coarse="linear", coarse_rows=0)
    b.set_coarse_bounds(list(range(0, n, 512)) + [n])
    c.set_preconditioner(0, 60.0, 512, coarse="linear", coarse_rows=0)
    c.set_coarse_bounds([0, 96, 800, 832, n + 20])  # ragged; the last start past n ends the list
    for s in (a, b, c):
        s.step(sc["dt"])
        assert s.stats()[2] == 0
    np.testing.assert_array_equal(a.coarse_system(), b.coarse_system())
    assert a.stats()[0] == b.stats()[0]
    assert c.coarse_system().shape[0] <= 36  # three blocks
    assert np.abs(c.state()[0] - a.state()[0]).max() < 1e-8
    for bad in ([1, 5, n], [0, 10, 10, n], [0]):
        with pytest.raises(ValueError):
            c.set_coarse_bounds(bad)
