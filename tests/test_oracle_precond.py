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


def test_coarse_level_alone_is_rejected():
    sc = scenes.config_small(side=8, steps=1)
    s = oracle_sim(sc, 1e-9)
    with pytest.raises(ValueError):
        s.set_preconditioner(0, 30.0, 256, coarse=True)
    with pytest.raises(ValueError):
        s.set_preconditioner(4, 30.0, 256)  # even degree
