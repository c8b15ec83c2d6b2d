"""GPU: chysx_mlp_gradients_noalloc (workspace in a static device array of the
library) against chysx_mlp_gradients (caller workspace) on the same inputs,
for two calls in a row, plus its size limit.

The file is named so that pytest collects it last: it must pass both on its
own and after every other test has used the device."""
import ctypes

import numpy as np
import pytest

import oracle.mlp_oracle as M
from chysx import capi

pytestmark = pytest.mark.gpu

# the library's own limit (CHYSX_MLP_NOALLOC_MAX_ROWS), so the boundary cases
# follow the header if it changes
MAX_ROWS = int(capi.lib().chysx_mlp_noalloc_max_rows())
# Same kernels and the same summation order on both paths: the results are
# expected to be identical; the bounds only leave room for FP32 re-association.
TOL_GRAD_REL = 1e-6   # relative to max |gradient| per parameter block
TOL_LOSS_REL = 1e-12


def _params(rng):
    p = M.init_params(rng, rng.standard_normal(M.N_IN) * 0.1, rng.uniform(0.5, 2.0, M.N_IN),
                      np.array([0.1, -0.2, 0.05]), np.array([0.5, 1.5, 1.0]))
    for k in ("b1", "b2", "b3", "b4"):
        a, b = M.OFF[k]
        p[a:b] = rng.standard_normal(b - a) * 0.1
    return p.astype(np.float32)


def _case(seed, rows):
    import torch

    rng = np.random.default_rng(seed)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    return (dev(_params(rng)), dev(rng.standard_normal((rows, M.N_IN)) * 1.5),
            dev(rng.standard_normal((rows, M.N_OUT)) * 0.7))


def _with_workspace(p, f, t, rows):
    import torch

    ws = torch.empty(int(capi.lib().chysx_mlp_workspace_bytes(rows)), dtype=torch.uint8, device="cuda")
    grad = torch.full_like(p, float("nan"))
    loss = ctypes.c_double()
    capi.check(capi.lib().chysx_mlp_gradients(p.data_ptr(), f.data_ptr(), t.data_ptr(), rows, grad.data_ptr(),
                                              ctypes.byref(loss), ws.data_ptr(), ws.numel(), 0))
    return grad.cpu().numpy(), loss.value


def _no_alloc(p, f, t, rows, grad):
    loss = ctypes.c_double()
    capi.check(capi.lib().chysx_mlp_gradients_noalloc(p.data_ptr(), f.data_ptr(), t.data_ptr(), rows,
                                                      grad.data_ptr(), ctypes.byref(loss), 0))
    return grad.cpu().numpy(), loss.value


def _assert_close(g, l, g_ref, l_ref):
    assert np.all(np.isfinite(g))
    for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4"):
        a, b = M.OFF[k]
        scale = max(float(np.abs(g_ref[a:b]).max()), 1e-30)
        assert float(np.abs(g[a:b] - g_ref[a:b]).max()) <= TOL_GRAD_REL * scale, k
    assert np.all(g[:M.OFF["w1"][0]] == 0.0)
    assert abs(l - l_ref) <= TOL_LOSS_REL * abs(l_ref)


def test_two_calls_in_a_row_match_the_workspace_entry_point():
    import torch

    # the largest batch first, then a smaller one: the second call must not
    # see anything the first left in the shared scratch
    cases = [(_case(11, MAX_ROWS), MAX_ROWS), (_case(12, 777), 777)]
    refs = [_with_workspace(*c, rows) for c, rows in cases]
    grads = [torch.full_like(c[0], float("nan")) for c, _ in cases]
    outs = [_no_alloc(*c, rows, g) for (c, rows), g in zip(cases, grads)]
    for (g, l), (g_ref, l_ref) in zip(outs, refs):
        _assert_close(g, l, g_ref, l_ref)


def test_rows_beyond_the_limit_are_rejected_before_any_launch():
    import torch

    p, f, t = _case(13, MAX_ROWS + 1)
    grad = torch.full_like(p, 7.0)
    loss = ctypes.c_double(-1.0)
    rc = capi.lib().chysx_mlp_gradients_noalloc(p.data_ptr(), f.data_ptr(), t.data_ptr(), MAX_ROWS + 1,
                                                grad.data_ptr(), ctypes.byref(loss), 0)
    assert rc == capi.ERR_INVALID_ARGUMENT
    assert str(MAX_ROWS) in capi.lib().chysx_last_error().decode()
    torch.cuda.synchronize()
    assert bool((grad == 7.0).all()) and loss.value == -1.0
