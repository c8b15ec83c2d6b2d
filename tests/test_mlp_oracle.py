"""CPU: the network oracle's analytic gradient against finite differences
(FP64, no BF16 emulation), and its parameter layout against the library's."""
import numpy as np

import oracle.mlp_oracle as M
from chysx import capi


def test_layout_matches_library():
    assert M.OFF["total"] == capi.lib().chysx_mlp_num_params()
    assert capi.lib().chysx_mlp_num_features() == M.N_IN


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    feat = rng.standard_normal((7, M.N_IN))
    targ = rng.standard_normal((7, M.N_OUT)) * 0.3
    p = M.init_params(rng, np.zeros(M.N_IN), np.ones(M.N_IN), np.zeros(3), np.ones(3)).astype(np.float64)
    for k in ("b1", "b2", "b3", "b4"):
        a, b = M.OFF[k]
        p[a:b] = rng.standard_normal(b - a) * 0.1
    loss, g = M.loss_and_grad(p, feat, targ, emulate_bf16=False)
    h = 1e-6
    for k in ("w1", "b1", "w2", "b3", "w4", "b4"):
        a, b = M.OFF[k]
        for q in rng.choice(np.arange(a, b), size=min(6, b - a), replace=False):
            pp, pm = p.copy(), p.copy()
            pp[q] += h
            pm[q] -= h
            fd = (M.loss_and_grad(pp, feat, targ, False)[0] - M.loss_and_grad(pm, feat, targ, False)[0]) / (2 * h)
            assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(fd), (k, q, fd, g[q])
