"""CPU: pin the MLP oracle (oracle/mlp_oracle.py) by central finite differences."""
import numpy as np

import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    P = rng.normal(0, 0.3, mo.N_PARAMS)
    x = rng.normal(0, 1, (7, mo.K_IN))
    t = rng.normal(0, 1, (7, mo.K_OUT))
    g = mo.grad(P, x, t)
    idx = list(range(0, mo.N_PARAMS, 97)) + [mo.O_B1, mo.O_B2 + 3, mo.O_B3, mo.O_B3 + 3]
    for i in idx:
        h = 1e-6
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (mo.loss(Pp, x, t) - mo.loss(Pm, x, t)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_layout():
    assert mo.N_PARAMS == 4740
