"""The oracle's SSAFEM restatement (oracle/ssafem_oracle.py) against the reference's SSAFEM
regression tables (test/regression/ssa/ssa_testi_fem.sh, ssa_testj_fem.sh,
ssafem_test_linear.sh, ssafem_test_plug.sh): the converged discrete solution reproduces every
printed error to its printed digits; plus the Jacobian against a finite difference of the
residual."""
import json
import os

import numpy as np
import pytest

from pism_b200 import verification as V
from oracle import ssafd_oracle as O
from oracle import ssafem_oracle as F

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_goldens.json")))
COLS = ("maxvector", "prcntavvec", "maxu", "maxv", "avu", "avv")
DIGITS = {"maxvector": 4, "prcntavvec": 5, "maxu": 4, "maxv": 4, "avu": 4, "avv": 4}

CASES = {
    "test_i_fem": lambda Mx, My: (V.build_test_i(My=My, Mx=Mx), lambda g, c: V.exact_velocity_i(g)),
    "test_j_fem": lambda Mx, My: (V.build_test_j(Mx, My), lambda g, c: V.exact_velocity_j(g)),
    "linear_fem": lambda Mx, My: (V.build_test_linear(Mx, My), V.exact_velocity_linear),
    "plug_fem": lambda Mx, My: (V.build_test_plug(Mx, My), V.exact_velocity_plug),
}


def fem_case(key, Mx, My):
    (g, c, f), exact = CASES[key](Mx, My)
    return g, c, f, exact(g, c)


@pytest.mark.parametrize("key,idx", [(k, i) for k in CASES for i in (0, 1)])
def test_oracle_reproduces_the_fem_regression_tables(key, idx):
    row = GOLDEN[key]["cases"][idx]
    g, c, f, exact = fem_case(key, row["Mx"], row["My"])
    vel, _ = F.SSAFEMOracle(*O.from_case(g, c, f)).solve()
    r = V.report(vel, exact)
    for col in COLS:
        assert round(r[col], DIGITS[col]) == pytest.approx(row[col], abs=0.6 * 10.0 ** -DIGITS[col]), col


def test_jacobian_is_the_derivative_of_the_residual():
    """central differences of F along a random direction at a random velocity, plastic till
    with grounded and floating quadrature points, against J d"""
    g, c, f = V.build_test_i(My=21, Mx=7)
    G, C, I = O.from_case(g, c, f)
    o = F.SSAFEMOracle(G, C, I)
    rng = np.random.default_rng(0)
    vel = rng.normal(0.0, 1e-4, (g.Mx, g.My, 2))
    d = rng.normal(0.0, 1e-4, vel.shape)
    d[o.bc] = 0.0
    h = 1e-4
    fd = (o.residual(vel + h * d) - o.residual(vel - h * d)) / (2 * h)
    Jd = (o.jacobian(vel) @ d.reshape(-1)).reshape(vel.shape)
    free = ~o.bc
    assert np.linalg.norm((fd - Jd)[free]) <= 1e-6 * np.linalg.norm(Jd[free])
    J = o.jacobian(vel)
    assert abs(J - J.T).max() <= 1e-9 * abs(J).max()   # the SSA's Newton Jacobian is symmetric
