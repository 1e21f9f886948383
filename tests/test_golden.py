"""The CPU oracle against golden vectors written by the reference's own CUDA
step (tests/golden/make_golden.py): 3 steps of a small channel with the rotor
and of a small cavity, fixed-iteration mode, relative L2 <= 1e-10."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import MAXIT, STEPS, TOL, golden_cases, pack
from tests.helpers import rel_l2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["channel", "cavity"])
def test_oracle_matches_reference_golden(oracle, name):
    path = os.path.join(HERE, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip("golden vectors not generated yet")
    gold = np.load(path)
    from falm_b200 import cases
    from oracle.oracle import CaseStruct
    case = golden_cases()[name]
    cs = CaseStruct(case, use_inflow=False, maxit=MAXIT, tol=TOL)
    m = oracle.setup(cs)
    st = cases.initial_state(case)
    oracle.init_state(cs, m, st)
    stats = [oracle.step(cs, st, m, (q + 1) * case.dt) for q in range(STEPS)]
    got = pack(case, st, stats)
    for k in ("u", "uu", "p", "nut"):
        assert rel_l2(got[k], gold[k]) < 1e-10, (k, rel_l2(got[k], gold[k]))
    np.testing.assert_array_equal(got["it"], gold["it"])
    np.testing.assert_allclose(got["torque"], gold["torque"], rtol=1e-10)
    np.testing.assert_allclose(got["thrust"], gold["thrust"], rtol=1e-10)
    np.testing.assert_allclose(got["divnorm"], gold["divnorm"], rtol=1e-6, atol=1e-20)
