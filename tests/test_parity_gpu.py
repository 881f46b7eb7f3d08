"""GPU: the sm_100a operators against the reference's golden outputs and the oracle.

FP64 applies must match to APPLY_TOL = 1e-13 relative in max norm per apply."""
import numpy as np
import pytest

from helpers import APPLY_TOL, cuda_apply, golden, inputs, make_operator, oracle, rel_max

pytestmark = pytest.mark.gpu
CASES, ARR = golden()


@pytest.mark.parametrize("case", CASES["mass"], ids=lambda c: c["id"])
def test_mass_vs_reference_golden(case):
    op = make_operator(case, "mass")
    y = cuda_apply(op, inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_advection_vs_reference_golden(case, mode):
    op = make_operator(case, "adv", mode)
    y = cuda_apply(op, inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_mode{mode}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_transpose_adjoint_identity(case, mode):
    """<A x, z> = <x, A^T z> for the linear part (inflow value 0)."""
    case = dict(case, g=0.0)
    op = make_operator(case, "adv", mode)
    x = inputs(case, seed=5)
    z = inputs(case, seed=6)
    ax = cuda_apply(op, x)
    atz = cuda_apply(op, z, transpose=True)
    lhs, rhs = float(ax @ z), float(x @ atz)
    assert abs(lhs - rhs) <= 1e-12 * (np.abs(ax).sum() * np.abs(z).max() + 1e-300)


def _c1():
    return {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16] * 3, "h": [1 / 16] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "sigma_kind": 0, "sigma_c": 1.0, "seed": 0}


def _c2(n=64):
    return {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [n] * 3, "h": [1 / n] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "beta_kind": 2, "g": 0.0, "seed": 1}


def test_config1_mass_full_size_vs_oracle():
    case = _c1()
    x = inputs(case)
    y = cuda_apply(make_operator(case, "mass"), x)
    assert rel_max(y, oracle().mass_apply(case, x)) <= APPLY_TOL


def test_config2_advection_full_size_vs_oracle():
    case = _c2(64)
    x = inputs(case)
    y = cuda_apply(make_operator(case, "adv", 1), x)
    assert rel_max(y, oracle().advection_apply(case, x, 1)) <= APPLY_TOL


def test_fp32_apply_error_bound():
    case = _c2(16)
    op = make_operator(case, "adv", 1)
    x = inputs(case)
    y64 = cuda_apply(op, x)
    y32 = cuda_apply(op, x, f32=True)
    assert rel_max(y32, y64) < 1e-5
