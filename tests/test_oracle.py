"""CPU: the oracle restatement against the reference's golden fixtures (and the live reference
library when it is built here)."""
import numpy as np
import pytest

from helpers import APPLY_TOL, golden, have_reference, inputs, oracle, rel_max

CASES, ARR = golden()


def test_fill_random_matches_reference():
    for seed in (0, 1, 2, 3, 12345):
        np.testing.assert_array_equal(oracle().fill_random(256, seed), ARR[f"rng_seed{seed}"])


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("n", range(1, 9))
def test_points_close_to_reference_tables(kind, n):
    x, w = oracle().points(kind, n)
    # the reference stores its tables to ~15 significant digits
    np.testing.assert_allclose(x, ARR[f"points_{kind}_{n}_x"], rtol=0, atol=5e-15)
    np.testing.assert_allclose(w, ARR[f"points_{kind}_{n}_w"], rtol=0, atol=5e-15)
    assert abs(w.sum() - 1.0) < 1e-14


@pytest.mark.parametrize("case", CASES["mass"], ids=lambda c: c["id"])
def test_mass_oracle_vs_reference(case):
    y = oracle().mass_apply(case, inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", CASES["advection"], ids=lambda c: c["id"])
def test_advection_oracle_vs_reference(case, mode):
    y = oracle().advection_apply(case, inputs(case), mode)
    assert rel_max(y, ARR[f"{case['id']}_mode{mode}_y"]) <= APPLY_TOL


@pytest.mark.parametrize("case", CASES["cg"], ids=lambda c: c["id"])
def test_cg_oracle_vs_reference(case):
    u = oracle().fill_random(len(ARR[f"{case['id']}_x"]), 0)
    b = oracle().mass_apply(case, u)
    x, info = oracle().mass_cg(case, b, np.zeros_like(b), case["max_iters"], case["tol"])
    # The reference's Dot is an OpenMP reduction (dot.hpp:117-131), so its own iteration count
    # moves with the thread count on long runs: +-1 iteration, or 1% beyond 100 iterations.
    assert abs(info["iterations"] - case["iterations"]) <= max(1, case["iterations"] // 100)
    assert info["success"] == case["success"]
    if case["success"]:
        assert rel_max(x, ARR[f"{case['id']}_x"]) < 1e-6


@pytest.mark.parametrize("case", CASES["gmres"], ids=lambda c: c["id"])
def test_gmres_oracle_vs_reference(case):
    b = oracle().fill_random(len(ARR[f"{case['id']}_x"]), 2)
    x, info = oracle().system_gmres(case, b, np.zeros_like(b), case["max_iters"], case["restart"], case["tol"])
    assert abs(info["iterations"] - case["iterations"]) <= 1
    assert info["success"] and info["relative_error"] <= case["tol"]
    assert rel_max(x, ARR[f"{case['id']}_x"]) < 1e-8


@pytest.mark.skipif(not have_reference(), reason="reference library not built here")
def test_oracle_vs_live_reference_config1_mass():
    """Config-1 size (16^3, p=3, q=4): the restatement against the reference itself."""
    from helpers import Reference
    case = {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16] * 3, "h": [1 / 16] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "sigma_kind": 0, "sigma_c": 1.0, "seed": 0}
    x = inputs(case)
    assert rel_max(oracle().mass_apply(case, x), Reference().mass_apply(case, x)) <= APPLY_TOL


@pytest.mark.skipif(not have_reference(), reason="reference library not built here")
def test_oracle_vs_live_reference_advection_16():
    from helpers import Reference
    case = {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16] * 3, "h": [1 / 16] * 3, "origin": [0.0] * 3,
            "periodic": [0] * 3, "beta_kind": 2, "g": 0.0, "seed": 1}
    x = inputs(case)
    assert rel_max(oracle().advection_apply(case, x, 1), Reference().advection_apply(case, x, 1)) <= APPLY_TOL


@pytest.mark.skipif(not have_reference(), reason="reference library not built here")
@pytest.mark.parametrize("case", CASES["sipdg"], ids=lambda c: c["id"])
def test_sipdg_fixtures_reproduce_live_reference(case):
    """The stored SIPDG fixtures are what the reference's generic weak form computes here."""
    from helpers import Reference
    ref = Reference()
    y = ref.sipdg_apply(case, ARR[f"{case['id']}_mu"], case["sigma"], case["kappa"], case["boundary"], inputs(case))
    assert rel_max(y, ARR[f"{case['id']}_y"]) <= 1e-14


@pytest.mark.skipif(not have_reference(), reason="reference library not built here")
@pytest.mark.parametrize("case", CASES["diffusion"], ids=lambda c: c["id"])
def test_legacy_diffusion_equals_generic_sipdg(case):
    """The reference's legacy MakeDiffusionOperator and its generic SIPDG weak form (constant
    diffusivity, boundary terms on) agree, as the reference's own diffusion tests check, and the
    stored fixture is the legacy operator's output."""
    from helpers import Reference
    ref = Reference()
    x = inputs(case)
    ne = int(np.prod(case["sizes"]))
    legacy = ref.diffusion_legacy_apply(case, case["diffusivity"], case["sigma"], case["kappa"], x)
    generic = ref.sipdg_apply(case, np.full(ne, case["diffusivity"]), case["sigma"], case["kappa"], 1, x)
    assert rel_max(legacy, ARR[f"{case['id']}_y"]) <= 1e-14
    assert rel_max(generic, legacy) <= 1e-13
