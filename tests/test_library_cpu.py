"""CPU: the C-ABI library loads, exports every declared symbol, and validates arguments
(no kernel launches here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = []
    for name in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", name)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms += re.findall(r"\b(dgop_[a-z0-9_]+)\s*\(", text)
    return sorted(set(syms))


def test_library_exports_every_declared_symbol():
    import gendil_b200 as g
    L = g.lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_version_string():
    import gendil_b200 as g
    assert b"sm_100a" in g.lib().dgop_version()


def test_space_create_and_counts():
    import gendil_b200 as g
    sp = g.Space(3, [4, 5, 6], order=3)
    assert sp.num_elements == 120
    assert sp.num_dofs == 120 * 64
    c = sp.coordinates(4, 1)
    assert c.shape == (5 * 6,)
    # element 2, lower face sits at 2 * h, upper face at 3 * h
    assert abs(c[2 * 6 + 4] - 2 / 5) < 1e-15 and abs(c[2 * 6 + 5] - 3 / 5) < 1e-15


@pytest.mark.parametrize("bad", [dict(dim=0), dict(dim=7), dict(order=8), dict(order=-1), dict(basis=3),
                                 dict(h=-1.0), dict(n_elem=0)])
def test_space_rejects_bad_arguments(bad):
    import gendil_b200 as g
    kw = dict(dim=3, n_elem=4, h=0.25, order=2, basis=g.GLL)
    kw.update(bad)
    dim = kw.pop("dim")
    with pytest.raises(g.DGOPError) as ei:
        g.Space(dim, kw["n_elem"] if dim < 1 or dim > 6 else [kw["n_elem"]] * dim,
                h=[kw["h"]] * max(dim, 1), order=kw["order"], basis=kw["basis"])
    assert ei.value.code == -1


def test_null_handles_are_errors_not_crashes():
    import gendil_b200 as g
    L = g.lib()
    out = ctypes.c_void_p()
    assert L.dgop_space_create(3, None, None, None, None, 1, 0, ctypes.byref(out)) == -1
    assert L.dgop_apply(None, None, None, None) == -1
    assert b"null" in L.dgop_last_error()
    assert L.dgop_operator_destroy(None) == 0


def test_coefficient_tables_match_pointwise_presets():
    from gendil_b200 import coefficients as C
    import gendil_b200 as g
    sp = g.Space(3, [4, 4, 4], order=3)
    coords = sp.coordinates(4, 1)
    beta = C.velocity_sincos(3)
    tab = C.Coefficient.tabulate(beta[0].terms[0][1], coords)
    np.testing.assert_array_equal(tab, 1.0 + 0.5 * np.sin(2.0 * np.pi * coords))
