"""Test infrastructure only: ctypes bindings to the CPU oracle libraries.

Imported by ``tests/`` and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``;
never by the product package.

Two libraries, one calling convention:

* ``oracle/_ref/libgendil_ref.so`` -- the GenDiL reference operators compiled from the
  reference's own headers (``oracle/ref_*.cpp``; built only where the reference source is
  present, then copied with the repository).
* ``oracle/_build/libdgoracle.so`` -- the plain-C restatement (``oracle/dg_oracle.c``).

A *case* is a dict describing one mesh/space/coefficient configuration::

    {"D": 3, "P": 3, "Q": 4, "basis": 0, "sizes": [16]*3, "h": [1/16]*3, "origin": [0]*3,
     "periodic": [0]*3, "sigma_kind": 0, "sigma_c": 1.0, "beta_kind": 2, "beta_c": [...],
     "g": 0.0}

Coefficient presets (shared with ``tests/coefficients.py``):
sigma 0 = constant ``sigma_c``; 1 = ``1 + x0*x1 + x_{D-1}^2`` (test-mass-3d-generic.cpp:114-120).
beta 0 = constant ``beta_c``; 1 = ``-x_i (1 - x_i)`` (test-advection-3d-generic.cpp);
2 = ``(1 + 0.5 sin 2 pi x1, 0.5 + 0.25 cos 2 pi x2, 0.25, ...)``; 3 = phase space ``(v, -x + 0.5)``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libgendil_ref.so")
ORACLE_LIB = os.path.join(HERE, "_build", "libdgoracle.so")

_cd = ctypes.c_double
_ci = ctypes.c_int


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def num_dofs(case):
    return int(np.prod(case["sizes"])) * (case["P"] + 1) ** case["D"]


class _Lib:
    prefix = ""

    def __init__(self, path):
        self.path = path
        self.lib = ctypes.CDLL(path)

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    @staticmethod
    def _mesh(case):
        D = case["D"]
        sizes = np.ascontiguousarray(case["sizes"], dtype=np.int64)
        h = np.ascontiguousarray(case["h"], dtype=np.float64)
        origin = np.ascontiguousarray(case.get("origin", [0.0] * D), dtype=np.float64)
        periodic = np.ascontiguousarray(case.get("periodic", [0] * D), dtype=np.int32)
        return sizes, h, origin, periodic

    def fill_random(self, n, seed, lo=-1.0, hi=1.0):
        out = np.empty(n, dtype=np.float64)
        self._fn("fill_random")(_p(out), ctypes.c_long(n), ctypes.c_uint(seed), _cd(lo), _cd(hi))
        return out

    def points(self, kind, npts):
        c = np.zeros(8)
        w = np.zeros(8)
        rc = self._fn("points")(kind, npts, _p(c), _p(w))
        if rc != 0:
            raise ValueError("points: unsupported")
        return c[:npts].copy(), w[:npts].copy()

    def mass_apply(self, case, x):
        sizes, h, origin, periodic = self._mesh(case)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        rc = self._fn("mass_apply")(case["D"], case["P"], case["Q"], case["basis"], _p(sizes), _p(h), _p(origin),
                                    _p(periodic), case.get("sigma_kind", 0), _cd(case.get("sigma_c", 1.0)), _p(x), _p(y))
        if rc != 0:
            raise NotImplementedError(f"{self.path}: mass case not available (rc={rc})")
        return y

    def advection_apply(self, case, x, mode):
        """mode 0: no boundary faces, 1: inflow value case['g'], 2: mass + advection (interior)."""
        sizes, h, origin, periodic = self._mesh(case)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        bc = np.zeros(8)
        bc[: case["D"]] = case.get("beta_c", [0.0] * case["D"])
        rc = self._fn("advection_apply")(case["D"], case["P"], case["Q"], case["basis"], _p(sizes), _p(h), _p(origin),
                                         _p(periodic), mode, case.get("beta_kind", 0), _p(bc), _cd(case.get("g", 0.0)),
                                         case.get("sigma_kind", 0), _cd(case.get("sigma_c", 1.0)), _p(x), _p(y))
        if rc != 0:
            raise NotImplementedError(f"{self.path}: advection case not available (rc={rc})")
        return y

    def mass_cg(self, case, b, x0, max_iters, tol):
        sizes, h, origin, periodic = self._mesh(case)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64, copy=True)
        it, rel, ok = _ci(), _cd(), _ci()
        rc = self._fn("mass_cg")(case["D"], case["P"], case["Q"], case["basis"], _p(sizes), _p(h), _p(origin),
                                 _p(periodic), case.get("sigma_kind", 0), _cd(case.get("sigma_c", 1.0)), _p(b), _p(x),
                                 max_iters, _cd(tol), ctypes.byref(it), ctypes.byref(rel), ctypes.byref(ok))
        if rc != 0:
            raise NotImplementedError(f"{self.path}: cg case not available (rc={rc})")
        return x, {"iterations": it.value, "relative_error": rel.value, "success": bool(ok.value)}

    def system_gmres(self, case, b, x0, max_iters, restart, tol):
        """GMRES(restart) on sigma_c * M + A(inflow g)."""
        sizes, h, origin, periodic = self._mesh(case)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x0, dtype=np.float64, copy=True)
        bc = np.zeros(8)
        bc[: case["D"]] = case.get("beta_c", [0.0] * case["D"])
        it, rel, ok = _ci(), _cd(), _ci()
        rc = self._fn("system_gmres")(case["D"], case["P"], case["Q"], case["basis"], _p(sizes), _p(h), _p(origin),
                                      _p(periodic), _cd(case.get("sigma_c", 1.0)), case.get("beta_kind", 0), _p(bc),
                                      _cd(case.get("g", 0.0)), _p(b), _p(x), max_iters, restart, _cd(tol),
                                      ctypes.byref(it), ctypes.byref(rel), ctypes.byref(ok))
        if rc != 0:
            raise NotImplementedError(f"{self.path}: gmres case not available (rc={rc})")
        return x, {"iterations": it.value, "relative_error": rel.value, "success": bool(ok.value)}


class Reference(_Lib):
    """The reference's own operators (compiled from its headers)."""

    prefix = "gref_"

    def __init__(self, path=REF_LIB):
        super().__init__(path)
        self.lib.gref_time_advection.restype = ctypes.c_double

    def num_threads(self):
        return int(self.lib.gref_num_threads())

    def sipdg_apply(self, case, mu_elem, sigma, kappa, boundary, x):
        """The reference's generic SIPDG form (part_sipdg.cpp): mu per element, tau = kappa / h,
        sigma = -1 SIPG / +1 NIPG / 0 IIPG, Dirichlet-0 boundary terms when `boundary`."""
        sizes, h, origin, periodic = self._mesh(case)
        x = np.ascontiguousarray(x, dtype=np.float64)
        mu = np.ascontiguousarray(mu_elem, dtype=np.float64)
        y = np.zeros_like(x)
        rc = self.lib.gref_sipdg_apply(case["D"], case["P"], case["Q"], case.get("basis", 0), _p(sizes), _p(h),
                                       _p(origin), _p(periodic),
                                       _p(mu), _cd(sigma), _cd(kappa), int(boundary), _p(x), _p(y))
        if rc != 0:
            raise NotImplementedError("sipdg_apply: case not instantiated")
        return y

    def diffusion_legacy_apply(self, case, d, sigma, kappa, x):
        """The reference's legacy MakeDiffusionOperator (part_sipdg.cpp): constant diffusivity d,
        interior and boundary faces, tau = kappa / h."""
        sizes, h, origin, periodic = self._mesh(case)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        rc = self.lib.gref_diffusion_legacy_apply(case["D"], case["P"], case["Q"], case.get("basis", 0), _p(sizes),
                                                  _p(h), _p(origin), _p(periodic), _cd(d), _cd(sigma), _cd(kappa), _p(x), _p(y))
        if rc != 0:
            raise NotImplementedError("diffusion_legacy_apply: case not instantiated")
        return y

    def time_advection(self, case, x, pairs):
        """Seconds per apply of the reference advection operator (inflow value case['g'])."""
        sizes, h, origin, _ = self._mesh(case)
        x = np.array(x, dtype=np.float64, copy=True)
        y = np.zeros_like(x)
        bc = np.zeros(8)
        bc[: case["D"]] = case.get("beta_c", [0.0] * case["D"])
        t = self.lib.gref_time_advection(case["D"], case["P"], case["Q"], case["basis"], _p(sizes), _p(h), _p(origin),
                                         case.get("beta_kind", 0), _p(bc), _cd(case.get("g", 0.0)), pairs, _p(x), _p(y))
        if t < 0:
            raise NotImplementedError("time_advection: case not instantiated")
        return t


class Oracle(_Lib):
    """The plain-C restatement."""

    prefix = "dgo_"

    def __init__(self, path=ORACLE_LIB):
        super().__init__(path)


def have_reference():
    return os.path.exists(REF_LIB)


def have_oracle():
    return os.path.exists(ORACLE_LIB)
