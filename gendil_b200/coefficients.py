"""Coefficients on Cartesian meshes.

A scalar coefficient is ``constant + sum_t prod_k f_{t,k}(x_k)`` (optionally times a per-element
device array).  Each ``f_{t,k}`` is a 1D function of the coordinate along axis ``k``; the library
samples it at the mesh's 1D quadrature and face coordinates, so its value at every quadrature
point is exactly the value the reference's pointwise lambda would return for functions of this
form (massoperator.hpp:78, advectionoperator.hpp:317).

Ready-made fields used by the reference's tests and benchmark configurations:
:func:`density_poly` (``1 + x0 x1 + x_{D-1}^2``, test-mass-3d-generic.cpp:114-120),
:func:`velocity_bubble` (``-x_i (1 - x_i)``, test-advection-3d-generic.cpp),
:func:`velocity_sincos` (``(1 + 0.5 sin 2 pi y, 0.5 + 0.25 cos 2 pi z, 0.25)``) and
:func:`velocity_phase_space` (``(v, -x + 0.5)`` on (x, v)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Coefficient:
    constant: float = 0.0
    terms: list = field(default_factory=list)  # list of {axis: callable(float) -> float | ndarray}
    element_factor: object = None               # device tensor (num_elements,) or None

    @staticmethod
    def tabulate(fn, coords):
        """Evaluate a 1D factor at the table coordinates (scalar Python calls: C-libm results)."""
        if isinstance(fn, np.ndarray):
            if fn.shape != coords.shape:
                raise ValueError("tabulated factor has the wrong length")
            return fn
        return np.array([fn(float(x)) for x in coords], dtype=np.float64)


def as_coefficient(c, dim):
    if isinstance(c, Coefficient):
        return c
    if np.isscalar(c):
        return Coefficient(constant=float(c))
    raise TypeError("coefficient must be a number or a Coefficient")


def constant(value):
    return Coefficient(constant=float(value))


def density_poly(dim):
    """1 + x0 * x_{1 % D} + x_{D-1}^2."""
    a1 = 1 % dim
    if a1 == 0:
        t1 = {0: lambda x: x * x}
    else:
        t1 = {0: lambda x: x, a1: lambda x: x}
    t2 = {dim - 1: lambda x: x * x}
    return Coefficient(constant=1.0, terms=[t1, t2])


def velocity_constant(values):
    return [Coefficient(constant=float(v)) for v in values]


def velocity_bubble(dim):
    return [Coefficient(terms=[{i: (lambda x: -x * (1.0 - x))}]) for i in range(dim)]


def velocity_sincos(dim):
    out = []
    for i in range(dim):
        if i == 0:
            out.append(Coefficient(terms=[{1 % dim: (lambda x: 1.0 + 0.5 * math.sin(2.0 * math.pi * x))}]))
        elif i == 1:
            out.append(Coefficient(terms=[{2 % dim: (lambda x: 0.5 + 0.25 * math.cos(2.0 * math.pi * x))}]))
        else:
            out.append(Coefficient(constant=0.25))
    return out


def velocity_phase_space(dim):
    if dim % 2:
        raise ValueError("phase-space velocity needs an even dimension")
    h = dim // 2
    out = []
    for i in range(dim):
        if i < h:
            out.append(Coefficient(terms=[{i + h: (lambda x: x)}]))
        else:
            out.append(Coefficient(terms=[{i - h: (lambda x: -x + 0.5)}]))
    return out


def density_separable(dim):
    """(1 + 0.5 x0) (1 + x1^2) (2 - x2): one separable product (dim >= 3)."""
    if dim < 3:
        raise ValueError("density_separable needs dim >= 3")
    return Coefficient(terms=[{0: lambda x: 1.0 + 0.5 * x, 1: lambda x: 1.0 + x * x, 2: lambda x: 2.0 - x}])


def sigma_preset(kind, dim, c=1.0):
    """The oracle's sigma presets: 0 constant c, 1 density_poly, 2 density_separable."""
    if kind == 0:
        return constant(c)
    return density_poly(dim) if kind == 1 else density_separable(dim)


def beta_preset(kind, dim, c=None):
    """The oracle's velocity presets: 0 constant, 1 bubble, 2 sin/cos, 3 phase space."""
    if kind == 0:
        return velocity_constant(list(c)[:dim])
    if kind == 1:
        return velocity_bubble(dim)
    if kind == 2:
        return velocity_sincos(dim)
    return velocity_phase_space(dim)
