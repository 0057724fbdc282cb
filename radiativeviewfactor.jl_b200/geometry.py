"""Element geometry exported by the reference (src/Geometry.jl, re-exported
at src/RadiativeViewFactor.jl:27-28,33-46): shape functions, the physical
point, and the unit normal with the area (surface) or length (curve) element
of Quad8, Quad4, Line3 and Line2 elements, plus element_area.

Host helpers for callers of the reference's API; the device evaluates the
same formulas in its own tables.  `coords` is 3 x n_nodes, `nodes` holds
1-based node indices in the element's Gmsh order, as in the reference.
Sums follow the reference's order: x = x + N_a x_a from zero over the nodes,
|c| = sqrt(c.c) with the components added left to right.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["quad8_shape", "quad8_physical_point", "quad8_normal_and_area_element", "quad4_shape",
           "quad4_physical_point", "quad4_normal_and_area_element", "element_area", "line3_shape",
           "line3_physical_point", "line3_normal_and_length_element", "line2_shape", "line2_physical_point",
           "line2_normal_and_length_element"]


def quad8_shape(xi: float, eta: float):
    """src/Geometry.jl:35-70: N, dN/dxi, dN/deta of the 8-node serendipity quad."""
    x, e = float(xi), float(eta)
    N = [0.25 * (1 - x) * (1 - e) * (-x - e - 1), 0.25 * (1 + x) * (1 - e) * (x - e - 1),
         0.25 * (1 + x) * (1 + e) * (x + e - 1), 0.25 * (1 - x) * (1 + e) * (-x + e - 1),
         0.5 * (1 - x * x) * (1 - e), 0.5 * (1 + x) * (1 - e * e),
         0.5 * (1 - x * x) * (1 + e), 0.5 * (1 - x) * (1 - e * e)]
    dx = [0.25 * (1 - e) * (2 * x + e), 0.25 * (1 - e) * (2 * x - e), 0.25 * (1 + e) * (2 * x + e),
          0.25 * (1 + e) * (2 * x - e), -x * (1 - e), 0.5 * (1 - e * e), -x * (1 + e), -0.5 * (1 - e * e)]
    de = [0.25 * (1 - x) * (x + 2 * e), 0.25 * (1 + x) * (-x + 2 * e), 0.25 * (1 + x) * (x + 2 * e),
          0.25 * (1 - x) * (-x + 2 * e), -0.5 * (1 - x * x), -e * (1 + x), 0.5 * (1 - x * x), -e * (1 - x)]
    return np.array(N), np.array(dx), np.array(de)


def quad4_shape(xi: float, eta: float):
    """src/Geometry.jl:119-128: bilinear quad."""
    x, e = float(xi), float(eta)
    N = [0.25 * (1 - x) * (1 - e), 0.25 * (1 + x) * (1 - e), 0.25 * (1 + x) * (1 + e), 0.25 * (1 - x) * (1 + e)]
    dx = [-0.25 * (1 - e), 0.25 * (1 - e), 0.25 * (1 + e), -0.25 * (1 + e)]
    de = [-0.25 * (1 - x), -0.25 * (1 + x), 0.25 * (1 + x), 0.25 * (1 - x)]
    return np.array(N), np.array(dx), np.array(de)


def line3_shape(xi: float):
    """src/Geometry.jl:236-244: N = (-xi(1-xi)/2, xi(1+xi)/2, 1-xi^2) and dN/dxi."""
    x = float(xi)
    return (np.array([-0.5 * x * (1.0 - x), 0.5 * x * (1.0 + x), 1.0 - x * x]),
            np.array([-0.5 + x, 0.5 + x, -2.0 * x]))


def line2_shape(xi: float):
    """src/Geometry.jl:309-311."""
    x = float(xi)
    return np.array([0.5 * (1.0 - x), 0.5 * (1.0 + x)]), np.array([-0.5, 0.5])


def _combine(coords, nodes, w):
    """sum_a w_a x_a, accumulated from zero in node order."""
    out = [0.0, 0.0, 0.0]
    for a, wa in enumerate(w):
        k = int(nodes[a]) - 1
        for c in range(3):
            out[c] = out[c] + float(wa) * float(coords[c, k])
    return out


def _unit_and_length(v):
    length = math.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return np.array([v[0] / length, v[1] / length, v[2] / length]), length


def _surface_normal(coords, nodes, dx, de):
    a = _combine(coords, nodes, dx)
    b = _combine(coords, nodes, de)
    c = [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]
    return _unit_and_length(c)


def quad8_physical_point(coords, nodes, xi: float, eta: float) -> np.ndarray:
    """src/Geometry.jl:77-88."""
    return np.array(_combine(coords, nodes, quad8_shape(xi, eta)[0]))


def quad8_normal_and_area_element(coords, nodes, xi: float, eta: float):
    """src/Geometry.jl:95-111: (unit normal, dA) = (c/|c|, |c|), c = x_xi x x_eta."""
    _, dx, de = quad8_shape(xi, eta)
    return _surface_normal(coords, nodes, dx, de)


def quad4_physical_point(coords, nodes, xi: float, eta: float) -> np.ndarray:
    """src/Geometry.jl:136-150."""
    return np.array(_combine(coords, nodes, quad4_shape(xi, eta)[0]))


def quad4_normal_and_area_element(coords, nodes, xi: float, eta: float):
    """src/Geometry.jl:154-171."""
    _, dx, de = quad4_shape(xi, eta)
    return _surface_normal(coords, nodes, dx, de)


def element_area(coords, nodes, nquad: int = 4) -> float:
    """src/Geometry.jl:180-210: area of one Quad8 element.  nquad <= 2: the
    2 x 2 Gauss rule; nquad = 3: the 3 x 3 rule with nodes +-sqrt(3/5), 0;
    nquad >= 4: gauss_legendre_2d(nquad) (the library's rule, bit for bit
    the reference's)."""
    if nquad >= 4:
        from . import _abi
        pts, wts = _abi.quadrature_rule(0, nquad)
        A = 0.0
        for k in range(wts.size):
            A += float(wts[k]) * quad8_normal_and_area_element(coords, nodes, pts[0, k], pts[1, k])[1]
        return A
    if nquad <= 2:
        p1 = [-1 / math.sqrt(3), 1 / math.sqrt(3)]
        w1 = [1.0, 1.0]
    else:
        p1 = [-math.sqrt(3 / 5), 0.0, math.sqrt(3 / 5)]
        w1 = [5 / 9, 8 / 9, 5 / 9]
    A = 0.0
    for x, wx in zip(p1, w1):
        for e, we in zip(p1, w1):
            A += wx * we * quad8_normal_and_area_element(coords, nodes, x, e)[1]
    return A


def line3_physical_point(coords, nodes, xi: float) -> np.ndarray:
    """src/Geometry.jl:252-262: nodes = (left corner, right corner, midpoint)."""
    return np.array(_combine(coords, nodes, line3_shape(xi)[0]))


def _line_normal(coords, nodes, dN):
    t = _combine(coords, nodes, dN)
    u, dL = _unit_and_length(t)
    return np.array([-u[1], u[0], 0.0]), dL  # the tangent turned 90 degrees counter-clockwise in xy


def line3_normal_and_length_element(coords, nodes, xi: float):
    """src/Geometry.jl:264-294: (in-plane unit normal, dL)."""
    return _line_normal(coords, nodes, line3_shape(xi)[1])


def line2_physical_point(coords, nodes, xi: float) -> np.ndarray:
    """src/Geometry.jl:318-330."""
    return np.array(_combine(coords, nodes, line2_shape(xi)[0]))


def line2_normal_and_length_element(coords, nodes, xi: float):
    """src/Geometry.jl:332-348."""
    return _line_normal(coords, nodes, line2_shape(xi)[1])
