"""The oracle against the reference's own known-answer tests.

Each test restates a testset of test/runtests.jl (line numbers cited) on the
CPU restatement in oracle/.  Values and tolerances are the reference's.
"""
import math

import numpy as np
import pytest

from conftest import load_pkg

ANALYTIC_PLATES = 0.19982  # test/runtests.jl:288,392,435


def _mesh(coords, elems, groups=None, soups=None, dim=2):
    rvf = load_pkg()
    SE = rvf.SurfaceElement
    tags = groups or {g: f"g{g}" for g in sorted({e[1] for e in elems})}
    return rvf.MeshData.from_elements(np.asarray(coords, dtype=float), [SE(tuple(n), g, f) for n, g, f in elems],
                                      tags, soups or {}, dim)


# ---------------------------------------------------------------- :16-31
def test_quadrature_pretabulated(orc):
    for n in range(1, 6):
        p, w = orc.gl_1d(n)
        assert len(p) == n
        assert abs(w.sum() - 2.0) < 1e-12
        P, W = orc.gl_2d(n)
        assert P.shape[1] == n * n
        assert abs(W.sum() - 4.0) < 1e-12
    p3, w3 = orc.gl_1d(3)
    assert abs(np.dot(w3, p3 ** 4) - 2 / 5) < 1e-12


# ---------------------------------------------------------------- :34-48
def test_quadrature_golub_welsch(orc):
    for n in range(6, 9):
        p, w = orc.gl_1d(n)
        assert len(p) == n and np.all(np.diff(p) > 0)
        assert abs(w.sum() - 2.0) < 1e-12
        P, W = orc.gl_2d(n)
        assert P.shape[1] == n * n and abs(W.sum() - 4.0) < 1e-12
    p6, w6 = orc.gl_1d(6)
    assert abs(np.dot(w6, p6 ** 10) - 2 / 11) < 1e-12


# ---------------------------------------------------------------- :51-67
def test_quad8_shape(orc):
    for xi, eta in [(-0.5, 0.3), (0.0, 0.0), (1.0, 1.0), (-1.0, -1.0)]:
        N, _, _ = orc.shape("quad8", xi, eta)
        assert abs(N.sum() - 1.0) < 1e-14
    ref = [(-1., -1.), (1., -1.), (1., 1.), (-1., 1.), (0., -1.), (1., 0.), (0., 1.), (-1., 0.)]
    for a, (xa, ea) in enumerate(ref):
        N, _, _ = orc.shape("quad8", xa, ea)
        for b in range(8):
            assert abs(N[b] - (1.0 if a == b else 0.0)) < 1e-13


# ---------------------------------------------------------------- :81-99
QUAD8_SQUARE = [[0.0, 1.0, 1.0, 0.0, 0.5, 1.0, 0.5, 0.0],
                [0.0, 0.0, 1.0, 1.0, 0.0, 0.5, 1.0, 0.5],
                [0.0] * 8]


def test_quad8_geometry(orc):
    m = orc.Mesh(_mesh(QUAD8_SQUARE, [((1, 2, 3, 4, 5, 6, 7, 8), 1, "quad")]))
    x, n, dA = orc.eval_point(m, 0, 0.0, 0.0)
    assert np.allclose(x, [0.5, 0.5, 0.0], atol=1e-14)
    assert np.allclose(n, [0.0, 0.0, 1.0], atol=1e-14)
    assert abs(dA - 0.25) < 1e-14
    # element_area(coords, nodes; nquad=4) (src/Geometry.jl:180-204)
    P, W = orc.gl_2d(4)
    A = sum(W[k] * orc.eval_point(m, 0, P[0, k], P[1, k])[2] for k in range(W.size))
    assert abs(A - 1.0) < 1e-12


# ---------------------------------------------------------------- :102-117
def _vertex_major_soup(v0, v1, v2):
    # the test fills soup[vertex, :, 1] = xyz (test/runtests.jl:105-107); as a
    # (T, nv, 3) array that is soup_T[0, c, v] = vertex v coordinate c.
    s = np.zeros((1, 3, 3))
    for v, p in enumerate((v0, v1, v2)):
        for c in range(3):
            s[0, c, v] = p[c]
    return s


def test_bvh_ray_casting(orc):
    bvh = orc.BVH(_vertex_major_soup([0, 0, 1], [1, 0, 1], [0, 1, 1]))
    d = np.array([0.0, 0.0, 1.0])
    assert bvh.intersect_ray_cpu([0.25, 0.25, 0.0], d, 2.0)
    assert not bvh.intersect_ray_cpu([2.0, 2.0, 0.0], d, 2.0)
    g = np.array([1], dtype=np.int32)
    assert bvh.intersect_flat(g, [0.25, 0.25, 0.0], d, 2.0)
    assert not bvh.intersect_flat(g, [2.0, 2.0, 0.0], d, 2.0)


# ---------------------------------------------------------------- :120-134
def test_visibility(orc):
    bvh = orc.BVH(_vertex_major_soup([-1, -1, 1], [1, -1, 1], [0, 1, 1]))
    xi = np.array([0.0, 0.0, 0.0])
    assert not bvh.is_visible_cpu(xi, [0.0, 0.0, 2.0])
    assert bvh.is_visible_cpu(xi, [5.0, 0.0, 2.0])


# ---------------------------------------------------------------- :137-153
def test_vf_kernel(orc):
    xi, ni = [0.0, 0.0, 0.0], [0.0, 0.0, 1.0]
    xj, nj = [0.0, 0.0, 1.0], [0.0, 0.0, -1.0]
    assert abs(orc.vf_kernel(xi, ni, xj, nj) - 1 / math.pi) < 1e-14
    assert orc.vf_kernel(xi, ni, xj, ni) == 0.0
    assert orc.vf_kernel(xi, ni, xi, nj) == 0.0


# ---------------------------------------------------------------- :160-198
PLATE_COORDS8 = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [.5, 0, 0], [1, .5, 0], [.5, 1, 0], [0, .5, 0],
                          [1, 0, 1], [0, 0, 1], [0, 1, 1], [1, 1, 1], [.5, 0, 1], [0, .5, 1], [.5, 1, 1],
                          [1, .5, 1]], dtype=float).T


def test_parallel_plates_quad8(orc):
    bot = ((1, 2, 3, 4, 5, 6, 7, 8), 1, "quad")
    top = ((9, 10, 11, 12, 13, 14, 15, 16), 2, "quad")
    m_ij = orc.Mesh(_mesh(PLATE_COORDS8, [bot, top]))
    m_ji = orc.Mesh(_mesh(PLATE_COORDS8, [top, bot]))
    raw_ij, a_ij, _, _ = orc.solve_plain(m_ij, 4)
    raw_ji, a_ji, _, _ = orc.solve_plain(m_ji, 4)
    assert abs(a_ij[0] - 1.0) < 1e-10 and abs(a_ji[0] - 1.0) < 1e-10
    assert raw_ij[0, 1] > 0
    assert abs(raw_ij[0, 1] - raw_ji[0, 1]) < 1e-12
    assert 0.1 < raw_ij[0, 1] / a_ij[0] < 1.0
    # the CPU-path restatement agrees (src/ViewFactorKernel.jl:199-241)
    raw_c, a_c, _ = orc.solve_cpu(m_ij, 4)
    assert abs(raw_c[0, 1] - raw_ij[0, 1]) < 1e-15 and abs(a_c[0] - a_ij[0]) < 1e-15


# ---------------------------------------------------------------- :201-224
def test_reciprocity_and_closure(rvf):
    r = rvf.ViewFactorResult(np.array([[0., 1.], [1., 0.]]), np.array([1., 1.]), np.array([[0., 1.], [1., 0.]]),
                             np.array([1., 1.]), [1, 2], ["surface1", "surface2"])
    assert rvf.check_reciprocity(r)
    assert rvf.check_closure(r)
    r2 = rvf.ViewFactorResult(np.array([[0., .5], [1., 0.]]), np.array([2., 1.]), np.array([[0., .5], [1., 0.]]),
                              np.array([2., 1.]), [1, 2], ["surface1", "surface2"])
    assert rvf.check_reciprocity(r2)


def test_reciprocity_oracle_matches_host(rvf, orc):
    rng = np.random.default_rng(0)
    F = rng.uniform(0, 0.1, (40, 40))
    A = rng.uniform(0.5, 2.0, 40)
    r = rvf.ViewFactorResult(F, A, np.zeros((1, 1)), np.zeros(1), [1], ["a"])
    assert abs(rvf.reciprocity_error(r) - orc.reciprocity_error(F, A)) < 1e-12


# ---------------------------------------------------------------- :227-255
def test_linear_shapes(orc):
    for xi, eta in [(-0.3, 0.7), (0.0, 0.0), (1.0, -1.0), (0.5, 0.5)]:
        assert abs(orc.shape("quad4", xi, eta)[0].sum() - 1.0) < 1e-14
    for b, (xi, eta) in enumerate([(-1., -1.), (1., -1.), (1., 1.), (-1., 1.)]):
        N = orc.shape("quad4", xi, eta)[0]
        for a in range(4):
            assert abs(N[a] - (1.0 if a == b else 0.0)) < 1e-14
    for xi in (-0.4, 0.0, 0.8):
        assert abs(orc.shape("line2", xi)[0].sum() - 1.0) < 1e-14
    assert abs(orc.shape("line2", -1.0)[0][0] - 1.0) < 1e-14
    assert abs(orc.shape("line2", 1.0)[0][1] - 1.0) < 1e-14
    for xi, eta in [(0.2, 0.3), (0.0, 0.0), (1.0, 0.0), (0.0, 1.0)]:
        assert abs(orc.shape("tri3", xi, eta)[0].sum() - 1.0) < 1e-14


# ---------------------------------------------------------------- :258-275
def test_dunavant_normalisation(orc):
    for n in range(1, 9):
        _, w = orc.tri_rule(n)
        assert abs(w.sum() - 0.5) < 1e-6
    P, W = orc.tri_rule(4)
    approx = float(np.sum(W * P[0] ** 3 * P[1] ** 4))
    assert abs(approx - 1 / 2520) < 1e-10


# ---------------------------------------------------------------- :278-300
PLATE_COORDS4 = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [1, 0, 1], [0, 0, 1], [0, 1, 1], [1, 1, 1]],
                         dtype=float).T


def test_linear_and_cross_order(orc):
    m4 = orc.Mesh(_mesh(PLATE_COORDS4, [((1, 2, 3, 4), 1, "quad4"), ((5, 6, 7, 8), 2, "quad4")]))
    raw4, a4, _, _ = orc.solve_plain(m4, 8)
    assert abs(a4[0] - 1.0) < 1e-10
    F4 = raw4[0, 1] / a4[0]
    assert abs(F4 - ANALYTIC_PLATES) < 2e-4
    c8 = np.zeros((3, 16))
    c8[:, 0:4] = PLATE_COORDS4[:, 0:4]
    c8[:, 4:8] = np.array([[.5, 0, 0], [1, .5, 0], [.5, 1, 0], [0, .5, 0]]).T
    c8[:, 8:12] = PLATE_COORDS4[:, 4:8]
    c8[:, 12:16] = np.array([[.5, 0, 1], [0, .5, 1], [.5, 1, 1], [1, .5, 1]]).T
    m8 = orc.Mesh(_mesh(c8, [((1, 2, 3, 4, 5, 6, 7, 8), 1, "quad"), ((9, 10, 11, 12, 13, 14, 15, 16), 2, "quad")]))
    raw8, a8, _, _ = orc.solve_plain(m8, 8)
    assert abs(raw8[0, 1] / a8[0] - F4) < 1e-6


# ---------------------------------------------------------------- :361-417
@pytest.mark.parametrize("family", ["tri3", "tri"])
def test_triangle_plates_end_to_end(rvf, orc, family):
    # Gmsh's unstructured h=0.2 triangulation is restated as a structured 5x5
    # triangulation of the same plates (Gmsh is not part of this backend).
    md = rvf.meshes.parallel_plates(5, family)
    m = orc.Mesh(md)
    raw, area, _ = orc.solve_cpu(m, 4)
    F = orc.f_from_raw(raw, area)
    Fg, Ag = orc.aggregate(F, area, md.elem_group, sorted(md.group_tags))
    assert abs(Fg[0, 1] - ANALYTIC_PLATES) < 5e-3
    assert orc.reciprocity_error(F, area) < 1e-4


# ---------------------------------------------------------------- :420-436
def test_gpu_kernel_semantics_linear_families(orc):
    m = orc.Mesh(_mesh(PLATE_COORDS4, [((1, 2, 3, 4), 1, "quad4"), ((5, 6, 7, 8), 2, "quad4")]))
    raw, area, _, _ = orc.solve_plain(m, 6)
    assert abs(area[0] - 1.0) < 1e-9
    assert abs(raw[0, 1] / area[0] - ANALYTIC_PLATES) < 2e-4


@pytest.mark.parametrize("geometric", [False, True])
def test_oracle_rows_equal_full_solve(rvf, orc, geometric):
    """orc_solve_rows (the row sample the full-size parity checks use) equals
    the full solve's rows bit for bit, for pairs below and above the row."""
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    m = orc.Mesh(md, [7])
    raw, area, _, _ = orc.solve_plain(m, 3, geometric=geometric)
    rows = [0, 5, 77, 200, md.n_elems - 1]
    out, area2, _ = orc.solve_rows(m, 3, rows, geometric=geometric)
    assert np.array_equal(area, area2)
    for r, i in enumerate(rows):
        assert np.array_equal(out[r], raw[i]), i
