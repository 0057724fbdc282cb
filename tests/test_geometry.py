"""The element geometry the reference exports (src/Geometry.jl): its own
known answers (test/runtests.jl:81-99, 225-250) and agreement with the
oracle's element evaluation on curved meshes of every family."""
import numpy as np
import pytest


def test_quad8_known_answers(rvf):
    """test/runtests.jl:81-99: unit square Quad8."""
    coords = np.array([[0.0, 1.0, 1.0, 0.0, 0.5, 1.0, 0.5, 0.0],
                       [0.0, 0.0, 1.0, 1.0, 0.0, 0.5, 1.0, 0.5],
                       [0.0] * 8])
    nodes = [1, 2, 3, 4, 5, 6, 7, 8]
    assert np.allclose(rvf.quad8_physical_point(coords, nodes, 0.0, 0.0), [0.5, 0.5, 0.0], atol=1e-14)
    n, dA = rvf.quad8_normal_and_area_element(coords, nodes, 0.0, 0.0)
    assert np.allclose(n, [0.0, 0.0, 1.0], atol=1e-14) and abs(dA - 0.25) <= 1e-14
    for nq in (2, 3, 4, 6):
        assert abs(rvf.element_area(coords, nodes, nquad=nq) - 1.0) <= 1e-12


def test_shape_functions_partition_of_unity(rvf):
    """test/runtests.jl:225-250 and the nodal interpolation property."""
    from rvf_b200 import geometry as g
    for xi, eta in [(-0.3, 0.7), (0.0, 0.0), (1.0, -1.0), (0.5, 0.5)]:
        assert abs(g.quad4_shape(xi, eta)[0].sum() - 1.0) <= 1e-14
        assert abs(g.quad8_shape(xi, eta)[0].sum() - 1.0) <= 1e-14
    corners = [(-1.0, -1.0), (1.0, -1.0), (1.0, 1.0), (-1.0, 1.0), (0.0, -1.0), (1.0, 0.0), (0.0, 1.0), (-1.0, 0.0)]
    for b, (xi, eta) in enumerate(corners):
        assert np.allclose(g.quad8_shape(xi, eta)[0], np.eye(8)[b], atol=1e-14)
        if b < 4:
            assert np.allclose(g.quad4_shape(xi, eta)[0], np.eye(4)[b], atol=1e-14)
    for xi in (-0.4, 0.0, 0.8):
        assert abs(g.line2_shape(xi)[0].sum() - 1.0) <= 1e-14
        assert abs(g.line3_shape(xi)[0].sum() - 1.0) <= 1e-14
    assert np.allclose(g.line3_shape(-1.0)[0], [1, 0, 0]) and np.allclose(g.line3_shape(0.0)[0], [0, 0, 1])


@pytest.mark.parametrize("kind", ["quad", "quad4", "line3", "line2"])
def test_geometry_matches_oracle(rvf, orc, kind):
    if kind in ("quad", "quad4"):
        md = rvf.meshes.cylinder(nc=8, na=3, cap_rings=2, jitter=0.01, seed=3) if kind == "quad" else \
            rvf.meshes.cube_enclosure(3, family="quad4", jitter=0.2, seed=1, box=False)
        point, normal = ((rvf.quad8_physical_point, rvf.quad8_normal_and_area_element) if kind == "quad" else
                         (rvf.quad4_physical_point, rvf.quad4_normal_and_area_element))
        k = 8 if kind == "quad" else 4
    else:
        md = rvf.meshes.cavity_2d(n_wall=4, n_circle=6, n_circles=1, seed=4)
        if kind == "line2":  # the same curves with their mid nodes dropped
            md = rvf.MeshData(md.coords, np.where(np.arange(8) < 2, md.elem_nodes, 0).astype(np.int32),
                              np.full(md.n_elems, rvf.FAMILY_CODES["line2"], dtype=np.int8), md.elem_group,
                              dict(md.group_tags), {}, 1)
        point, normal = ((rvf.line3_physical_point, rvf.line3_normal_and_length_element) if kind == "line3" else
                         (rvf.line2_physical_point, rvf.line2_normal_and_length_element))
        k = 3 if kind == "line3" else 2
    m = orc.Mesh(md)
    rng = np.random.default_rng(0)
    for e in range(0, md.n_elems, max(1, md.n_elems // 12)):
        nodes = md.elem_nodes[e, :k]
        xi, eta = rng.uniform(-1, 1, size=2)
        if kind.startswith("line"):
            x, (n, d) = point(md.coords, nodes, xi), normal(md.coords, nodes, xi)
            xo, no, do = orc.eval_point(m, e, xi)
        else:
            x, (n, d) = point(md.coords, nodes, xi, eta), normal(md.coords, nodes, xi, eta)
            xo, no, do = orc.eval_point(m, e, xi, eta)
        assert np.allclose(x, xo, rtol=0, atol=1e-13)
        assert np.allclose(n, no, rtol=0, atol=1e-13)
        assert abs(d - do) <= 1e-13 * abs(do)
