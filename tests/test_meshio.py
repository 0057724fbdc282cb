"""Mesh ingest (load_mesh on Gmsh .msh 4.1 / 2.2 ASCII files, src/MeshIO.jl:94-149).

tests/golden/plate_quad9.msh is written by hand in the format Gmsh writes
(corner nodes on point entities, edge nodes on curves, interior nodes on the
surface; point, Line3 and Quad9 element blocks); plate_quad9_v22.msh is the
same plate in the legacy 2.2 format.  The other files are written
by write_msh from the package's meshes or from Delaunay triangulations, which
stand in for Gmsh's unstructured meshing in the reference's own load_mesh
tests (test/runtests.jl:303-420: families by order, total plate area 1, the
synthetic "default" group, F(bottom -> top) = 0.19982 within 5e-3).
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
PLATE = GOLDEN / "plate_quad9.msh"


def areas(orc, md, nquad=4):
    return orc.self_gpu(orc.Mesh(md), nquad)[1]


def delaunay_plates(rvf, order=1, h=0.2, seed=0):
    """Two unit squares 1 apart (bottom z=0 normal +z, group 1; top z=1 normal
    -z, group 2), each an unstructured Delaunay triangulation of jittered
    points; order 2 adds shared mid-edge nodes (Tri6)."""
    from scipy.spatial import Delaunay
    rng = np.random.default_rng(seed)
    n = int(round(1 / h))
    g = np.linspace(0.0, 1.0, n + 1)
    P = np.array([(x, y) for y in g for x in g])
    inner = (P[:, 0] > 0) & (P[:, 0] < 1) & (P[:, 1] > 0) & (P[:, 1] < 1)
    P[inner] += rng.uniform(-0.3 * h, 0.3 * h, size=(int(inner.sum()), 2))
    T = Delaunay(P).simplices
    coords, elems, groups = [], [], []
    for grp, z in ((1, 0.0), (2, 1.0)):
        base = len(coords)
        coords += [(x, y, z) for x, y in P]
        mids = {}
        for t in T:
            a, b, c = (int(v) for v in t)
            s = (P[b, 0] - P[a, 0]) * (P[c, 1] - P[a, 1]) - (P[b, 1] - P[a, 1]) * (P[c, 0] - P[a, 0])
            if (s > 0) != (grp == 1):  # bottom counter-clockwise (+z), top clockwise (-z)
                b, c = c, b
            el = [base + a + 1, base + b + 1, base + c + 1]
            if order == 2:
                for u, v in ((a, b), (b, c), (c, a)):
                    key = (min(u, v), max(u, v))
                    if key not in mids:
                        coords.append(((P[u, 0] + P[v, 0]) / 2, (P[u, 1] + P[v, 1]) / 2, z))
                        mids[key] = len(coords)
                    el.append(mids[key])
            elems.append(el)
            groups.append(grp)
    en = np.zeros((len(elems), 8), dtype=np.int32)
    for e, el in enumerate(elems):
        en[e, :len(el)] = el
    fam = rvf.FAMILY_CODES["tri3" if order == 1 else "tri"]
    md = rvf.MeshData(np.asfortranarray(np.array(coords).T), en, np.full(len(elems), fam, dtype=np.int8),
                      np.array(groups, dtype=np.int32), {1: "bottom", 2: "top"}, {}, 2)
    md.group_tri_soup = rvf.build_group_obs_soups(md)
    return md


def element_geometry(md):
    """Coordinates of every element's nodes (independent of node numbering)."""
    out = []
    for e in range(md.n_elems):
        k = int(np.count_nonzero(md.elem_nodes[e]))
        out.append(md.coords[:, md.elem_nodes[e, :k] - 1].T.copy())
    return out


def test_golden_plate_quad9(rvf, orc):
    md = rvf.load_mesh(str(PLATE), verbose=False)
    assert md.group_tags == {1: "plate"} and md.mesh_dim == 2
    assert list(md.elem_family) == [rvf.FAMILY_CODES["quad"]] * 2
    assert md.elem_nodes.tolist() == [[1, 6, 10, 4, 5, 14, 11, 12], [6, 2, 3, 10, 7, 8, 9, 14]]
    assert np.array_equal(md.coords[:, 12], [0.25, 0.5, 0.0])  # node 13 (surface), dropped from the Quad9
    A = areas(orc, md)
    assert np.allclose(A, 0.5, atol=1e-12) and abs(A.sum() - 1.0) < 1e-12
    assert set(md.group_tri_soup) == {1} and md.group_tri_soup[1].shape == (4, 3, 3)


def test_golden_plate_curves_default_group(rvf):
    md = rvf.load_mesh(str(PLATE), surface_dim=1, verbose=False)
    # no physical curve group: one synthetic group with the next free tag
    assert md.group_tags == {2: "default"} and md.mesh_dim == 1
    assert md.elem_nodes[:, :3].tolist() == [[1, 6, 5], [6, 2, 7]]  # normals already point into the plate


def test_legacy_v22_matches_v41(rvf):
    """The same plate written in the .msh 2.2 format: same elements (by
    geometry), families, groups and curve orientation."""
    v22 = GOLDEN / "plate_quad9_v22.msh"
    for dim in (2, 1):
        a = rvf.load_mesh(str(PLATE), surface_dim=dim, verbose=False)
        b = rvf.load_mesh(str(v22), surface_dim=dim, verbose=False)
        assert a.group_tags == b.group_tags
        assert np.array_equal(a.elem_family, b.elem_family) and np.array_equal(a.elem_group, b.elem_group)
        for x, y in zip(element_geometry(a), element_geometry(b)):
            assert np.array_equal(x, y)


def test_legacy_v22_lines_turned_toward_the_surface(rvf, tmp_path):
    text = (GOLDEN / "plate_quad9_v22.msh").read_text().replace("2 8 2 0 1 1 6 5\n", "2 8 2 0 1 6 1 5\n")
    f = tmp_path / "reversed_v22.msh"
    f.write_text(text)
    md = rvf.load_mesh(str(f), surface_dim=1, verbose=False)
    ref = rvf.load_mesh(str(GOLDEN / "plate_quad9_v22.msh"), surface_dim=1, verbose=False)
    assert np.array_equal(md.elem_nodes, ref.elem_nodes)


def test_line_elements_turned_toward_the_surface(rvf, tmp_path, capsys):
    text = PLATE.read_text().replace("2 1 6 5\n3 6 2 7\n", "2 6 1 5\n3 2 6 7\n")
    f = tmp_path / "reversed.msh"
    f.write_text(text)
    md = rvf.load_mesh(str(f), surface_dim=1, verbose=True)
    assert md.elem_nodes[:, :3].tolist() == [[1, 6, 5], [6, 2, 7]]
    assert "Reoriented 2 Line3 element(s)" in capsys.readouterr().out


def test_parametric_node_block(rvf, tmp_path):
    """A 4.1 node block flagged parametric carries the curve parameter after
    x y z on each coordinate line; the reader keeps x y z."""
    text = PLATE.read_text().replace("1 1 0 3\n5\n6\n7\n0.25 0 0\n0.5 0 0\n0.75 0 0\n",
                                     "1 1 1 3\n5\n6\n7\n0.25 0 0 0.25\n0.5 0 0 0.5\n0.75 0 0 0.75\n")
    assert text != PLATE.read_text()
    f = tmp_path / "parametric.msh"
    f.write_text(text)
    a = rvf.load_mesh(str(PLATE), verbose=False)
    b = rvf.load_mesh(str(f), verbose=False)
    assert np.array_equal(a.coords, b.coords) and np.array_equal(a.elem_nodes, b.elem_nodes)


def test_reverse_normals_follows_the_reference(rvf):
    md = rvf.load_mesh(str(PLATE), reverse_normals=True, verbose=False)
    # Quad8: corners 1<->3 and mid-side nodes 5<->7, as src/MeshIO.jl:624-626 swaps them
    assert md.elem_nodes[0].tolist() == [10, 6, 1, 4, 11, 14, 5, 12]


def test_entity_in_two_groups_and_unnamed_group(rvf, tmp_path):
    text = PLATE.read_text().replace("1 0 0 0 1 1 0 1 1 4 1 2 3 4", "1 0 0 0 1 1 0 2 1 7 4 1 2 3 4")
    f = tmp_path / "two_groups.msh"
    f.write_text(text)
    md = rvf.load_mesh(str(f), verbose=False)
    assert md.group_tags == {1: "plate", 7: "group_7"}
    assert md.elem_group.tolist() == [1, 1, 7, 7]
    assert np.array_equal(md.elem_nodes[:2], md.elem_nodes[2:])


@pytest.mark.parametrize("family", ["tri3", "quad4", "tri", "quad"])
def test_round_trip(rvf, tmp_path, family):
    src = rvf.meshes.cube_enclosure(3, family=family, box_m=2)
    f = tmp_path / f"cube_{family}.msh"
    rvf.meshio.write_msh(str(f), src)
    md = rvf.load_mesh(str(f), verbose=False)
    assert md.group_tags == src.group_tags
    assert np.array_equal(md.elem_family, src.elem_family) and np.array_equal(md.elem_group, src.elem_group)
    for a, b in zip(element_geometry(md), element_geometry(src)):
        assert np.array_equal(a, b)
    for g in src.group_tags:
        assert np.array_equal(md.group_tri_soup[g], src.group_tri_soup[g])


def test_round_trip_curves(rvf, tmp_path):
    src = rvf.meshes.cavity_2d(n_wall=6, n_circle=8, n_circles=2, seed=4)
    f = tmp_path / "cavity.msh"
    rvf.meshio.write_msh(str(f), src)
    md = rvf.load_mesh(str(f), surface_dim=1, verbose=False)
    assert md.group_tags == src.group_tags and np.array_equal(md.elem_group, src.elem_group)
    for a, b in zip(element_geometry(md), element_geometry(src)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("order", [1, 2])
def test_unstructured_plates_area(rvf, orc, tmp_path, order):
    """test/runtests.jl:331-349: families by element order, total area 1."""
    f = tmp_path / f"plates{order}.msh"
    rvf.meshio.write_msh(str(f), delaunay_plates(rvf, order))
    md = rvf.load_mesh(str(f), verbose=False)
    fam = rvf.FAMILY_CODES["tri3" if order == 1 else "tri"]
    assert (md.elem_family == fam).all() and md.group_tags == {1: "bottom", 2: "top"}
    A = areas(orc, md)
    for g in (1, 2):
        assert abs(A[md.elem_group == g].sum() - 1.0) < 1e-9


def test_xml_vtk_is_routed_to_load_vtu(rvf, tmp_path):
    """src/MeshIO.jl:101-103 and 158-170: XML VTK goes to load_vtu, which
    needs ReadVTK in the reference and is not provided here."""
    f = tmp_path / "plate.vtu"
    f.write_text('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid"></VTKFile>\n')
    with pytest.raises(NotImplementedError, match="ReadVTK"):
        rvf.load_mesh(str(f))
    g = tmp_path / "xml.vtk"
    g.write_text('<VTKFile type="UnstructuredGrid"></VTKFile>\n')
    legacy = tmp_path / "legacy.vtk"
    legacy.write_text("# vtk DataFile Version 3.0\nmesh\nASCII\n")
    assert rvf.meshio.is_xml_vtk(str(g)) and not rvf.meshio.is_xml_vtk(str(PLATE))
    assert not rvf.meshio.is_xml_vtk(str(legacy))  # test/runtests.jl:453-456
    with pytest.raises(NotImplementedError):
        rvf.plot_mesh_normals(None)


def test_load_errors(rvf, tmp_path):
    with pytest.raises(FileNotFoundError):
        rvf.load_mesh(str(tmp_path / "missing.msh"))
    with pytest.raises(ValueError, match="surface_dim"):
        rvf.load_mesh(str(PLATE), surface_dim=3)
    old = tmp_path / "v30.msh"
    old.write_text("$MeshFormat\n3.0 0 8\n$EndMeshFormat\n")
    with pytest.raises(ValueError, match="not supported"):
        rvf.load_mesh(str(old))
    binary = tmp_path / "bin.msh"
    binary.write_text("$MeshFormat\n4.1 1 8\n$EndMeshFormat\n")
    with pytest.raises(ValueError, match="binary"):
        rvf.load_mesh(str(binary))
    # a physical surface group holding no supported element type
    text = PLATE.read_text().replace("2 1 10 2\n", "2 1 99 2\n")
    bad = tmp_path / "unsupported.msh"
    bad.write_text(text)
    with pytest.raises(ValueError, match="No supported elements"):
        rvf.load_mesh(str(bad), verbose=False)


@pytest.mark.gpu
@pytest.mark.parametrize("order", [1, 2])
def test_unstructured_plates_view_factor(rvf, tmp_path, order):
    """test/runtests.jl:357-420 on the device: F(bottom -> top) of two
    unstructured unit plates 1 apart within 5e-3 of 0.19982, reciprocity."""
    f = tmp_path / f"plates{order}.msh"
    rvf.meshio.write_msh(str(f), delaunay_plates(rvf, order))
    md = rvf.load_mesh(str(f), verbose=False)
    r = rvf.compute_view_factors(md, nquad=4, verbose=False)
    b, t = r.group_names.index("bottom"), r.group_names.index("top")
    assert abs(r.F_group[b, t] - 0.19982) < 5e-3
    assert rvf.check_reciprocity(r)
