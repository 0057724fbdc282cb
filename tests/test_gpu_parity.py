"""Parity of the CUDA path (called through the C ABI) with the oracle.

Tolerances (FP64 plain path): every element view factor within 1e-10
relative of the oracle (|dF| <= 1e-10 |F_oracle| + 1e-300), areas bit for bit,
and every shadow-ray decision identical (the per point-pair ray logs are
compared byte for byte).
"""
import numpy as np
import pytest

from conftest import load_pkg

pytestmark = pytest.mark.gpu

RTOL = 1e-10
ATOL = 1e-300


def assert_rel(a, b, rtol=RTOL, atol=ATOL):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    nan = np.isnan(a) & np.isnan(b)
    bad = ~((np.abs(a - b) <= rtol * np.abs(b) + atol) | nan)
    if bad.any():
        idx = np.argwhere(bad)[:5]
        msg = ", ".join(f"{tuple(i)}: {a[tuple(i)]!r} vs {b[tuple(i)]!r}" for i in idx)
        raise AssertionError(f"{int(bad.sum())} entries outside rtol={rtol}: {msg}")


def concat(*meshes):
    """Concatenate meshes (renumbering nodes) -- mixed-family test meshes."""
    rvf = load_pkg()
    coords, en, fam, grp, tags, soups, off = [], [], [], [], {}, {}, 0
    for m in meshes:
        coords.append(m.coords)
        e = m.elem_nodes.copy()
        e[e > 0] += off
        en.append(e)
        fam.append(m.elem_family)
        grp.append(m.elem_group)
        tags.update(m.group_tags)
        soups.update(m.group_tri_soup)
        off += m.coords.shape[1]
    return rvf.MeshData(np.hstack(coords), np.vstack(en), np.concatenate(fam), np.concatenate(grp), tags, soups,
                        meshes[0].mesh_dim)


def device_solve(rvf, session, md, nquad, obstruction_groups=(), geometric=False, log_pm=None, lists=True):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obstruction_groups))
    try:
        N = md.n_elems
        G = len(md.group_tags)
        o = rvf.make_options(nquad, geometric_soup=geometric, seed=0)
        o.disable_pair_lists = 0 if lists else 1
        log = None
        if log_pm:
            log = np.zeros(N * N * log_pm * log_pm, dtype=np.uint8)
            o.ray_log = log.ctypes.data_as(_abi._pu8)
            o.ray_log_pm = log_pm
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        Fg = np.empty((G, G), order="F")
        Ag = np.empty(G)
        rs = np.empty(N)
        st = dm.solve(o, F, A, Fg, Ag, rs)
        return F, A, Fg, Ag, rs, log, st
    finally:
        dm.release()


def oracle_solve(orc, md, nquad, obstruction_groups=(), geometric=False, log_pm=None):
    m = orc.Mesh(md, obstruction_groups)
    raw, area, log, cnt = orc.solve_plain(m, nquad, geometric=geometric, ray_log_pm=log_pm)
    F = orc.f_from_raw(raw, area)
    Fg, Ag = orc.aggregate(F, area, md.elem_group, sorted(md.group_tags))
    return F, area, Fg, Ag, log, cnt


def test_parallel_plates_config(rvf, orc, session):
    """20 x 20 Quad4 plates, nquad=4 (the CPU-runnable configuration)."""
    md = rvf.meshes.parallel_plates(20, "quad4")
    F, A, Fg, Ag, rs, _, st = device_solve(rvf, session, md, 4)
    Fo, Ao, Fgo, Ago, _, _ = oracle_solve(orc, md, 4)
    assert np.array_equal(A, Ao)
    assert_rel(F, Fo)
    assert_rel(Fg, Fgo, rtol=1e-12)
    assert abs(Fg[0, 1] - 0.19982) < 2e-4
    assert_rel(rs, Fo.sum(axis=1), rtol=1e-12)
    assert st.n_pairs == 800 * 799 // 2


@pytest.mark.parametrize("lists", [True, False])
@pytest.mark.parametrize("geometric", [False, True])
def test_cube_with_obstruction_rays_identical(rvf, orc, session, geometric, lists):
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    F, A, Fg, Ag, rs, log, st = device_solve(rvf, session, md, 3, [7], geometric, log_pm=7, lists=lists)
    Fo, Ao, Fgo, Ago, logo, cnt = oracle_solve(orc, md, 3, [7], geometric, log_pm=7)
    assert np.array_equal(A, Ao)
    assert int((logo > 0).sum()) == st.n_rays == cnt[1]
    assert (logo == 2).sum() > 0, "the box must block some rays"
    assert np.array_equal(log, logo), f"{int((log != logo).sum())} ray decisions differ"
    assert_rel(F, Fo)
    assert_rel(Fg, Fgo, rtol=1e-12)


@pytest.mark.parametrize("lists", [True, False])
def test_surface_groups_as_obstructions(rvf, orc, session, lists):
    """Faces that are both surfaces and obstructions: each ray skips the
    triangles of its own two groups (src/GPUBVH.jl:239-240), in the pair
    lists as in the walk; ray decisions identical to the oracle's."""
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    obs = [2, 5, 7]
    F, A, Fg, Ag, rs, log, st = device_solve(rvf, session, md, 3, obs, log_pm=7, lists=lists)
    Fo, Ao, Fgo, Ago, logo, cnt = oracle_solve(orc, md, 3, obs, log_pm=7)
    assert (logo == 2).sum() > 0
    assert np.array_equal(log, logo), f"{int((log != logo).sum())} ray decisions differ"
    assert_rel(F, Fo)


def test_pair_lists_fine_cube(rvf, orc, session):
    """Elements much smaller than the obstruction's leaves (the headline
    shape at 20 x 20 per face): pending pairs test a short per-pair triangle
    list instead of walking the tree.  Every row the oracle computes (one in
    23) agrees to 1e-10, and with the lists disabled (every ray walks the
    tree) F is bit for bit the same."""
    md = rvf.meshes.cube_enclosure(20, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12)
    N = md.n_elems
    F, A, Fg, Ag, rs, _, st = device_solve(rvf, session, md, 3, [7])
    d = st.as_dict()
    assert d["n_list_pairs"] > 100 * d["n_walk_pairs"], d
    Fw, Aw, *_, stw = device_solve(rvf, session, md, 3, [7], lists=False)
    assert stw.as_dict()["n_list_pairs"] == 0 and stw.as_dict()["n_walk_pairs"] == d["n_list_pairs"] + d["n_walk_pairs"]
    assert np.array_equal(F, Fw, equal_nan=True)
    m = orc.Mesh(md, [7])
    raw, area, _, _ = orc.solve_plain(m, 3, row_stride=23)
    assert np.array_equal(A, area)
    rows = np.arange(0, N, 23)
    for i in rows:
        Fo = raw[i, i + 1:] / area[i]
        assert_rel(F[i, i + 1:], Fo)


@pytest.mark.parametrize("family,nquad", [("quad4", 2), ("quad", 3), ("tri", 4), ("tri3", 1), ("quad", 2)])
def test_families_with_obstruction(rvf, orc, session, family, nquad):
    md = rvf.meshes.cube_enclosure(3, family=family, box_m=2, box_edge=0.5)
    pm = {1: 3, 2: 9, 3: 9, 4: 16}[nquad] if family in ("quad", "quad4") else 13
    F, A, *_, log, st = device_solve(rvf, session, md, nquad, [7], log_pm=pm)
    Fo, Ao, *_, logo, cnt = oracle_solve(orc, md, nquad, [7], log_pm=pm)
    assert np.array_equal(A, Ao)
    assert np.array_equal(log, logo)
    assert_rel(F, Fo)


def test_mixed_families(rvf, orc, session):
    md = concat(rvf.meshes.parallel_plates(3, "quad"), rvf.meshes.cube_enclosure(2, family="tri", box=False))
    md.group_tags = {**md.group_tags}
    for nq in (2, 3, 4):
        F, A, *_ = device_solve(rvf, session, md, nq)
        Fo, Ao, *_ = oracle_solve(orc, md, nq)
        assert np.array_equal(A, Ao)
        assert_rel(F, Fo)


@pytest.mark.parametrize("nquad", [1, 2, 3, 4, 5, 6, 8])
def test_nquad_sweep(rvf, orc, session, nquad):
    md = rvf.meshes.parallel_plates(4, "quad4")
    F, A, *_ = device_solve(rvf, session, md, nquad)
    Fo, Ao, *_ = oracle_solve(orc, md, nquad)
    assert np.array_equal(A, Ao)
    assert_rel(F, Fo)


def test_curve_mesh_with_obstruction(rvf, orc, session):
    md = rvf.meshes.cavity_2d(n_wall=24, n_circle=16, n_circles=2, seed=4)
    F, A, *_, log, st = device_solve(rvf, session, md, 3, [5, 6], log_pm=3)
    Fo, Ao, *_, logo, cnt = oracle_solve(orc, md, 3, [5, 6], log_pm=3)
    assert np.array_equal(A, Ao)
    assert (logo == 2).sum() > 0
    assert np.array_equal(log, logo)
    assert_rel(F, Fo)


@pytest.mark.parametrize("n_side", [1, 2, 3, 5])
def test_ragged_sizes(rvf, orc, session, n_side):
    # N = 2, 8, 18, 50 elements: tiles partially filled, diagonal tiles
    md = rvf.meshes.parallel_plates(n_side, "tri3")
    F, A, *_ = device_solve(rvf, session, md, 2)
    Fo, Ao, *_ = oracle_solve(orc, md, 2)
    assert_rel(F, Fo)
    assert np.array_equal(A, Ao)


def test_single_element(rvf, session):
    """N = 1: no pair writes the area, so A = 0 and F = 0/0 as in the reference."""
    md = rvf.MeshData(np.array([[0., 1., 0.], [0., 0., 1.], [0., 0., 0.]]), np.array([[1, 2, 3, 0, 0, 0, 0, 0]]),
                      np.array([3]), np.array([1]), {1: "a"})
    F, A, *_ = device_solve(rvf, session, md, 2)
    assert A[0] == 0.0 and np.isnan(F[0, 0])


def test_deterministic(rvf, session):
    md = rvf.meshes.cube_enclosure(5, box_m=2)
    F1, *_ = device_solve(rvf, session, md, 3, [7])
    F2, *_ = device_solve(rvf, session, md, 3, [7])
    assert np.array_equal(F1, F2)


def test_invalid_mesh_is_rejected(rvf, session):
    md = rvf.meshes.parallel_plates(2, "quad4")
    md.elem_nodes[3, 2] = 10_000
    from rvf_b200 import _abi
    with pytest.raises(rvf.RVFError) as ei:
        _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, ()))
    assert ei.value.status == -1 and "node id" in str(ei.value)


def test_public_api_end_to_end(rvf, orc, session):
    md = rvf.meshes.cube_enclosure(5, box_m=2)
    r = rvf.compute_view_factors(md, nquad=3, obstruction_groups=[7], verbose=False)
    assert r.F_elem.shape == (md.n_elems, md.n_elems)
    assert rvf.check_reciprocity(r)
    # a 5x5-per-face cube under a 7-point rule over-integrates the pairs that
    # share a cube edge (row sums up to ~1.3): closure follows the oracle
    Fo, Ao, *_ = oracle_solve(orc, md, 3, [7])
    assert rvf.check_closure(r) == (Fo.sum(axis=1).max() <= 1.0 + 1e-3)
    assert_rel(r.F_elem.sum(axis=1), Fo.sum(axis=1), rtol=1e-12)
    Fg, Ag, tags, names = rvf.aggregate_by_group(r, md)
    assert_rel(Fg, r.F_group, rtol=1e-12)
    assert tags == [1, 2, 3, 4, 5, 6]
    plates = rvf.compute_view_factors(rvf.meshes.parallel_plates(6, "quad"), nquad=4, verbose=False)
    assert rvf.check_closure(plates) and rvf.check_reciprocity(plates)
