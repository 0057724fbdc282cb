"""Stratified Monte Carlo path (src/GPUMCKernels.jl) on the device vs the oracle.

Every pair draws the reference's own xorshift64 stream, so the device result
is not a statistical match but an exact one: element areas, view factors and
every per-sample shadow-ray decision (logged as 0 = no ray, 1 = visible,
2 = blocked) equal the oracle's bit for bit.
"""
import numpy as np
import pytest

from conftest import load_pkg
from test_gpu_parity import concat

pytestmark = pytest.mark.gpu


def device_mc(rvf, session, md, n_samples, seed, obstruction_groups=(), exclude=False, geometric=False, log=False):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obstruction_groups))
    try:
        N = md.n_elems
        o = rvf.make_options(4, monte_carlo=True, n_samples=n_samples, seed=seed, geometric_soup=geometric,
                             mc_exclude_groups=exclude)
        lg = None
        if log:
            lg = np.zeros(N * N * n_samples, dtype=np.uint8)
            o.ray_log = lg.ctypes.data_as(_abi._pu8)
            o.ray_log_pm = 1
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        st = dm.solve(o, F, A)
        return F, A, lg, st
    finally:
        dm.release()


def oracle_mc(orc, md, n_samples, seed, obstruction_groups=(), exclude=False, geometric=False, log=False):
    m = orc.Mesh(md, obstruction_groups)
    raw, area, lg, cnt = orc.solve_mc(m, n_samples, seed, exclude_groups=exclude, geometric=geometric, ray_log=log)
    return orc.f_from_raw(raw, area), area, lg, cnt


def assert_same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{int((~same).sum())} entries differ, max |d| {np.nanmax(np.abs(a - b))}"


@pytest.mark.parametrize("exclude", [False, True])
@pytest.mark.parametrize("geometric", [False, True])
def test_mc_cube_with_box_exact(rvf, orc, session, exclude, geometric):
    md = rvf.meshes.cube_enclosure(4, family="quad4", box_m=2)
    F, A, lg, st = device_mc(rvf, session, md, 16, 1234, [7], exclude, geometric, log=True)
    Fo, Ao, lgo, cnt = oracle_mc(orc, md, 16, 1234, [7], exclude, geometric, log=True)
    assert np.array_equal(A, Ao)
    assert (lgo == 2).sum() > 0, "the box must block some rays"
    assert np.array_equal(lg, lgo), f"{int((lg != lgo).sum())} ray decisions differ"
    assert_same(F, Fo)
    assert st.n_rays == cnt[1] == int((lgo > 0).sum())
    N = md.n_elems
    assert st.n_point_pairs == 16 * N * (N - 1) // 2


@pytest.mark.parametrize("family,n_samples", [("tri3", 10), ("tri", 7), ("quad", 9), ("quad4", 1)])
def test_mc_families_remainder_samples(rvf, orc, session, family, n_samples):
    """n_samples not a square: floor(sqrt(n))^2 strata plus uniform remainder."""
    md = rvf.meshes.cube_enclosure(3, family=family, box_m=2, box_edge=0.5)
    F, A, lg, _ = device_mc(rvf, session, md, n_samples, 77, [7], log=True)
    Fo, Ao, lgo, _ = oracle_mc(orc, md, n_samples, 77, [7], log=True)
    assert np.array_equal(A, Ao)
    assert np.array_equal(lg, lgo)
    assert_same(F, Fo)


def test_mc_mixed_families_no_occlusion(rvf, orc, session):
    md = concat(rvf.meshes.parallel_plates(3, "quad"), rvf.meshes.cube_enclosure(2, family="tri", box=False))
    F, A, _, st = device_mc(rvf, session, md, 25, 5)
    Fo, Ao, _, _ = oracle_mc(orc, md, 25, 5)
    assert np.array_equal(A, Ao)
    assert_same(F, Fo)
    assert st.n_rays == 0


def test_mc_curves_2d(rvf, orc, session):
    md = rvf.meshes.cavity_2d(n_wall=24, n_circle=16, n_circles=2, seed=4)
    F, A, lg, _ = device_mc(rvf, session, md, 9, 42, [5, 6], log=True)
    Fo, Ao, lgo, _ = oracle_mc(orc, md, 9, 42, [5, 6], log=True)
    assert np.array_equal(A, Ao)
    assert (lgo == 2).sum() > 0
    assert np.array_equal(lg, lgo)
    assert_same(F, Fo)


def test_mc_ragged_tiles(rvf, orc, session):
    """N not a multiple of the 32-element tile; seeds above 2^63."""
    md = rvf.meshes.cube_enclosure(3, family="tri3", box_m=1)  # 108 triangles
    seed = 2**64 - 12345
    F, A, lg, _ = device_mc(rvf, session, md, 4, seed, [7], log=True)
    Fo, Ao, lgo, _ = oracle_mc(orc, md, 4, seed, [7], log=True)
    assert np.array_equal(A, Ao)
    assert np.array_equal(lg, lgo)
    assert_same(F, Fo)


def test_mc_single_element(rvf, orc, session):
    md = rvf.meshes.parallel_plates(1, "quad4")
    md.elem_nodes = md.elem_nodes[:1]
    md.elem_family = md.elem_family[:1]
    md.elem_group = md.elem_group[:1]
    F, A, _, _ = device_mc(rvf, session, md, 4, 1)
    assert A[0] == 0.0 and np.isnan(F[0, 0])


def test_mc_converges_to_plates_factor(rvf, session):
    """Unit plates at unit gap: the MC group factor approaches 0.19982."""
    md = rvf.meshes.parallel_plates(4, "quad4")
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, ()))
    try:
        Fg = np.empty((2, 2), order="F")
        Ag = np.empty(2)
        dm.solve(rvf.make_options(4, monte_carlo=True, n_samples=4096, seed=3), None, None, Fg, Ag)
    finally:
        dm.release()
    assert abs(Fg[0, 1] - 0.19982) < 2e-3
    assert abs(Ag[0] - 1.0) < 1e-12


def test_mc_public_api(rvf, orc):
    md = rvf.meshes.cube_enclosure(3, family="quad4", box_m=2)
    res = rvf.compute_view_factors(md, backend=rvf.B200Backend(), monte_carlo=True, n_samples=16, seed=99,
                                   obstruction_groups=[7], verbose=False)
    Fo, Ao, _, _ = oracle_mc(orc, md, 16, 99, [7])
    assert_same(res.F_elem, Fo)
    assert np.array_equal(res.A_elem, Ao)


def _mc_solve(rvf, session, md, obs, n_samples, seed, exclude, cull):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
    try:
        N = md.n_elems
        o = rvf.make_options(4, monte_carlo=True, n_samples=n_samples, seed=seed, mc_exclude_groups=exclude)
        o.disable_tile_cull = 0 if cull else 1
        lg = np.zeros(N * N * n_samples, dtype=np.uint8)
        o.ray_log = lg.ctypes.data_as(_abi._pu8)
        o.ray_log_pm = 1
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        st = dm.solve(o, F, A).as_dict()
        return F, A, lg, st
    finally:
        dm.release()


def _box_cylinder(rvf):
    """Curved Quad8 walls and caps around a box: sample points bulge past the
    elements' node hulls, which the classification's radii must cover."""
    M = rvf.meshes
    md = M.cylinder(nc=16, na=8, cap_rings=2, seed=3)
    md.group_tri_soup[99] = M.obstruction_box(center=(0.0, 0.0, 0.5), edge=0.3, m=4)
    return md, [99]


@pytest.mark.parametrize("case", ["quad8_cube", "tri6_cube", "quad8_cylinder"])
@pytest.mark.parametrize("exclude", [False, True])
def test_mc_tile_masks_exact(rvf, orc, session, case, exclude):
    """Surface Monte Carlo with occlusion skips the traversal of pairs outside
    the tile classification's masks; every sample ray's decision, and so F,
    stays the oracle's bit for bit, and equal to the unclassified solve."""
    M = rvf.meshes
    if case == "quad8_cube":
        md, obs = M.cube_enclosure(16, family="quad", box_m=4), [7]
    elif case == "tri6_cube":
        md, obs = M.cube_enclosure(6, family="tri", box_m=4), [7]
    else:
        md, obs = _box_cylinder(rvf)
    F, A, lg, st = _mc_solve(rvf, session, md, obs, 8, 4321, exclude, True)
    F0, A0, lg0, st0 = _mc_solve(rvf, session, md, obs, 8, 4321, exclude, False)
    assert st["n_tiles_culled"] > 0 and st0["n_tiles_culled"] == 0
    assert st["n_rays"] == st0["n_rays"]
    assert st["n_node_visits"] < st0["n_node_visits"]
    assert np.array_equal(lg, lg0), f"{int((lg != lg0).sum())} ray decisions differ"
    assert_same(F, F0)
    Fo, Ao, lgo, _ = oracle_mc(orc, md, 8, 4321, obs, exclude, log=True)
    assert (lgo == 2).sum() > 0, "the box must block some rays"
    assert np.array_equal(lg, lgo), f"{int((lg != lgo).sum())} ray decisions differ from the oracle"
    assert np.array_equal(A, Ao)
    assert_same(F, Fo)
