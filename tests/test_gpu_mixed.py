"""Mixed-precision path (FP32 far field and traversal, FP64 where stability
needs it) against the oracle.

Tolerances: every element view factor within |dF| <= 1e-6 of the FP64
oracle, areas bit for bit, and every shadow-ray decision identical to the
reference's (ray logs compared byte for byte).
"""
import numpy as np
import pytest

from test_gpu_parity import concat, oracle_solve

pytestmark = pytest.mark.gpu

ATOL_MIXED = 1e-6


def mixed_solve(rvf, session, md, nquad, obstruction_groups=(), geometric=False, log_pm=None, near=2.0, lists=True):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obstruction_groups))
    try:
        N = md.n_elems
        o = rvf.make_options(nquad, precision="mixed", geometric_soup=geometric, seed=0)
        o.near_field_factor = near
        o.disable_pair_lists = 0 if lists else 1
        log = None
        if log_pm:
            log = np.zeros(N * N * log_pm * log_pm, dtype=np.uint8)
            o.ray_log = log.ctypes.data_as(_abi._pu8)
            o.ray_log_pm = log_pm
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        rs = np.empty(N)
        st = dm.solve(o, F, A, None, None, rs)
        return F, A, rs, log, st.as_dict()
    finally:
        dm.release()


@pytest.mark.parametrize("lists", [True, False])
@pytest.mark.parametrize("near", [2.0, 0.0, 1e9])
@pytest.mark.parametrize("geometric", [False, True])
def test_cube_mixed_rays_identical(rvf, orc, session, near, geometric, lists):
    md = rvf.meshes.cube_enclosure(8, box_m=4)
    F, A, rs, log, st = mixed_solve(rvf, session, md, 3, [7], geometric, log_pm=7, near=near, lists=lists)
    Fo, Ao, Fgo, Ago, logo, cnt = oracle_solve(orc, md, 3, [7], geometric, log_pm=7)
    assert np.array_equal(A, Ao)
    assert (logo == 2).sum() > 0
    diff = int((log != logo).sum())
    assert diff == 0, f"{diff} ray decisions differ (stats {st})"
    assert np.max(np.abs(F - Fo)) <= ATOL_MIXED
    assert np.max(np.abs(rs - Fo.sum(axis=1))) <= 1e-5
    if near == 1e9:
        assert st["n_pairs_fp64"] > 0


@pytest.mark.parametrize("lists", [True, False])
def test_surface_groups_as_obstructions_mixed(rvf, orc, session, lists):
    """Faces that are both surfaces and obstructions, FP32 rays: own groups
    skipped, ray decisions identical to the FP64 oracle's."""
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    obs = [2, 5, 7]
    F, A, rs, log, st = mixed_solve(rvf, session, md, 3, obs, log_pm=7, lists=lists)
    Fo, Ao, Fgo, Ago, logo, cnt = oracle_solve(orc, md, 3, obs, log_pm=7)
    assert (logo == 2).sum() > 0
    assert np.array_equal(log, logo), f"{int((log != logo).sum())} ray decisions differ (stats {st})"
    assert np.max(np.abs(F - Fo)) <= ATOL_MIXED


def test_pair_lists_fine_cube_mixed(rvf, orc, session):
    """Per-pair triangle lists under FP32 rays (certified decisions, FP64
    re-tests): every sampled row within 1e-6 of the FP64 oracle."""
    md = rvf.meshes.cube_enclosure(20, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12)
    N = md.n_elems
    F, A, rs, _, st = mixed_solve(rvf, session, md, 3, [7])
    assert st["n_list_pairs"] > 100 * st["n_walk_pairs"], st
    Fw, *_ = mixed_solve(rvf, session, md, 3, [7], lists=False)
    assert np.array_equal(F, Fw, equal_nan=True)
    m = orc.Mesh(md, [7])
    raw, area, _, _ = orc.solve_plain(m, 3, row_stride=23)
    assert np.array_equal(A, area)
    for i in range(0, N, 23):
        assert np.max(np.abs(F[i, i + 1:] - raw[i, i + 1:] / area[i])) <= ATOL_MIXED


@pytest.mark.parametrize("family,nquad", [("quad", 3), ("quad4", 4), ("tri", 4)])
def test_families_mixed(rvf, orc, session, family, nquad):
    md = rvf.meshes.cube_enclosure(4, family=family, box_m=2, box_edge=0.5)
    pm = 16 if family in ("quad", "quad4") else 13
    F, A, rs, log, st = mixed_solve(rvf, session, md, nquad, [7], log_pm=pm)
    Fo, Ao, *_, logo, cnt = oracle_solve(orc, md, nquad, [7], log_pm=pm)
    assert np.array_equal(log, logo)
    assert np.max(np.abs(F - Fo)) <= ATOL_MIXED


def test_plates_mixed_accuracy(rvf, orc, session):
    md = rvf.meshes.parallel_plates(20, "quad4")
    F, A, rs, _, st = mixed_solve(rvf, session, md, 4)
    Fo, Ao, *_ = oracle_solve(orc, md, 4)
    assert np.max(np.abs(F - Fo)) <= ATOL_MIXED
    assert st["n_pairs_fp64"] > 0  # neighbouring elements run in FP64


def test_mixed_families_mesh(rvf, orc, session):
    md = concat(rvf.meshes.parallel_plates(3, "quad"), rvf.meshes.cube_enclosure(2, family="tri", box=False))
    F, A, *_ = mixed_solve(rvf, session, md, 3)
    Fo, Ao, *_ = oracle_solve(orc, md, 3)
    assert np.max(np.abs(F - Fo)) <= ATOL_MIXED


def test_curve_mesh_mixed_runs_fp64(rvf, orc, session):
    md = rvf.meshes.cavity_2d(n_wall=16, n_circle=12, n_circles=2)
    F, A, rs, log, st = mixed_solve(rvf, session, md, 3, [5, 6], log_pm=3)
    Fo, Ao, *_, logo, _ = oracle_solve(orc, md, 3, [5, 6], log_pm=3)
    assert np.array_equal(log, logo)
    assert np.max(np.abs(F - Fo) / np.maximum(np.abs(Fo), 1e-300)) <= 1e-10
