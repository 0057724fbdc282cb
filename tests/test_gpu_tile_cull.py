"""Tile classification (kernels_cull.cu) and the generation's quadrature-only
tiles, against the same solve with the classification off and against the
oracle.

With occlusion, a tile whose pairs' shadow rays can provably not be blocked
skips all ray work, and inside the other tiles only the pairs of the tile's
mask send their rays through the ray pipeline.  Neither may change a single
ray decision: F agrees with the unclassified solve to rounding (1e-12
relative in FP64 -- only the order in which visible terms are added
differs -- and 1e-6 in mixed precision), and with the oracle to the parity
tolerances.  Without occlusion the quadrature-only tiles form every term
exactly as the ray pipeline does, so F is identical bit for bit.
"""
import numpy as np
import pytest

from test_gpu_parity import assert_rel

pytestmark = pytest.mark.gpu


def solve(rvf, session, md, nquad, obs, precision="fp64", cull=True, geometric=False, near=2.0):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
    try:
        N = md.n_elems
        o = rvf.make_options(nquad, precision=precision, geometric_soup=geometric, seed=0)
        o.disable_tile_cull = 0 if cull else 1
        o.near_field_factor = near
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        st = dm.solve(o, F, A)
        return F, A, st.as_dict()
    finally:
        dm.release()


@pytest.mark.parametrize("geometric", [False, True])
def test_culled_cube_fp64(rvf, orc, session, geometric):
    md = rvf.meshes.cube_enclosure(20, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12)
    N = md.n_elems
    F, A, st = solve(rvf, session, md, 3, [7], geometric=geometric)
    F0, A0, st0 = solve(rvf, session, md, 3, [7], cull=False, geometric=geometric)
    assert st["n_tiles_culled"] > 0 and st0["n_tiles_culled"] == 0
    assert st["n_rays"] == st0["n_rays"]  # every cast ray is counted, traced or not
    assert np.array_equal(A, A0)
    assert_rel(F, F0, rtol=1e-12)
    if geometric:
        # true triangles cover the box: every ray through its box can hit one,
        # so the masks keep exactly the rays the root-box test keeps
        assert st["n_rays_traced"] == st0["n_rays_traced"]
    else:
        # the reference's transposed read leaves many of them unblockable
        assert st["n_rays_traced"] < st0["n_rays_traced"]
    m = orc.Mesh(md, [7])
    raw, area, _, _ = orc.solve_plain(m, 3, geometric=geometric, row_stride=37)
    assert np.array_equal(A, area)
    for i in range(0, N, 37):
        assert_rel(F[i, i + 1:], raw[i, i + 1:] / area[i])
        assert_rel(F[i + 1:, i], raw[i, i + 1:] / area[i + 1:])


def test_culled_cube_mixed(rvf, orc, session):
    md = rvf.meshes.cube_enclosure(20, jitter=0.3, seed=2, box=True, box_edge=0.3, box_m=12)
    N = md.n_elems
    F, A, st = solve(rvf, session, md, 3, [7], precision="mixed")
    F0, A0, st0 = solve(rvf, session, md, 3, [7], precision="mixed", cull=False)
    assert st["n_tiles_culled"] > 0
    assert np.max(np.abs(F - F0)) <= 1e-6
    m = orc.Mesh(md, [7])
    raw, area, _, _ = orc.solve_plain(m, 3, row_stride=41)
    for i in range(0, N, 41):
        assert np.max(np.abs(F[i, i + 1:] - raw[i, i + 1:] / area[i])) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_surface_groups_as_obstructions_culled(rvf, orc, session, precision):
    """Faces that are also obstructions: the tile walk keeps their triangles
    unless both of a tile's blocks lie in those very groups."""
    md = rvf.meshes.cube_enclosure(8, box_m=4)
    obs = [2, 5, 7]
    F, A, st = solve(rvf, session, md, 3, obs, precision=precision)
    F0, *_ = solve(rvf, session, md, 3, obs, precision=precision, cull=False)
    m = orc.Mesh(md, obs)
    raw, area, _, _ = orc.solve_plain(m, 3)
    Fo = orc.f_from_raw(raw, area)
    if precision == "fp64":
        assert_rel(F, F0, rtol=1e-12)
        assert_rel(F, Fo)
    else:
        assert np.max(np.abs(F - F0)) <= 1e-6
        assert np.max(np.abs(F - Fo)) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("family,nquad", [("quad4", 4), ("quad", 5), ("tri3", 3), ("tri", 4), ("tri3", 2)])
def test_quadrature_only_tiles_bit_identical(rvf, session, precision, family, nquad):
    """No obstruction: every far-field tile runs the quadrature-only loop,
    which forms each term in the ray pipeline's order and arithmetic."""
    md = rvf.meshes.parallel_plates(12, family)
    F, A, st = solve(rvf, session, md, nquad, [], precision=precision)
    F0, A0, _ = solve(rvf, session, md, nquad, [], precision=precision, cull=False)
    assert np.array_equal(A, A0)
    assert np.array_equal(F, F0, equal_nan=True), f"max |dF| {np.nanmax(np.abs(F - F0))}"


def test_near_tiles_keep_fp64_in_mixed(rvf, orc, session):
    """Mixed precision with the near-field rule off (factor 0) and on (2):
    both within 1e-6 of the oracle, near-field pairs counted in FP64 only
    when the rule is on."""
    md = rvf.meshes.parallel_plates(20, "quad4")
    m = orc.Mesh(md)
    raw, area, _, _ = orc.solve_plain(m, 4)
    Fo = orc.f_from_raw(raw, area)
    for near in (0.0, 2.0):
        F, A, st = solve(rvf, session, md, 4, [], precision="mixed", near=near)
        assert np.max(np.abs(F - Fo)) <= 1e-6
        assert (st["n_pairs_fp64"] > 0) == (near > 0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fast_kernel_shapes_bit_identical(rvf, session, precision):
    """Every compiled shape of the quadrature-only kernel (points per lane
    block, warp tasks per tile) forms each pair by the same loop: F is
    identical bit for bit, with and without occlusion."""
    from rvf_b200 import _abi
    cases = [(rvf.meshes.cube_enclosure(9, family="tri3", box_m=3), [7], 3),
             (rvf.meshes.parallel_plates(10, "quad"), [], 3)]
    points = (2, 3, 4) if precision == "fp64" else (2, 3, 4, 5, 7, 8)
    for md, obs, nquad in cases:
        dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
        try:
            N = md.n_elems
            ref = None
            for qb in (0,) + points:
                for groups in (0, 1, 2, 4, 8, 32):
                    o = rvf.make_options(nquad, precision=precision, seed=0)
                    o.fast_points, o.fast_row_groups = qb, groups
                    F = np.empty((N, N), order="F")
                    dm.solve(o, F)
                    if ref is None:
                        ref = F
                    assert np.array_equal(F, ref, equal_nan=True), (qb, groups)
            o = rvf.make_options(nquad, precision=precision, seed=0)
            o.fast_points = 6
            with pytest.raises(_abi.RVFError) as ei:
                dm.solve(o, np.empty((N, N), order="F"))
            assert ei.value.status == _abi.RVF_EINVAL
        finally:
            dm.release()
