"""Self view factors (self_vf): the diagonal pairs (i, i), which the reference
integrates on its CPU path only (src/Assembly.jl:173,193: j_start = i), here
on the device for quadrature solves (plain and Duffy).

Oracle: orc_self_gpu, the GPU path's arithmetic applied to the diagonal
(points, kernel, summation order, shadow rays with the element's own group
skipped), pinned bit for bit to orc_solve_cpu(self_vf=1) -- the restatement of
the reference's CPU path -- where no ray meets an obstruction; Duffy self
pairs against orc_pair_duffy(i, i), which the reference classifies as a
common-edge pair (every corner is shared; the first two matches are taken).
Device tolerance as the other FP64 parity tests: 1e-10 relative.
"""
import math

import numpy as np
import pytest

RTOL = 1e-10


def cylinder(rvf):
    """Curved Quad8 wall (concave seen from inside) with flat annular caps."""
    return rvf.meshes.cylinder(nc=8, na=3, cap_rings=2, jitter=0.01, seed=3)


def cylinder_with_box(rvf):
    """A small box between the chord and the arc of the wall element that
    spans 0-45 degrees, where that element's self rays pass (group 99)."""
    md = cylinder(rvf)
    th = math.radians(22.5)
    md.group_tri_soup[99] = rvf.meshes.obstruction_box(center=(0.48 * math.cos(th), 0.48 * math.sin(th), 1 / 6),
                                                        edge=0.02, m=2)
    return md


def ring_2d(rvf):
    """The 2-D cavity with its circles reversed to counter-clockwise: inward
    normals, so every arc element sees itself (groups 5 and 6)."""
    md = rvf.meshes.cavity_2d(n_wall=8, n_circle=12, n_circles=2, seed=4)
    en = md.elem_nodes.copy()
    c = md.elem_group >= 5
    en[c, 0], en[c, 1] = md.elem_nodes[c, 1], md.elem_nodes[c, 0]
    out = rvf.MeshData(md.coords, en, md.elem_family, md.elem_group, dict(md.group_tags), {}, 1)
    out.group_tri_soup = rvf.build_group_obs_soups(out)
    return out


def oracle_self(orc, md, nquad, obs=(), geometric=False):
    m = orc.Mesh(md, obs)
    raw, area = orc.self_gpu(m, nquad, geometric=geometric)
    return raw / area


# ---------------------------------------------------------------------------
# oracle pins and host plumbing (no GPU)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("nquad", [2, 3])
def test_oracle_self_equals_cpu_path(rvf, orc, nquad):
    for md, obs in ((cylinder(rvf), ()), (ring_2d(rvf), (5, 6))):
        m = orc.Mesh(md, obs)
        raw, area, _ = orc.solve_cpu(m, nquad, self_vf=True)
        g_raw, g_area = orc.self_gpu(m, nquad)
        assert np.array_equal(np.diag(raw), g_raw)
        assert np.array_equal(area, g_area)


def test_oracle_self_concave_positive_flat_rounding(rvf, orc):
    """Concave elements see themselves; flat ones only at rounding level
    (interpolated coordinates of a plane at z = 1 differ by an ulp, so the
    reference's K can be a few 1e-33 there, not exactly 0)."""
    md = cylinder(rvf)
    d = oracle_self(orc, md, 3)
    wall = md.elem_group == 1
    assert (d[wall] > 1e-3).all() and (np.abs(d[~wall]) < 1e-20).all()
    plates = rvf.meshes.parallel_plates(3, "quad")
    assert np.abs(oracle_self(orc, plates, 3)).max() < 1e-20
    r = ring_2d(rvf)
    assert (oracle_self(orc, r, 3, (5, 6))[r.elem_group >= 5] > 0).all()


def test_oracle_box_blocks_self_rays_only_with_true_vertices(rvf, orc):
    """The reference reads soup triangles transposed, so a small box's
    effective triangles lie outside its boxes; with true vertices it blocks."""
    free = oracle_self(orc, cylinder(rvf), 3)
    md = cylinder_with_box(rvf)
    assert np.array_equal(oracle_self(orc, md, 3, (99,)), free)
    assert (oracle_self(orc, md, 3, (99,), geometric=True) != free).sum() >= 1


def test_oracle_duffy_self_pair_is_common_edge(rvf, orc):
    m = orc.Mesh(cylinder(rvf))
    for i in range(m.N):
        t, ci, cj = orc.singularity_type(m, i, i)
        assert t == 2 and list(ci) == [1, 2] and list(cj) == [1, 2]


def test_self_vf_reaches_the_hook(rvf):
    from rvf_b200 import assembly
    md = rvf.meshes.parallel_plates(2, "quad4")
    seen = {}

    def fake(mesh, nquad, backend, FloatT, ArrayT, **kw):
        seen.clear()
        seen.update(kw)
        return "ok"
    prev = assembly._GPU_HOOK_REF[0]
    try:
        rvf.register_gpu_hook(fake)
        rvf.compute_view_factors(md, self_vf=True, verbose=False)
        assert seen["self_vf"] is True
        rvf.compute_view_factors(md, verbose=False)
        assert "self_vf" not in seen
        with pytest.warns(UserWarning, match="self_vf with monte_carlo"):
            rvf.compute_view_factors(md, self_vf=True, monte_carlo=True, verbose=False)
        assert "self_vf" not in seen

        class Other:  # a backend without the capability: dropped silently, as the reference's GPU path does
            pass
        assert not assembly._gpu_supports(Other(), "self_vf")
    finally:
        rvf.register_gpu_hook(prev)
    o = rvf.make_options(3, self_vf=True, seed=0)
    assert o.self_vf == 1 and rvf.make_options(3, seed=0).self_vf == 0


# ---------------------------------------------------------------------------
# device parity
# ---------------------------------------------------------------------------
def device_solve(rvf, session, md, nquad, obs=(), **kw):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
    try:
        N = md.n_elems
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        st = dm.solve(rvf.make_options(nquad, seed=0, **kw), F, A)
        return F, A, st
    finally:
        dm.release()


def assert_rel(a, b, rtol=RTOL):
    bad = ~(np.abs(a - b) <= rtol * np.abs(b) + 1e-300)
    assert not bad.any(), f"{int(bad.sum())} entries differ, e.g. {a[bad][:3]} vs {b[bad][:3]}"


def off_diagonal_equal(F1, F2):
    off = ~np.eye(F1.shape[0], dtype=bool)
    return np.array_equal(F1[off], F2[off])


@pytest.mark.gpu
@pytest.mark.parametrize("nquad", [2, 3, 5])
def test_self_matches_oracle(rvf, orc, session, nquad):
    md = cylinder(rvf)
    F, A, _ = device_solve(rvf, session, md, nquad, self_vf=True)
    F0, A0, _ = device_solve(rvf, session, md, nquad)
    expect = oracle_self(orc, md, nquad)
    assert (expect > 1e-3).sum() == 24  # the wall
    assert_rel(np.diag(F), expect)
    assert off_diagonal_equal(F, F0) and np.array_equal(A, A0)
    assert not np.diag(F0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("geometric", [False, True])
def test_self_with_obstruction(rvf, orc, session, geometric):
    md = cylinder_with_box(rvf)
    F, _, st = device_solve(rvf, session, md, 3, (99,), self_vf=True, geometric_soup=geometric)
    assert_rel(np.diag(F), oracle_self(orc, md, 3, (99,), geometric=geometric))
    assert st.n_rays > 0


@pytest.mark.gpu
@pytest.mark.parametrize("nquad", [2, 3])
def test_self_duffy_matches_oracle(rvf, orc, session, nquad):
    md = cylinder(rvf)
    m = orc.Mesh(md)
    F, A, st = device_solve(rvf, session, md, nquad, self_vf=True, use_duffy=True)
    F0, _, st0 = device_solve(rvf, session, md, nquad, use_duffy=True)
    expect = np.array([orc.pair_duffy(m, i, i, nquad, None, gpu_semantics=True)[0] for i in range(m.N)]) / A
    assert_rel(np.diag(F), expect)
    assert off_diagonal_equal(F, F0)
    assert st.n_duffy_pairs == st0.n_duffy_pairs
    # the Duffy value replaces the plain one (they differ on curved elements)
    Fp, _, _ = device_solve(rvf, session, md, nquad, self_vf=True)
    assert (np.diag(Fp) != np.diag(F)).any()


@pytest.mark.gpu
def test_self_curves(rvf, orc, session):
    md = ring_2d(rvf)
    F, _, _ = device_solve(rvf, session, md, 3, (5, 6), self_vf=True)
    expect = oracle_self(orc, md, 3, (5, 6))
    assert (expect > 1e-3).sum() == int((md.elem_group >= 5).sum())
    assert_rel(np.diag(F), expect)


@pytest.mark.gpu
def test_self_mixed_equals_fp64(rvf, session):
    """The self pairs run in FP64 in both modes."""
    md = cylinder_with_box(rvf)
    F64, _, _ = device_solve(rvf, session, md, 3, (99,), self_vf=True, geometric_soup=True)
    Fmx, _, _ = device_solve(rvf, session, md, 3, (99,), self_vf=True, geometric_soup=True, precision="mixed")
    assert np.array_equal(np.diag(F64), np.diag(Fmx))


@pytest.mark.gpu
def test_self_flat_elements(rvf, orc, session):
    md = rvf.meshes.parallel_plates(4, "quad")
    F, _, _ = device_solve(rvf, session, md, 3, self_vf=True)
    assert_rel(np.diag(F), oracle_self(orc, md, 3))
    assert np.abs(np.diag(F)).max() < 1e-20


@pytest.mark.gpu
def test_self_monte_carlo_rejected(rvf, session):
    from rvf_b200 import _abi
    with pytest.raises(_abi.RVFError, match="quadrature only"):
        device_solve(rvf, session, cylinder(rvf), 3, self_vf=True, monte_carlo=True, n_samples=16)


@pytest.mark.gpu
def test_self_served_identical_to_solo(rvf, session):
    from rvf_b200 import _abi
    mix = [(cylinder(rvf), (), dict(self_vf=True)),
           (cylinder(rvf), (), dict(self_vf=True, use_duffy=True)),
           (cylinder_with_box(rvf), (99,), dict(self_vf=True, geometric_soup=True, precision="mixed"))]
    expect = [device_solve(rvf, session, md, 3, obs, **kw)[0] for md, obs, kw in mix]
    sv = _abi.Server(session)
    try:
        ids = [sv.submit(rvf.mesh_desc_arrays(md, obs), rvf.make_options(3, seed=0, **kw)) for md, obs, kw in mix]
        for k, rid in enumerate(ids):
            sv.wait(rid, 120000)
            assert np.array_equal(sv.result(rid)[0], expect[k])
            sv.release(rid)
    finally:
        sv.close()
