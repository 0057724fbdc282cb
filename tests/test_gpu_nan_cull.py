"""Rays that lie in the plane of a flat BVH box (src/GPUBVH.jl:219-229).

The reference's slab test takes Julia's min / max, which propagate NaN: a
ray with a zero direction component whose origin lies exactly on a box
bound gives (lo - o) * (1/0) = 0 * Inf = NaN, and a box that is flat in
that coordinate (lo == hi == o) then fails the test -- C's fmin / fmax would
drop the NaN and pass it.  Here two facing plates (x = 0 and x = 1, Quad4,
nquad 3) have element centres exactly on z = 0.625, so the rays between them
run in that plane with d_z = 0; a flat obstruction plate at z = 0.625 gives
the tree flat nodes and leaves at that height, while a second obstruction
stretches the root box above and below it.  Every ray decision must equal
the oracle's (which follows the reference's NaN semantics), in both
precisions, with and without pair lists and tile classification.
"""
import numpy as np
import pytest

from conftest import load_pkg

Z_PLANE = 0.625


def nan_plane_mesh():
    rvf = load_pkg()
    nodes, xyz = {}, []

    def nid(p):
        if p not in nodes:
            xyz.append(p)
            nodes[p] = len(xyz)
        return nodes[p]

    ys = [0.0, 0.25, 0.5, 0.75, 1.0]
    zs = [0.25, 0.5, 0.75, 1.0]  # the middle row's centres lie on z = 0.625 exactly
    elems, grp = [], []
    for x, g in ((0.0, 1), (1.0, 2)):
        for a in range(4):
            for b in range(3):
                y0, y1, z0, z1 = ys[a], ys[a + 1], zs[b], zs[b + 1]
                if g == 1:  # normal +x
                    el = (nid((x, y0, z0)), nid((x, y1, z0)), nid((x, y1, z1)), nid((x, y0, z1)))
                else:  # normal -x
                    el = (nid((x, y0, z0)), nid((x, y0, z1)), nid((x, y1, z1)), nid((x, y1, z0)))
                elems.append(el)
                grp.append(g)
    en = np.zeros((len(elems), 8), dtype=np.int32)
    en[:, :4] = elems
    md = rvf.MeshData(np.array(xyz).T, en, np.full(len(elems), 2, dtype=np.int8), np.array(grp, dtype=np.int32),
                      {1: "x0", 2: "x1"}, {}, 2)
    g = np.linspace(0.25, 0.75, 5)
    tris = []
    for i in range(4):
        for j in range(4):
            c00, c10 = (g[i], g[j], Z_PLANE), (g[i + 1], g[j], Z_PLANE)
            c11, c01 = (g[i + 1], g[j + 1], Z_PLANE), (g[i], g[j + 1], Z_PLANE)
            tris += [(c00, c10, c11), (c00, c11, c01)]
    md.group_tri_soup[8] = np.ascontiguousarray(np.array(tris, dtype=np.float64))
    md.group_tri_soup[9] = rvf.meshes.obstruction_box(center=(0.5, 2.0, 0.5), edge=0.8, m=1)
    return md


def test_nan_plane_geometry(orc):
    """The case exercises the branch: flat nodes at the plane below a root
    that spans it, and rays in the plane with an exactly zero z component."""
    md = nan_plane_mesh()
    soup = np.concatenate([md.group_tri_soup[8], md.group_tri_soup[9]])
    lo, hi, meta, _ = orc.BVH(soup).export()
    assert lo[0, 2] < Z_PLANE < hi[0, 2]
    assert any(lo[k, 2] == hi[k, 2] == Z_PLANE and meta[k, 3] > 0 for k in range(lo.shape[0]))
    m = orc.Mesh(md, [8, 9])
    on_plane = [e for e in range(md.n_elems) if orc.eval_point(m, e, 0.0, 0.0)[0][2] == Z_PLANE]
    assert len(on_plane) == 8  # the middle row of both plates


@pytest.mark.gpu
@pytest.mark.parametrize("cull", [True, False])
@pytest.mark.parametrize("lists", [True, False])
@pytest.mark.parametrize("geometric", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rays_in_flat_box_planes_match_oracle(rvf, orc, session, precision, geometric, lists, cull):
    from rvf_b200 import _abi
    md = nan_plane_mesh()
    obs = [8, 9]
    N = md.n_elems
    pm = 9
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
    try:
        o = rvf.make_options(3, precision=precision, geometric_soup=geometric, seed=0)
        o.disable_pair_lists = 0 if lists else 1
        o.disable_tile_cull = 0 if cull else 1
        log = np.zeros(N * N * pm * pm, dtype=np.uint8)
        o.ray_log = log.ctypes.data_as(_abi._pu8)
        o.ray_log_pm = pm
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        dm.solve(o, F, A)
    finally:
        dm.release()
    m = orc.Mesh(md, obs)
    raw, area, logo, _ = orc.solve_plain(m, 3, geometric=geometric, ray_log_pm=pm)
    Fo = orc.f_from_raw(raw, area)
    assert (logo > 0).sum() > 0
    assert np.array_equal(log, logo), f"{int((log != logo).sum())} ray decisions differ"
    if precision == "fp64":
        ok = (np.abs(F - Fo) <= 1e-10 * np.abs(Fo) + 1e-300) | (np.isnan(F) & np.isnan(Fo))
        assert ok.all()
    else:
        assert np.nanmax(np.abs(F - Fo)) <= 1e-6
