"""Host F downloaded column by column while later chunks compute: a session
with a small HBM budget runs the pair pipeline in many chunks, so the
finished columns of each chunk's tile rows go to the host early.  Every
column must arrive, bit for bit the result of a one-chunk solve, into pinned
(overlapped copies) and pageable (synchronous copies) host memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chunked_solve_downloads_every_column(rvf, session, pinned, precision):
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(16, box_m=6)
    N = md.n_elems
    o = rvf.make_options(3, seed=0, precision=precision)
    # every ray through the queues (no tile classification), so that a small
    # budget forces many chunks
    o.disable_tile_cull = 1
    ref = np.empty((N, N), order="F")
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))
    st_ref = dm.solve(o, ref)
    dm.release()
    small = _abi.Session(0, hbm_budget_bytes=256 << 20)
    buf = _abi.PinnedArray((N, N), order="F") if pinned else None
    try:
        F = buf.array if pinned else np.empty((N, N), order="F")
        F.fill(-7.0)  # a column never written keeps this
        dm = _abi.DeviceMesh(small, rvf.mesh_desc_arrays(md, [7]))
        st = dm.solve(o, F)
        dm.release()
        assert st.n_chunks > 4 * st_ref.n_chunks, (st.n_chunks, st_ref.n_chunks)
        assert np.array_equal(F, ref, equal_nan=True)
    finally:
        if buf is not None:
            buf.free()
        small.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_odd_size_pinned_equals_pageable(rvf, session, precision):
    """An odd N (columns of F not 16-byte aligned in host memory): pinned
    (overlapped copies) and pageable destinations receive the same F."""
    from rvf_b200 import _abi
    full = rvf.meshes.cube_enclosure(5, box_m=2)
    md = rvf.MeshData(full.coords, full.elem_nodes[:-1], full.elem_family[:-1], full.elem_group[:-1],
                      dict(full.group_tags), dict(full.group_tri_soup), 2)
    N = md.n_elems
    assert N % 2 == 1
    o = rvf.make_options(3, seed=0, precision=precision)
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))
    buf = _abi.PinnedArray((N, N), order="F")
    try:
        ref = np.empty((N, N), order="F")
        dm.solve(o, ref)
        F = buf.array
        F.fill(-7.0)
        dm.solve(o, F)
        assert np.array_equal(F, ref, equal_nan=True)
    finally:
        buf.free()
        dm.release()
