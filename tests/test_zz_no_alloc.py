"""rvf_solve_fp64_noalloc, the entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc themselves or through the
library (an allocator that owns all device memory, a memory-capped service, a
host that only hands over pre-placed buffers): its scratch is one fixed array
inside the library.  torch stands in for such a caller's allocator here: it
owns every input and output buffer, and the entry point, called through the C
ABI, must reproduce rvf_solve's F and A (same tolerance as the parity tests)
on two calls in a row with meshes of different sizes, so that contents left
in the shared array by the first call cannot leak into the second.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _existing_entry_point(rvf, session, md, nquad, obstruction_groups=()):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obstruction_groups))
    try:
        N = md.n_elems
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        dm.solve(rvf.make_options(nquad, seed=0, occlusion=False), F, A)
        return F, A
    finally:
        dm.release()


def _oracle(orc, md, nquad):
    """The oracle's plain FP64 assembly without obstructions."""
    m = orc.Mesh(md)
    raw, area, _, _ = orc.solve_plain(m, nquad)
    return orc.f_from_raw(raw, area), area


def _noalloc(rvf, md, nquad):
    import torch
    from rvf_b200 import _abi
    lib = _abi.load_library()
    dev = torch.device("cuda:0")
    N = md.n_elems
    coords = torch.from_numpy(np.asfortranarray(md.coords).ravel(order="F").copy()).to(dev)
    fam = torch.from_numpy(np.ascontiguousarray(md.elem_family, dtype=np.int8)).to(dev)
    nodes = torch.from_numpy(np.ascontiguousarray(md.elem_nodes, dtype=np.int32)).to(dev)
    grp = torch.from_numpy(np.ascontiguousarray(md.elem_group, dtype=np.int32)).to(dev)
    F = torch.full((N * N,), float("nan"), dtype=torch.float64, device=dev)
    A = torch.full((N,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = lib.rvf_solve_fp64_noalloc(coords.data_ptr(), md.coords.shape[1], fam.data_ptr(), nodes.data_ptr(),
                                    grp.data_ptr(), N, md.mesh_dim, nquad, F.data_ptr(), A.data_ptr(), None)
    return rc, F.cpu().numpy().reshape((N, N), order="F"), A.cpu().numpy()


def _assert_rel(a, b):
    assert a.shape == b.shape
    bad = ~((np.abs(a - b) <= RTOL * np.abs(b) + 1e-300) | (np.isnan(a) & np.isnan(b)))
    assert not bad.any(), f"{int(bad.sum())} entries differ beyond rtol={RTOL}"


def test_noalloc_matches_rvf_solve_on_two_calls(rvf, orc, session):
    first = rvf.meshes.parallel_plates(10, "quad")        # 200 Quad8, nquad 4 (16 points)
    second = rvf.meshes.cube_enclosure(3, box=False)      # 108 Tri3, nquad 3 (7 points)
    for md, nq in ((first, 4), (second, 3)):
        F_ref, A_ref = _existing_entry_point(rvf, session, md, nq)
        rc, F, A = _noalloc(rvf, md, nq)
        assert rc == 0, rvf._abi.last_error()
        _assert_rel(A, A_ref)
        _assert_rel(F, F_ref)
        F_orc, A_orc = _oracle(orc, md, nq)
        _assert_rel(A, A_orc)
        _assert_rel(F, F_orc)


def test_noalloc_ignores_obstructions(rvf, session):
    """No obstruction: on a cube with an obstructing box (and faces that hide
    one another behind it) the result equals rvf_solve with occlusion off."""
    md = rvf.meshes.cube_enclosure(4, box_m=2)
    F_ref, A_ref = _existing_entry_point(rvf, session, md, 3, obstruction_groups=[7])
    rc, F, A = _noalloc(rvf, md, 3)
    assert rc == 0, rvf._abi.last_error()
    _assert_rel(A, A_ref)
    _assert_rel(F, F_ref)


def test_noalloc_rejects_unsupported_nquad(rvf, session):
    md = rvf.meshes.parallel_plates(2, "quad4")
    rc, _, _ = _noalloc(rvf, md, 100000)
    assert rc == -7  # RVF_EUNSUPPORTED, before any rule is built
    assert "nquad" in rvf._abi.last_error()


def test_noalloc_rejects_host_pointers(rvf, session):
    import torch
    from rvf_b200 import _abi
    lib = _abi.load_library()
    md = rvf.meshes.parallel_plates(2, "quad4")
    N = md.n_elems
    dev = torch.device("cuda:0")
    coords_host = np.asfortranarray(md.coords).ravel(order="F").copy()
    fam = torch.from_numpy(np.ascontiguousarray(md.elem_family, dtype=np.int8)).to(dev)
    nodes = torch.from_numpy(np.ascontiguousarray(md.elem_nodes, dtype=np.int32)).to(dev)
    grp = torch.from_numpy(np.ascontiguousarray(md.elem_group, dtype=np.int32)).to(dev)
    F = torch.zeros(N * N, dtype=torch.float64, device=dev)
    A = torch.zeros(N, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = lib.rvf_solve_fp64_noalloc(coords_host.ctypes.data, md.coords.shape[1], fam.data_ptr(), nodes.data_ptr(),
                                    grp.data_ptr(), N, md.mesh_dim, 2, F.data_ptr(), A.data_ptr(), None)
    assert rc == -1
    assert "coords" in _abi.last_error()


def test_noalloc_rejects_meshes_beyond_its_scratch(rvf, session):
    md = rvf.meshes.parallel_plates(70, "quad4")  # 9,800 elements x 64 points at nquad 8: > 16 MiB of tables
    rc, _, _ = _noalloc(rvf, md, 8)
    assert rc == -1
    assert "scratch" in rvf._abi.last_error()


def test_noalloc_rejects_bad_node_ids(rvf, session):
    md = rvf.meshes.parallel_plates(2, "quad4")
    md.elem_nodes[1, 3] = 10_000
    rc, _, _ = _noalloc(rvf, md, 2)
    assert rc == -1
    assert "node id" in rvf._abi.last_error()
