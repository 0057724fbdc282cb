"""Failure paths in the allowed forms: each failure is made on the host or by
a bounded device loop that gives up, never by a fault, trap or hang of the
GPU, and the session must solve correctly right after it.

* RVF_FAULT_ALLOC fails the first device allocation of a call: the solve
  returns RVF_ENOMEM (the reference raises a Julia error where an allocation
  fails, src/GPUAssembly.jl:54) and the next solve on the same session
  succeeds with the unfaulted result.
* RVF_FAULT_CLAIM gives the pair pipeline's tile claims no compare-and-swap
  retries, so every claim gives up at once: the host sees a chunk that
  claimed nothing and returns RVF_ETIMEDOUT; the next solve succeeds.
* A malformed option (unknown fault bits) is RVF_EINVAL before any work.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _opts(rvf, fault=0, precision="fp64"):
    o = rvf.make_options(3, seed=0, precision=precision)
    o.fault_inject = fault
    return o


def _solve(dm, o, N):
    F = np.empty((N, N), order="F")
    A = np.empty(N)
    dm.solve(o, F, A)
    return F, A


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_injected_allocation_failure_then_recovery(rvf, session, precision):
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    N = md.n_elems
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))  # fresh mesh: its tables are not built yet
    try:
        with pytest.raises(_abi.RVFError) as ei:
            _solve(dm, _opts(rvf, _abi.FAULT_ALLOC, precision), N)
        assert ei.value.status == _abi.RVF_ENOMEM
        assert "injected" in str(ei.value)
        F, A = _solve(dm, _opts(rvf, 0, precision), N)
    finally:
        dm.release()
    dm2 = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))
    try:
        F2, A2 = _solve(dm2, _opts(rvf, 0, precision), N)
    finally:
        dm2.release()
    assert np.array_equal(A, A2)
    assert np.array_equal(F, F2, equal_nan=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tile_claims_that_give_up_time_out_then_recovery(rvf, session, precision):
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(6, box_m=3)
    N = md.n_elems
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))
    try:
        F0, A0 = _solve(dm, _opts(rvf, 0, precision), N)
        with pytest.raises(_abi.RVFError) as ei:
            _solve(dm, _opts(rvf, _abi.FAULT_CLAIM, precision), N)
        assert ei.value.status == _abi.RVF_ETIMEDOUT
        assert "gave up" in str(ei.value)
        F1, A1 = _solve(dm, _opts(rvf, 0, precision), N)
    finally:
        dm.release()
    assert np.array_equal(F0, F1, equal_nan=True)
    assert np.array_equal(A0, A1)


def test_unknown_fault_bits_are_rejected(rvf, session):
    from rvf_b200 import _abi
    md = rvf.meshes.parallel_plates(2, "quad4")
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, ()))
    try:
        with pytest.raises(_abi.RVFError) as ei:
            _solve(dm, _opts(rvf, 64), md.n_elems)
        assert ei.value.status == _abi.RVF_EINVAL
    finally:
        dm.release()
