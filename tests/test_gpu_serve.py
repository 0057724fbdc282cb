"""The serving loop (rvf_server): requests of different sizes, families,
methods and precisions submitted together are admitted by device footprint,
batched into shared launches, and each result is bit-identical to a
one-at-a-time rvf_solve of the same mesh and options."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solo(rvf, session, md, obs, opts):
    from rvf_b200 import _abi
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, obs))
    try:
        N, G = md.n_elems, len(md.group_tags)
        F = np.empty((N, N), order="F")
        A = np.empty(N)
        Fg = np.empty((G, G), order="F")
        Ag = np.empty(G)
        dm.solve(opts, F, A, Fg, Ag)
        return F, A, Fg, Ag
    finally:
        dm.release()


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    ok = (a == b) | (np.isnan(a) & np.isnan(b))
    return bool(ok.all())


def request_mix(rvf):
    """(mesh, obstruction groups, options): two launch classes with several
    members each, curves, Duffy and Monte Carlo."""
    m = rvf.meshes
    mk = rvf.make_options
    return [
        (m.cube_enclosure(6, family="tri3", box_m=3), [7], mk(3, seed=0)),
        (m.cube_enclosure(4, family="quad4", box_m=2), [7], mk(2, seed=0)),
        (m.cube_enclosure(5, family="tri", box_m=2, box_edge=0.5), [7], mk(4, seed=0)),
        (m.parallel_plates(6, "quad"), [], mk(3, seed=0)),
        (m.cube_enclosure(6, family="tri3", box_m=3), [7], mk(3, seed=0, precision="mixed")),
        (m.cube_enclosure(4, family="quad", box_m=2), [7], mk(3, seed=0, precision="mixed")),
        (m.cube_enclosure(3, family="quad", box_m=2, box_edge=0.5), [7], mk(3, seed=0, use_duffy=True)),
        (m.cavity_2d(n_wall=24, n_circle=16, n_circles=2, seed=4), [5, 6], mk(3, seed=0)),
        (m.cube_enclosure(3, family="quad4", box_m=2), [7], mk(4, monte_carlo=True, n_samples=16, seed=5)),
    ]


@pytest.mark.parametrize("use_graphs", [True, False])
def test_batched_results_identical_to_solo(rvf, session, use_graphs):
    from rvf_b200 import _abi
    mix = request_mix(rvf)
    expect = [solo(rvf, session, md, obs, o) for md, obs, o in mix]
    sv = _abi.Server(session, use_graphs=use_graphs)
    try:
        ids = [sv.submit(rvf.mesh_desc_arrays(md, obs), o) for md, obs, o in mix]
        for k, rid in enumerate(ids):
            sv.wait(rid, 120000)
            F, A, Fg, Ag = sv.result(rid)
            eF, eA, eFg, eAg = expect[k]
            assert same(F, eF), f"request {k}: F differs from rvf_solve"
            assert same(A, eA) and same(Fg, eFg) and same(Ag, eAg), f"request {k}"
            sv.release(rid)
        st = sv.stats()
        assert st["completed"] == len(mix) and st["failed"] == 0
        assert st["batched_requests"] > st["chunks"], "same-class requests should share launches"
        if use_graphs:
            assert st["graph_replays"] > 0
        assert 0 < st["p50_ms"] <= st["p99_ms"]
    finally:
        sv.close()


def test_admission_budget(rvf, session):
    """With room for one request at a time every request still completes, the
    admitted footprint never exceeds the budget, and a request larger than
    the whole budget fails with RVF_EBUDGET."""
    from rvf_b200 import _abi
    small = rvf.meshes.cube_enclosure(4, family="tri3", box_m=2)
    big = rvf.meshes.cube_enclosure(20, family="tri3", box_m=2)
    o = rvf.make_options(3, seed=0)
    probe = _abi.Server(session)
    rid = probe.submit(rvf.mesh_desc_arrays(small, [7]), o)
    probe.wait(rid, 60000)
    _, _, info = probe.poll(rid)
    one = int(info.footprint_bytes)
    probe.release(rid)
    probe.close()
    ref = solo(rvf, session, small, [7], o)[0]
    sv = _abi.Server(session, admit_bytes=int(one * 1.5))
    try:
        ids = [sv.submit(rvf.mesh_desc_arrays(small, [7]), o) for _ in range(3)]
        huge = sv.submit(rvf.mesh_desc_arrays(big, [7]), o)
        for rid in ids:
            sv.wait(rid, 60000)
            assert same(sv.result(rid)[0], ref)
            sv.release(rid)
        with pytest.raises(_abi.RVFError) as ei:
            sv.wait(huge, 60000)
        assert ei.value.status == _abi.RVF_EBUDGET
        st = sv.stats()
        assert st["admitted_bytes_peak"] <= int(one * 1.5)
        assert st["completed"] == 3 and st["failed"] == 1
    finally:
        sv.close()


def test_cancel_timeout_release(rvf, session):
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(16, family="tri3", box_m=3)
    o = rvf.make_options(3, seed=0)
    sv = _abi.Server(session)
    try:
        a = sv.submit(rvf.mesh_desc_arrays(md, [7]), o)
        b = sv.submit(rvf.mesh_desc_arrays(md, [7]), o)
        sv.cancel(b)
        with pytest.raises(_abi.RVFError) as ei:
            sv.wait(a, 0)  # no time at all: still queued or running
        assert ei.value.status == _abi.RVF_ETIMEDOUT
        sv.wait(a, 120000)
        with pytest.raises(_abi.RVFError) as ei:
            sv.wait(b, 120000)
        assert ei.value.status == _abi.RVF_ECANCELED
        with pytest.raises(_abi.RVFError):
            sv.result(b)
        sv.release(a)
        sv.release(b)
        assert sv.poll(a)[1] == _abi.RVF_EINVAL  # released: unknown id
        st = sv.stats()
        assert st["completed"] == 1 and st["canceled"] == 1 and st["in_flight"] == 0
    finally:
        sv.close()


def test_autotuned_shapes_reported_and_identical(rvf, session):
    """The first admissions of a launch class and size class each run one
    candidate shape of the quadrature-only kernel; the sweep's choice is
    reported in rvf_server_stats, and every result stays bit-identical to
    rvf_solve whatever shape computed it."""
    from rvf_b200 import _abi
    m = rvf.meshes
    mk = rvf.make_options
    mix = []
    for prec in ("fp64", "mixed"):
        md = m.cube_enclosure(10, family="tri3", box_m=3)
        mix += [(md, [7], mk(3, seed=0, precision=prec))] * 6
    expect = {prec: solo(rvf, session, mix[k][0], [7], mix[k][2]) for k, prec in ((0, "fp64"), (6, "mixed"))}
    own = rvf.Session(0)  # a session of its own: no choices of earlier tests
    sv = _abi.Server(own, max_batch=1)
    try:
        ids = [sv.submit(rvf.mesh_desc_arrays(md, obs), o) for md, obs, o in mix]
        for k, rid in enumerate(ids):
            sv.wait(rid, 120000)
            F, A, Fg, Ag = sv.result(rid)
            eF, eA, eFg, eAg = expect["fp64" if k < 6 else "mixed"]
            assert same(F, eF) and same(A, eA) and same(Fg, eFg), f"request {k}"
            sv.release(rid)
        st = sv.stats()
        assert st["completed"] == len(mix)
        # this class in both precisions
        tuned = st["tuned"]
        assert sorted(t["mixed"] for t in tuned) == [0, 1], st["tuned"]
        for t in tuned:
            assert t["occlusion"] == 1 and t["dim3"] == 1 and t["rule_points"] == 7
            assert t["fast_points"] >= 2 and t["fast_row_groups"] in (1, 2, 4, 8, 32)
            assert 0 < t["fast_ms_per_gpp"] <= t["fast_ms_per_gpp_default"]
        assert len(st["tuned"]) == 2
    finally:
        sv.close()
        own.close()


def test_wait_any_returns_each_finished_request_once(rvf, session):
    """rvf_wait_any hands out every finished request once, in the order they
    finished, and times out when no unreported request is finished."""
    from rvf_b200 import _abi
    m = rvf.meshes
    mix = [(m.cube_enclosure(8, family="tri3", box_m=3), [7], rvf.make_options(3, seed=0)),
           (m.parallel_plates(4, "quad4"), [], rvf.make_options(2, seed=0)),
           (m.cube_enclosure(3, family="quad4", box_m=2), [7], rvf.make_options(2, monte_carlo=True, n_samples=4, seed=1))]
    sv = _abi.Server(session)
    try:
        ids = [sv.submit(rvf.mesh_desc_arrays(md, obs), o) for md, obs, o in mix]
        got = []
        for _ in ids:
            rid = sv.wait_any(120000)
            assert rid is not None
            assert sv.poll(rid)[0] == "done"
            got.append(rid)
            sv.release(rid)
        assert sorted(got) == sorted(ids)
        assert sv.wait_any(50) is None
    finally:
        sv.close()
