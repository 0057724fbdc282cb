"""CPU tests of the boundary: the C-ABI library loads and exports every
symbol declared in include/rvf_b200.h, its host-side pieces (quadrature rules,
BVH build) match the oracle bit for bit, and the Python mirror of the
reference API behaves like src/Assembly.jl.  No compute call needs a GPU."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_pkg

HEADER = ROOT / "include" / "rvf_b200.h"


@pytest.fixture(scope="module")
def lib(rvf):
    from importlib import import_module
    import_module("rvf_b200.build").build()
    return rvf.load_library()


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rvf_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(lib, rvf):
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared in rvf_b200.h but not exported"
    # and the ctypes table binds exactly the declared set
    from rvf_b200 import _abi
    assert sorted(_abi.SIGNATURES) == names


def test_version_and_defaults(lib, rvf):
    from rvf_b200 import _abi
    assert b"sm_100a" in lib.rvf_version()
    assert lib.rvf_abi_version() == 2
    o = _abi.default_options()
    assert o.nquad == 4 and o.n_samples == 10000 and o.method == 0 and o.precision == 0
    assert o.near_field_factor == 2.0


def test_struct_sizes_match_header(lib):
    """Compile-free layout check: the C ABI structs as ctypes sees them."""
    from rvf_b200 import _abi
    assert ctypes.sizeof(_abi.Options) == 4 * 4 + 8 + 4 * 4 + 8 + 8 + 4 + 4 * 8 + 4  # trailing pad to 8
    assert ctypes.sizeof(_abi.MeshDesc) % 8 == 0


def test_struct_layouts_match_compiled_header(tmp_path, rvf):
    """sizeof / offsetof of every ABI struct, compiled from the header with
    gcc, against the ctypes mirror."""
    import shutil
    import subprocess
    from rvf_b200 import _abi
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    structs = {"rvf_session_opts": _abi.SessionOpts, "rvf_mesh_desc": _abi.MeshDesc, "rvf_options": _abi.Options,
               "rvf_stats": _abi.Stats, "rvf_server_opts": _abi.ServerOpts, "rvf_request_info": _abi.RequestInfo,
               "rvf_server_stats": _abi.ServerStats, "rvf_tuned_shape": _abi.TunedShape}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for cname, ct in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        c, f, v = ln.split()
        got[(c, f)] = int(v)
    for cname, ct in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert got[(cname, fname)] == getattr(ct, fname).offset, (cname, fname)


def test_session_without_gpu_reports_enodev(lib, rvf):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(rvf.RVFError) as ei:
        rvf.Session(0)
    assert ei.value.status == -8


@pytest.mark.parametrize("family,code", [("quad", 0), ("tri", 1), ("line3", 4)])
@pytest.mark.parametrize("nquad", [1, 2, 3, 4, 5, 6, 8])
def test_quadrature_rules_bitwise(orc, family, code, nquad):
    from rvf_b200 import _abi
    P, W = _abi.quadrature_rule(code, nquad)
    if family == "quad":
        Po, Wo = orc.gl_2d(nquad)
    elif family == "tri":
        Po, Wo = orc.tri_rule(nquad)
    else:
        p, Wo = orc.gl_1d(nquad)
        Po = np.vstack([p, np.zeros_like(p)])
    assert P.shape == Po.shape
    assert np.array_equal(P, Po) and np.array_equal(W, Wo)


def _random_soup(rng, T, nv=3, jitter_ties=True):
    s = rng.uniform(0, 1, size=(T, nv, 3))
    if jitter_ties:  # many equal centroid keys: exercises the stable sort
        s[: T // 2, :, 0] = np.round(s[: T // 2, :, 0], 1)
    return s


@pytest.mark.parametrize("T,nv", [(1, 3), (8, 3), (9, 3), (100, 3), (1728, 3), (37, 2), (800, 2), (50000, 3),
                                  (20001, 2)])
def test_bvh_build_matches_oracle(rvf, orc, T, nv):
    from rvf_b200 import _abi
    rng = np.random.default_rng(T)
    soup = _random_soup(rng, T, nv)
    lo, hi, meta, idx = _abi.bvh_build_host(soup)
    b = orc.BVH(soup)
    lo2, hi2, meta2, idx2 = b.export()
    assert np.array_equal(lo, lo2) and np.array_equal(hi, hi2)
    assert np.array_equal(meta, meta2) and np.array_equal(idx, idx2)
    # pre-order: every interior node's left child is the next node
    for k in range(meta.shape[0]):
        if meta[k, 0] != 0:
            assert meta[k, 0] == k + 2


def test_bvh_build_with_ties_matches_oracle(rvf, orc):
    """A structured soup (many equal centroids along every axis) large enough
    for the threaded build: the stable sort keeps ties in their current order."""
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(40, family="tri3", jitter=0.0)
    soup = np.concatenate([md.group_tri_soup[g] for g in sorted(md.group_tri_soup)])
    assert soup.shape[0] >= 9000
    lo, hi, meta, idx = _abi.bvh_build_host(soup)
    lo2, hi2, meta2, idx2 = orc.BVH(soup).export()
    assert np.array_equal(meta, meta2) and np.array_equal(idx, idx2)
    assert np.array_equal(lo, lo2) and np.array_equal(hi, hi2)


def test_exceptions_do_not_cross_the_interface(rvf):
    """A C++ exception inside an entry point comes back as a status: 2^62
    primitives overflow the build's index array (std::length_error)."""
    import ctypes as C
    from rvf_b200 import _abi
    lib = _abi.load_library()
    soup = np.zeros((1, 3, 3))
    n = C.c_int64(-1)
    rc = lib.rvf_bvh_build_host(soup.ctypes.data_as(C.POINTER(C.c_double)), 3, 1 << 62, None, None, None, None,
                                C.byref(n))
    assert rc in (_abi.RVF_ENOMEM, _abi.RVF_EINTERNAL)
    assert n.value == -1
    assert "internal error" in _abi.last_error(lib) or "allocation" in _abi.last_error(lib)


def test_bvh_box_soup_matches_oracle(rvf, orc):
    from rvf_b200 import _abi
    soup = rvf.meshes.obstruction_box()
    lo, hi, meta, idx = _abi.bvh_build_host(soup)
    lo2, hi2, meta2, idx2 = orc.BVH(soup).export()
    assert meta.shape[0] == 511
    assert np.array_equal(meta, meta2) and np.array_equal(idx, idx2) and np.array_equal(lo, lo2)


def test_flatten_mirrors_build_gpu_arrays(rvf):
    md = rvf.meshes.parallel_plates(3, "quad")
    node_idx, tables = rvf.flatten(md)
    assert tables[0].shape == (18, 8) and all(t.shape[0] == 0 for f, t in enumerate(tables) if f != 0)
    assert np.array_equal(node_idx, np.arange(1, 19))
    assert np.array_equal(tables[0], md.elem_nodes)


def test_merged_obstruction_order(rvf):
    md = rvf.meshes.cube_enclosure(4, box_m=2)
    soup, g = rvf.merged_obstruction(md, [7, 2, 99])
    assert soup.shape == (48 + 32, 3, 3)
    assert np.all(g[:48] == 7) and np.all(g[48:] == 2)
    assert np.array_equal(soup[:48], md.group_tri_soup[7])


def test_obs_soups_follow_reference_layout(rvf):
    md = rvf.meshes.parallel_plates(2, "quad4")
    s = md.group_tri_soup[1]
    # quads split into (1,2,3) and (1,3,4), corner nodes (src/MeshIO.jl:660-671)
    e0 = md.elem_nodes[0] - 1
    X = md.coords.T
    assert np.array_equal(s[0], X[[e0[0], e0[1], e0[2]]])
    assert np.array_equal(s[1], X[[e0[0], e0[2], e0[3]]])


def test_hook_registry_and_guards(rvf):
    from rvf_b200 import assembly
    md = rvf.meshes.parallel_plates(2, "quad4")
    with pytest.raises(ValueError, match="cannot both be true"):
        rvf.compute_view_factors(md, use_duffy=True, monte_carlo=True, backend=rvf.B200Backend())
    with pytest.raises(NotImplementedError):
        rvf.compute_view_factors(md, backend=rvf.CPU())
    seen = {}

    def fake(mesh, nquad, backend, FloatT, ArrayT, **kw):
        seen.update(kw, nquad=nquad, FloatT=FloatT, ArrayT=ArrayT)
        return "ok"
    prev = assembly._GPU_HOOK_REF[0]
    try:
        rvf.register_gpu_hook(fake)
        assert rvf.compute_view_factors(md, nquad=3, obstruction_groups=[1], verbose=False) == "ok"
        assert seen["nquad"] == 3 and seen["obstruction_groups"] == [1] and seen["FloatT"] is np.float64
        assert seen["monte_carlo"] is False and seen["n_samples"] == 10000
        assert seen["ArrayT"] is np.ndarray
    finally:
        rvf.register_gpu_hook(prev)
    assert assembly._GPU_HOOK_REF[0] is rvf.compute_view_factors_b200


def test_unknown_backend_errors_like_reference(rvf):
    md = rvf.meshes.parallel_plates(2, "quad4")

    class Other:
        pass
    with pytest.raises(RuntimeError, match="No GPU array type registered"):
        rvf.compute_view_factors(md, backend=Other())


def test_curve_mesh_guard_for_backends_without_support(rvf):
    md = rvf.meshes.cavity_2d(4, 4, 1)
    from rvf_b200 import assembly

    class Other:
        pass
    assert not assembly._gpu_supports(Other(), "curves")
    with pytest.raises(ValueError, match="curve meshes"):
        rvf.compute_view_factors(md, backend=Other())


def test_mc_element_bound_covers_quadratic_elements():
    """The Monte Carlo classification's element radius (k_mc_bounds): corner
    radius about the corners' centroid plus the mid-side nodes' largest
    deviation from their edges' midpoints times 2 (Quad8) or 4/3 (Tri6).
    Every point of random curved elements, evaluated with the shape
    functions of shape_surface (same node order), lies inside it."""
    import numpy as np
    rng = np.random.default_rng(11)

    def quad8(x, e):
        return np.array([0.25 * (1 - x) * (1 - e) * (-x - e - 1), 0.25 * (1 + x) * (1 - e) * (x - e - 1),
                         0.25 * (1 + x) * (1 + e) * (x + e - 1), 0.25 * (1 - x) * (1 + e) * (-x + e - 1),
                         0.5 * (1 - x * x) * (1 - e), 0.5 * (1 + x) * (1 - e * e), 0.5 * (1 - x * x) * (1 + e),
                         0.5 * (1 - x) * (1 - e * e)])

    def tri6(x, e):
        l1, l2, l3 = 1 - x - e, x, e
        return np.array([l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), 4 * l1 * l2, 4 * l2 * l3,
                         4 * l1 * l3])

    fams = {"quad8": (quad8, 4, [(4, 0, 1), (5, 1, 2), (6, 2, 3), (7, 3, 0)], 2.0, np.linspace(-1, 1, 121)),
            "tri6": (tri6, 3, [(3, 0, 1), (4, 1, 2), (5, 0, 2)], 4.0 / 3.0, np.linspace(0, 1, 121))}
    for name, (shape, nc, mids, lam, g) in fams.items():
        X, E = np.meshgrid(g, g)
        if name == "tri6":
            keep = X + E <= 1
            X, E = X[keep], E[keep]
        N = shape(X.ravel(), E.ravel())
        for _ in range(200):
            nodes = np.zeros((nc + len(mids), 3))
            nodes[:nc] = rng.normal(size=(nc, 3))
            for m, a, b in mids:
                nodes[m] = 0.5 * (nodes[a] + nodes[b]) + rng.normal(size=3) * rng.uniform(0, 0.6)
            c = nodes[:nc].mean(axis=0)
            dev = max(np.linalg.norm(nodes[m] - 0.5 * (nodes[a] + nodes[b])) for m, a, b in mids)
            r = np.linalg.norm(nodes[:nc] - c, axis=1).max() + lam * dev
            pts = N.T @ nodes
            assert np.linalg.norm(pts - c, axis=1).max() <= r * (1 + 1e-12), name
