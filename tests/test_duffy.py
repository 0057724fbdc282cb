"""Duffy (Sauter-Schwab) integrals for Quad8 pairs sharing a vertex or an edge.

The reference's tests hold no vectors for src/DuffyKernel.jl, so the C++
oracle is pinned here against a second, independent restatement in plain
Python (same file:line citations), and the device is checked against the
oracle.  The reference's Duffy path does not reconcile the direction of a
shared edge between the two elements; its results for such pairs are not
physical view factors, and parity reproduces them as they are.
"""
import math

import numpy as np
import pytest

from conftest import load_pkg

# --------------------------------------------------------------- pure Python
CORNER_UV = [(0.0, 0.0), (1.0, 0.0), (1.0, 1.0), (0.0, 1.0)]  # src/DuffyKernel.jl:122-127


def gl1(n):
    from oracle import pyoracle as orc
    return orc.gl_1d(n)


def quad8_point(coords, nodes, xi, eta):
    """src/Geometry.jl:36-110 (point, normal, dA) in the reference's order."""
    x, e = xi, eta
    N = [((0.25 * (1 - x)) * (1 - e)) * (((-x) - e) - 1), ((0.25 * (1 + x)) * (1 - e)) * ((x - e) - 1),
         ((0.25 * (1 + x)) * (1 + e)) * ((x + e) - 1), ((0.25 * (1 - x)) * (1 + e)) * (((-x) + e) - 1),
         (0.5 * (1 - x * x)) * (1 - e), (0.5 * (1 + x)) * (1 - e * e), (0.5 * (1 - x * x)) * (1 + e),
         (0.5 * (1 - x)) * (1 - e * e)]
    dX = [(0.25 * (1 - e)) * (2 * x + e), (0.25 * (1 - e)) * (2 * x - e), (0.25 * (1 + e)) * (2 * x + e),
          (0.25 * (1 + e)) * (2 * x - e), (-x) * (1 - e), 0.5 * (1 - e * e), (-x) * (1 + e), (-0.5) * (1 - e * e)]
    dE = [(0.25 * (1 - x)) * (x + 2 * e), (0.25 * (1 + x)) * ((-x) + 2 * e), (0.25 * (1 + x)) * (x + 2 * e),
          (0.25 * (1 - x)) * ((-x) + 2 * e), (-0.5) * (1 - x * x), (-(1 + x)) * e, 0.5 * (1 - x * x),
          (-(1 - x)) * e]
    p = [0.0, 0.0, 0.0]
    a = [0.0, 0.0, 0.0]
    b = [0.0, 0.0, 0.0]
    for k in range(8):
        xa = coords[:, nodes[k] - 1]
        for c in range(3):
            p[c] = p[c] + N[k] * xa[c]
            a[c] = a[c] + dX[k] * xa[c]
            b[c] = b[c] + dE[k] * xa[c]
    cx = a[1] * b[2] - a[2] * b[1]
    cy = a[2] * b[0] - a[0] * b[2]
    cz = a[0] * b[1] - a[1] * b[0]
    d = math.sqrt((cx * cx + cy * cy) + cz * cz)
    return p, [cx / d, cy / d, cz / d], d


def vf_kernel(xi, ni, xj, nj):  # src/DuffyKernel.jl:141-151
    r = [xj[c] - xi[c] for c in range(3)]
    r2 = (r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]
    if r2 < 1e-30:
        return 0.0
    rl = math.sqrt(r2)
    h = [r[c] / rl for c in range(3)]
    ci = (ni[0] * h[0] + ni[1] * h[1]) + ni[2] * h[2]
    cj = (nj[0] * -h[0] + nj[1] * -h[1]) + nj[2] * -h[2]
    if ci <= 0.0 or cj <= 0.0:
        return 0.0
    return (ci * cj) / (math.pi * r2)


def vertex_map(region, r, a, b, c, u0i, v0i, u0j, v0j):  # :288-314
    du, dv, ds, dt = {1: (r, r * a, r * b, r * b * c), 2: (r, r * a, r * b * c, r * b),
                      3: (r * a, r, r * b, r * b * c), 4: (r * a, r, r * b * c, r * b),
                      5: (r * b, r * b * c, r, r * a), 6: (r * b * c, r * b, r, r * a),
                      7: (r * b, r * b * c, r * a, r), 8: (r * b * c, r * b, r * a, r)}[region]
    return (u0i + (du if u0i == 0.0 else -du), v0i + (dv if v0i == 0.0 else -dv),
            u0j + (ds if u0j == 0.0 else -ds), v0j + (dt if v0j == 0.0 else -dt))


def edge_map(region, r, a, b, c):  # :375-408, region 4 in its overriding form
    if region == 1:
        return (r * (1 - a * (1 - c)), r * a * b * c, r * (1 - a * (1 - c)) - r * a * (1 - b) * c + r * a * b * c,
                r * a * (1 - b) * c)
    if region == 2:
        return (r * (1 - a * b * c), r * a * c * (1 - b), r * (1 - a * b * c) + r * a * b * c - r * a * c,
                r * a * b * c)
    if region == 3:
        return (r * (1 - a * b), r * a * b * c, r * (1 - a * b) - r * a * b * (1 - c), r * a * b * (1 - c))
    if region == 4:
        return (r * (b * c + a * (1 - b * c)), r * (1 - a) * b * c, r * b * c, r * (1 - a) * b * c)
    return (r * a * c, r * (1 - a) * b * c, r * a * c * (1 - b) + r * a * b * c, r * (1 - a) * b * c)


def rotate(u, v, e):  # :423-429
    return {1: (u, v), 2: (1.0 - v, u), 3: (1.0 - u, 1.0 - v), 4: (v, 1.0 - u)}[e]


def corners_to_edge(c1, c2):  # :411-419
    a, b = min(c1, c2), max(c1, c2)
    return {(1, 2): 1, (2, 3): 2, (3, 4): 3, (1, 4): 4}.get((a, b), 1)


def duffy_python(coords, ni_, nj_, nquad):
    """element_pair_view_factor_duffy without occlusion (:452-487) for two Quad8."""
    shared_i, shared_j = [], []
    for ci in range(4):
        for cj in range(4):
            if ni_[ci] == nj_[cj]:
                shared_i.append(ci + 1)
                shared_j.append(cj + 1)
    p1, w1 = gl1(nquad)
    p01 = [(p + 1.0) / 2.0 for p in p1]
    w01 = [w / 2.0 for w in w1]
    if len(shared_i) == 1:
        regions, stype = 8, 1
    else:
        regions, stype = 5, 2
        ei, ej = corners_to_edge(shared_i[0], shared_i[1]), corners_to_edge(shared_j[0], shared_j[1])
    u0i, v0i = CORNER_UV[shared_i[0] - 1]
    u0j, v0j = CORNER_UV[shared_j[0] - 1]
    F = 0.0
    for region in range(1, regions + 1):
        for ir in range(nquad):
            for i1 in range(nquad):
                for i2 in range(nquad):
                    for i3 in range(nquad):
                        r, a, b, c = p01[ir], p01[i1], p01[i2], p01[i3]
                        if stype == 1:
                            u, v, s, t = vertex_map(region, r, a, b, c, u0i, v0i, u0j, v0j)
                        else:
                            E = edge_map(region, r, a, b, c)
                            u, v = rotate(E[0], E[1], ei)
                            s, t = rotate(E[2], E[3], ej)
                        if u < 0 or u > 1 or v < 0 or v > 1 or s < 0 or s > 1 or t < 0 or t > 1:
                            continue
                        xi, nni, dAi = quad8_point(coords, ni_, 2 * u - 1.0, 2 * v - 1.0)
                        xj, nnj, dAj = quad8_point(coords, nj_, 2 * s - 1.0, 2 * t - 1.0)
                        K = vf_kernel(xi, nni, xj, nnj)
                        if K == 0.0:
                            continue
                        jac = r * r * r
                        F += w01[ir] * w01[i1] * w01[i2] * w01[i3] * jac * K * (dAi * 4.0) * (dAj * 4.0)
    return F, stype


def small_cylinder():
    rvf = load_pkg()
    return rvf.meshes.cylinder(nc=8, na=3, cap_rings=2, jitter=0.01, seed=3)


def singular_pairs(orc, m):
    out = []
    for i in range(m.N):
        for j in range(i + 1, m.N):
            t, ci, cj = orc.singularity_type(m, i, j)
            if t:
                out.append((i, j, t))
    return out


def test_oracle_duffy_matches_python_restatement(orc):
    md = small_cylinder()
    m = orc.Mesh(md)
    pairs = singular_pairs(orc, m)
    assert any(t == 1 for *_, t in pairs) and any(t == 2 for *_, t in pairs)
    rng = np.random.default_rng(0)
    pick = [pairs[k] for k in rng.choice(len(pairs), size=10, replace=False)]
    for i, j, t in pick:
        raw, Ai, st = orc.pair_duffy(m, i, j, 3)
        ref, st2 = duffy_python(md.coords, md.elem_nodes[i], md.elem_nodes[j], 3)
        assert st == t == st2
        assert abs(raw - ref) <= 1e-12 * max(abs(ref), 1e-300), (i, j, raw, ref)


def oracle_duffy_F(orc, md, nquad, obstruction_groups=()):
    m = orc.Mesh(md, obstruction_groups)
    raw, area, _, _ = orc.solve_plain(m, nquad)
    bvh = orc.BVH(m.soup) if m.soup is not None else None
    n_sing = 0
    for i, j, t in singular_pairs(orc, m):
        r, Ai, st = orc.pair_duffy(m, i, j, nquad, bvh, gpu_semantics=True)
        raw[i, j] = raw[j, i] = r
        n_sing += 1
    return orc.f_from_raw(raw, area), area, n_sing


@pytest.mark.gpu
@pytest.mark.parametrize("nquad", [2, 3, 5])
def test_device_duffy_matches_oracle(rvf, orc, session, nquad):
    from rvf_b200 import _abi
    md = small_cylinder()
    Fo, Ao, n_sing = oracle_duffy_F(orc, md, nquad)
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, ()))
    N = md.n_elems
    F = np.empty((N, N), order="F")
    A = np.empty(N)
    st = dm.solve(rvf.make_options(nquad, use_duffy=True, seed=0), F, A)
    dm.release()
    assert st.n_duffy_pairs == n_sing
    assert np.array_equal(A, Ao)
    bad = np.abs(F - Fo) > 1e-10 * np.abs(Fo) + 1e-300
    assert not bad.any(), f"{int(bad.sum())} entries differ"


@pytest.mark.gpu
def test_device_duffy_with_obstruction(rvf, orc, session):
    from rvf_b200 import _abi
    md = rvf.meshes.cube_enclosure(3, family="quad", box_m=2, box_edge=0.5)
    Fo, Ao, n_sing = oracle_duffy_F(orc, md, 3, [7])
    assert n_sing > 0
    dm = _abi.DeviceMesh(session, rvf.mesh_desc_arrays(md, [7]))
    N = md.n_elems
    F = np.empty((N, N), order="F")
    A = np.empty(N)
    dm.solve(rvf.make_options(3, use_duffy=True, seed=0), F, A)
    dm.release()
    bad = np.abs(F - Fo) > 1e-10 * np.abs(Fo) + 1e-300
    assert not bad.any(), f"{int(bad.sum())} entries differ"
