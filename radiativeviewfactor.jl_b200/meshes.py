"""Seeded synthetic meshes with the shapes, sizes and node layouts of the
benchmark configurations (the reference reads meshes through Gmsh, which is
not part of this backend; these builders produce the same MeshData a Gmsh
import of those geometries would).

* parallel_plates  -- two coaxial unit squares, gap 1 (analytic F12 = 0.19982)
* cube_enclosure   -- closed unit cube, inward normals, jittered Tri3/Quad4/Quad8
* obstruction_box  -- centred box soup (obstruction-only group)
* cylinder         -- open cylinder of Quad8 with annular end caps sharing nodes
* cavity_2d        -- square cavity of Line3 with circular obstructions
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

from .mesh import FAMILY_CODES, MeshData, build_group_obs_soups


class _Nodes:
    """Node registry keyed by an integer lattice key (shared nodes get one id)."""

    def __init__(self):
        self.ids: Dict[tuple, int] = {}
        self.xyz: List[Tuple[float, float, float]] = []

    def get(self, key, make):
        i = self.ids.get(key)
        if i is None:
            self.xyz.append(make())
            i = len(self.xyz)  # 1-based
            self.ids[key] = i
        return i

    def coords(self):
        return np.asfortranarray(np.asarray(self.xyz, dtype=np.float64).reshape(-1, 3).T)


def _finish(nodes: _Nodes, elems, fams, groups, group_tags, mesh_dim=2, extra_soups=None) -> MeshData:
    en = np.zeros((len(elems), 8), dtype=np.int32)
    for e, el in enumerate(elems):
        en[e, :len(el)] = el
    m = MeshData(nodes.coords(), en, np.asarray(fams, dtype=np.int8), np.asarray(groups, dtype=np.int32),
                 dict(group_tags), {}, mesh_dim)
    soups = build_group_obs_soups(m)
    if extra_soups:
        soups.update(extra_soups)
    m.group_tri_soup = {int(k): np.ascontiguousarray(v) for k, v in soups.items()}
    return m


def _cells(family: str, c):
    """Elements of one structured cell; c(a, b) gives the node of the 2m
    sub-lattice point (2i+a, 2j+b), a, b in 0..2.  Winding follows (u, v)."""
    if family == "quad4":
        return [(c(0, 0), c(2, 0), c(2, 2), c(0, 2))]
    if family == "quad":
        return [(c(0, 0), c(2, 0), c(2, 2), c(0, 2), c(1, 0), c(2, 1), c(1, 2), c(0, 1))]
    if family == "tri3":
        return [(c(0, 0), c(2, 0), c(2, 2)), (c(0, 0), c(2, 2), c(0, 2))]
    if family == "tri":
        return [(c(0, 0), c(2, 0), c(2, 2), c(1, 0), c(2, 1), c(1, 1)),
                (c(0, 0), c(2, 2), c(0, 2), c(1, 1), c(1, 2), c(0, 1))]
    raise ValueError(f"unsupported family {family!r}")


def parallel_plates(n: int = 20, family: str = "quad4", gap: float = 1.0) -> MeshData:
    """Bottom plate z=0 (normal +z, group 1) and top plate z=gap (normal -z,
    group 2), each an n x n structured grid of the given family."""
    nodes = _Nodes()
    elems, fams, groups = [], [], []
    h = 1.0 / (2 * n)
    for g, z in ((1, 0.0), (2, gap)):
        for j in range(n):
            for i in range(n):
                def c(a, b, i=i, j=j, g=g, z=z):
                    key = (g, 2 * i + a, 2 * j + b)
                    return nodes.get(key, lambda: ((2 * i + a) * h, (2 * j + b) * h, z))
                for el in _cells(family, c):
                    if g == 2:  # reverse winding: normal -z
                        el = _reverse(family, el)
                    elems.append(el)
                    fams.append(FAMILY_CODES[family])
                    groups.append(g)
    return _finish(nodes, elems, fams, groups, {1: "bottom", 2: "top"})


def _reverse(family: str, el):
    """Reverse the winding (and so the normal) of one element, keeping every
    mid-side node between its two corners: corners 1,2,3,4 -> 1,4,3,2."""
    el = list(el)
    if family == "quad4":
        return (el[0], el[3], el[2], el[1])
    if family == "quad":
        return (el[0], el[3], el[2], el[1], el[7], el[6], el[5], el[4])
    if family == "tri3":
        return (el[0], el[2], el[1])
    if family == "tri":
        return (el[0], el[2], el[1], el[5], el[4], el[3])
    raise ValueError(family)


# faces of the unit cube: (fixed axis, value, a1, a2) with a1 x a2 = inward normal
_CUBE_FACES = [(0, 0.0, 1, 2), (0, 1.0, 2, 1), (1, 0.0, 2, 0), (1, 1.0, 0, 2), (2, 0.0, 0, 1), (2, 1.0, 1, 0)]
_FACE_NAMES = ["x0", "x1", "y0", "y1", "z0", "z1"]


def cube_enclosure(m: int = 60, family: str = "tri3", jitter: float = 0.3, seed: int = 2,
                   box: bool = True, box_edge: float = 0.3, box_m: int = 12) -> MeshData:
    """Closed unit cube with inward normals; each face an m x m grid whose
    face-interior corner nodes are jittered uniformly by +-jitter*h in-plane
    (edge nodes are shared between faces).  Tri3 splits each cell in two.
    With box=True a centred box of edge box_edge (box_m x box_m cells per face,
    Tri3) is added as obstruction-only group 7 (present in group_tri_soup,
    absent from the radiating elements)."""
    rng = np.random.default_rng(seed)
    nodes = _Nodes()
    elems, fams, groups = [], [], []
    h = 1.0 / m
    M2 = 2 * m
    corner_xyz: Dict[tuple, np.ndarray] = {}

    def lattice_key(face, u2, v2):
        ax, val, a1, a2 = _CUBE_FACES[face]
        k = [0, 0, 0]
        k[ax] = 0 if val == 0.0 else M2
        k[a1] = u2
        k[a2] = v2
        return tuple(k)

    def corner(face, iu, iv):
        key = lattice_key(face, 2 * iu, 2 * iv)
        if key not in corner_xyz:
            ax, val, a1, a2 = _CUBE_FACES[face]
            p = np.zeros(3)
            p[ax] = val
            p[a1] = iu * h
            p[a2] = iv * h
            if 0 < iu < m and 0 < iv < m and jitter > 0:
                du, dv = rng.uniform(-jitter * h, jitter * h, size=2)
                p[a1] += du
                p[a2] += dv
            corner_xyz[key] = p
        return corner_xyz[key]

    # draw jitter in a fixed order: faces, then rows, then columns
    for face in range(6):
        for iv in range(m + 1):
            for iu in range(m + 1):
                corner(face, iu, iv)

    for face in range(6):
        for jv in range(m):
            for ju in range(m):
                def c(a, b, face=face, ju=ju, jv=jv):
                    u2, v2 = 2 * ju + a, 2 * jv + b
                    key = lattice_key(face, u2, v2)

                    def make():
                        # sub-lattice point: average of the surrounding corners
                        us = [u2 // 2] if u2 % 2 == 0 else [u2 // 2, u2 // 2 + 1]
                        vs = [v2 // 2] if v2 % 2 == 0 else [v2 // 2, v2 // 2 + 1]
                        if len(us) == 2 and len(vs) == 2:  # cell centre: diagonal midpoint
                            p = 0.5 * (corner(face, us[0], vs[0]) + corner(face, us[1], vs[1]))
                        else:
                            p = np.mean([corner(face, uu, vv) for uu in us for vv in vs], axis=0)
                        return tuple(float(t) for t in p)
                    return nodes.get(key, make)
                for el in _cells(family, c):
                    elems.append(el)
                    fams.append(FAMILY_CODES[family])
                    groups.append(face + 1)
    tags = {k + 1: _FACE_NAMES[k] for k in range(6)}
    extra = {7: obstruction_box(edge=box_edge, m=box_m)} if box else None
    return _finish(nodes, elems, fams, groups, tags, extra_soups=extra)


def obstruction_box(center=(0.5, 0.5, 0.5), edge: float = 0.3, m: int = 12) -> np.ndarray:
    """Tri3 soup (6*2*m*m, 3, 3) of an axis-aligned box, reference layout."""
    lo = np.asarray(center, dtype=np.float64) - edge / 2
    tris = []
    for ax, val, a1, a2 in _CUBE_FACES:
        for jv in range(m):
            for ju in range(m):
                def p(iu, iv):
                    q = lo.copy()
                    q[ax] = lo[ax] + val * edge
                    q[a1] = lo[a1] + edge * iu / m
                    q[a2] = lo[a2] + edge * iv / m
                    return q
                c00, c10, c11, c01 = p(ju, jv), p(ju + 1, jv), p(ju + 1, jv + 1), p(ju, jv + 1)
                tris.append((c00, c10, c11))
                tris.append((c00, c11, c01))
    return np.ascontiguousarray(np.asarray(tris, dtype=np.float64))


def cylinder(nc: int = 64, na: int = 32, radius: float = 0.5, height: float = 1.0, caps: bool = True,
             cap_rings: int = 8, r_inner: float = 0.25, jitter: float = 0.01, seed: int = 3) -> MeshData:
    """Open cylinder (inner surface, normals towards the axis) of nc x na Quad8
    with mid-side nodes on the exact arcs and +-jitter radial jitter on nodes
    off the end rings; with caps, two annular Quad8 caps (cap_rings x nc,
    r in [r_inner, radius], normals into the volume) share the end-ring nodes."""
    rng = np.random.default_rng(seed)
    nodes = _Nodes()
    elems, fams, groups = [], [], []
    T2 = 2 * nc
    Z2 = 2 * na
    R2 = 2 * cap_rings

    def wall(it, iz):
        it %= T2
        key = ("w", it, iz)

        def make():
            th = math.pi * it / nc
            r = radius
            if 0 < iz < Z2 and jitter > 0:
                r = radius * (1.0 + rng.uniform(-jitter, jitter))
            return (r * math.cos(th), r * math.sin(th), height * iz / Z2)
        return nodes.get(key, make)

    def cap(which, ir, it):
        it %= T2
        if ir == R2:
            return wall(it, 0 if which == 0 else Z2)
        key = ("c", which, ir, it)

        def make():
            th = math.pi * it / nc
            rho = r_inner + (radius - r_inner) * ir / R2
            if 0 < ir < R2 and jitter > 0:
                rho *= 1.0 + rng.uniform(-jitter, jitter)
            return (rho * math.cos(th), rho * math.sin(th), 0.0 if which == 0 else height)
        return nodes.get(key, make)

    for l in range(na):
        for k in range(nc):
            t0, z0 = 2 * k, 2 * l
            el = (wall(t0, z0), wall(t0, z0 + 2), wall(t0 + 2, z0 + 2), wall(t0 + 2, z0),
                  wall(t0, z0 + 1), wall(t0 + 1, z0 + 2), wall(t0 + 2, z0 + 1), wall(t0 + 1, z0))
            elems.append(el)
            fams.append(0)
            groups.append(1)
    tags = {1: "wall"}
    if caps:
        for which, g in ((0, 2), (1, 3)):
            for a in range(cap_rings):
                for k in range(nc):
                    r0, t0 = 2 * a, 2 * k
                    if which == 0:  # normal +z
                        el = (cap(0, r0, t0), cap(0, r0 + 2, t0), cap(0, r0 + 2, t0 + 2), cap(0, r0, t0 + 2),
                              cap(0, r0 + 1, t0), cap(0, r0 + 2, t0 + 1), cap(0, r0 + 1, t0 + 2), cap(0, r0, t0 + 1))
                    else:  # normal -z
                        el = (cap(1, r0, t0), cap(1, r0, t0 + 2), cap(1, r0 + 2, t0 + 2), cap(1, r0 + 2, t0),
                              cap(1, r0, t0 + 1), cap(1, r0 + 1, t0 + 2), cap(1, r0 + 2, t0 + 1), cap(1, r0 + 1, t0))
                    elems.append(el)
                    fams.append(0)
                    groups.append(g)
        tags.update({2: "cap_bottom", 3: "cap_top"})
    return _finish(nodes, elems, fams, groups, tags)


def cavity_2d(n_wall: int = 800, n_circle: int = 200, n_circles: int = 4, r: float = 0.1, seed: int = 4,
              min_sep: float = 0.25, wall_clear: float = 0.15) -> MeshData:
    """1 x 1 square cavity of Line3 (walls traversed counter-clockwise, normals
    inward, groups 1-4) with n_circles circles of radius r (clockwise, normals
    outward, groups 5..) whose centres are drawn with rejection: >= min_sep
    apart and >= wall_clear from the walls.  mesh_dim = 1."""
    rng = np.random.default_rng(seed)
    centres = []
    while len(centres) < n_circles:
        c = rng.uniform(wall_clear, 1.0 - wall_clear, size=2)
        if all(np.hypot(*(c - d)) >= min_sep for d in centres):
            centres.append(c)
    nodes = _Nodes()
    elems, fams, groups = [], [], []
    # perimeter corner nodes, counter-clockwise from (0,0)
    per = 4 * n_wall

    def pnode(k):
        k %= per
        w, s = divmod(k, n_wall)
        t = s / n_wall
        xy = [(t, 0.0), (1.0, t), (1.0 - t, 1.0), (0.0, 1.0 - t)][w]
        return nodes.get(("p", k), lambda: (xy[0], xy[1], 0.0))

    for w in range(4):
        for s in range(n_wall):
            k = w * n_wall + s
            a, b = pnode(k), pnode(k + 1)
            xa, xb = nodes.xyz[a - 1], nodes.xyz[b - 1]
            mid = nodes.get(("pm", k), lambda: ((xa[0] + xb[0]) / 2, (xa[1] + xb[1]) / 2, 0.0))
            elems.append((a, b, mid))
            fams.append(FAMILY_CODES["line3"])
            groups.append(w + 1)
    tags = {1: "bottom", 2: "right", 3: "top", 4: "left"}
    for ci, c in enumerate(centres):
        g = 5 + ci
        tags[g] = f"circle{ci + 1}"

        def cnode(k, ci=ci, c=c):
            k %= n_circle
            th = -2.0 * math.pi * k / n_circle
            return nodes.get(("c", ci, k), lambda: (c[0] + r * math.cos(th), c[1] + r * math.sin(th), 0.0))
        for s in range(n_circle):
            a, b = cnode(s), cnode(s + 1)
            th = -2.0 * math.pi * (s + 0.5) / n_circle
            mid = nodes.get(("cm", ci, s), lambda: (c[0] + r * math.cos(th), c[1] + r * math.sin(th), 0.0))
            elems.append((a, b, mid))
            fams.append(FAMILY_CODES["line3"])
            groups.append(g)
    return _finish(nodes, elems, fams, groups, tags, mesh_dim=1)
