"""Mesh data model: the Python mirror of MeshIO.MeshData / SurfaceElement
(src/MeshIO.jl:36-64) and the flattening of build_gpu_arrays
(src/GPUKernels.jl:336-412) into the C ABI's rvf_mesh_desc layout.

Conventions
-----------
* ``coords`` is (3, n_nodes) float64 in column-major (Fortran) order, column k =
  node k+1 (node ids in element connectivity are 1-based, as in the reference).
* Element indices (rows of F_elem, ``group_elems`` values) are 0-based.
* A soup is a C-contiguous float64 array of shape (n_prims, nv, 3): memory
  identical to the reference's column-major (3, nv, n_prims) soup, i.e.
  ``soup[t, v, c]`` is coordinate c of vertex v (src/MeshIO.jl:661-669).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, NamedTuple, Sequence

import numpy as np

# family symbols of src/MeshIO.jl:26-34 -> codes of src/GPUKernels.jl:344 (+ curves)
FAMILY_CODES = {"quad": 0, "tri": 1, "quad4": 2, "tri3": 3, "line3": 4, "line2": 5}
FAMILY_NAMES = {v: k for k, v in FAMILY_CODES.items()}
FAMILY_NODES = {0: 8, 1: 6, 2: 4, 3: 3, 4: 3, 5: 2}


class SurfaceElement(NamedTuple):
    """src/MeshIO.jl:36-40: node ids (1-based), physical group tag, family symbol."""

    nodes: tuple
    group: int
    family: str


@dataclass
class MeshData:
    """src/MeshIO.jl:57-64, stored as arrays.

    elem_nodes  : (N, 8) int32, 1-based node ids, zero padded
    elem_family : (N,) int8 family codes (FAMILY_CODES)
    elem_group  : (N,) int32 physical group tags
    """

    coords: np.ndarray
    elem_nodes: np.ndarray
    elem_family: np.ndarray
    elem_group: np.ndarray
    group_tags: Dict[int, str]
    group_tri_soup: Dict[int, np.ndarray] = field(default_factory=dict)
    mesh_dim: int = 2

    def __post_init__(self):
        # (3, n_nodes) column-major: node k's xyz contiguous at 3k (Julia's layout)
        self.coords = np.asfortranarray(np.asarray(self.coords, dtype=np.float64))
        if self.coords.ndim != 2 or self.coords.shape[0] != 3:
            raise ValueError("coords must be a (3, n_nodes) array")
        self.elem_nodes = np.ascontiguousarray(np.asarray(self.elem_nodes, dtype=np.int32))
        self.elem_family = np.ascontiguousarray(np.asarray(self.elem_family, dtype=np.int8))
        self.elem_group = np.ascontiguousarray(np.asarray(self.elem_group, dtype=np.int32))
        if self.elem_nodes.ndim != 2 or self.elem_nodes.shape[1] != 8:
            raise ValueError("elem_nodes must be (N, 8)")
        n = self.elem_nodes.shape[0]
        if self.elem_family.shape != (n,) or self.elem_group.shape != (n,):
            raise ValueError("elem_family / elem_group must have one entry per element")
        if self.mesh_dim not in (1, 2):
            raise ValueError(f"mesh_dim must be 1 or 2, got {self.mesh_dim}")
        self.group_tri_soup = {int(k): np.ascontiguousarray(np.asarray(v, dtype=np.float64))
                               for k, v in self.group_tri_soup.items()}

    @property
    def n_elems(self) -> int:
        return int(self.elem_nodes.shape[0])

    @property
    def surface_elems(self) -> List[SurfaceElement]:
        out = []
        for e in range(self.n_elems):
            f = int(self.elem_family[e])
            k = FAMILY_NODES[f]
            out.append(SurfaceElement(tuple(int(v) for v in self.elem_nodes[e, :k]),
                                      int(self.elem_group[e]), FAMILY_NAMES[f]))
        return out

    @property
    def group_elems(self) -> Dict[int, np.ndarray]:
        return {int(t): np.nonzero(self.elem_group == t)[0] for t in sorted(self.group_tags)}

    @classmethod
    def from_elements(cls, coords, elems: Sequence[SurfaceElement], group_tags, group_tri_soup=None,
                      mesh_dim: int = 2) -> "MeshData":
        n = len(elems)
        en = np.zeros((n, 8), dtype=np.int32)
        fam = np.zeros(n, dtype=np.int8)
        grp = np.zeros(n, dtype=np.int32)
        for e, el in enumerate(elems):
            fam[e] = FAMILY_CODES[el.family.lstrip(":")]
            en[e, :len(el.nodes)] = el.nodes
            grp[e] = el.group
        return cls(np.asarray(coords, dtype=np.float64), en, fam, grp, dict(group_tags),
                   dict(group_tri_soup or {}), mesh_dim)


def build_group_obs_soups(mesh: MeshData) -> Dict[int, np.ndarray]:
    """_build_group_obs_soups (src/MeshIO.jl:648-685): triangles (c1,c2,c3)
    (+ (c1,c3,c4) for quads) from corner nodes; segments (c1,c2) for curves."""
    soups = {}
    X = mesh.coords.T
    for tag in sorted(mesh.group_tags):
        idx = np.nonzero(mesh.elem_group == tag)[0]
        if mesh.mesh_dim == 2:
            tris = []
            for e in idx:
                c = mesh.elem_nodes[e] - 1
                tris.append((c[0], c[1], c[2]))
                if mesh.elem_family[e] in (0, 2):
                    tris.append((c[0], c[2], c[3]))
            t = np.asarray(tris, dtype=np.int64).reshape(-1, 3)
            soups[tag] = np.ascontiguousarray(X[t])  # (T, 3 vertices, 3 coords)
        else:
            c = mesh.elem_nodes[idx][:, :2] - 1
            soups[tag] = np.ascontiguousarray(X[c])  # (S, 2 endpoints, 3 coords)
    return soups


def merged_obstruction(mesh: MeshData, obstruction_groups: Sequence[int]):
    """build_flat_bvh_from_mesh (src/GPUBVH.jl:146-174): soups of the given
    groups (those present) concatenated in the given order, with a group tag
    per primitive.  Returns (soup (T, nv, 3), groups (T,)) or (None, None)."""
    parts, tags = [], []
    for g in obstruction_groups:
        s = mesh.group_tri_soup.get(int(g))
        if s is None or s.shape[0] == 0:
            continue
        parts.append(s)
        tags.append(np.full(s.shape[0], int(g), dtype=np.int32))
    if not parts:
        return None, None
    return np.ascontiguousarray(np.concatenate(parts)), np.ascontiguousarray(np.concatenate(tags))


def flatten(mesh: MeshData):
    """build_gpu_arrays (src/GPUKernels.jl:336-412): per-family node tables
    (k x n_family, column-major == (n_family, k) C-order, 1-based ids) and the
    1-based column of each element in its family table."""
    n = mesh.n_elems
    fam = mesh.elem_family
    node_idx = np.zeros(n, dtype=np.int32)
    tables = []
    for f in range(6):
        sel = np.nonzero(fam == f)[0]
        node_idx[sel] = np.arange(1, len(sel) + 1, dtype=np.int32)
        tables.append(np.ascontiguousarray(mesh.elem_nodes[sel, :FAMILY_NODES[f]].astype(np.int32)))
    bad = (fam < 0) | (fam > 5)
    if bad.any():
        raise ValueError(f"element {int(np.nonzero(bad)[0][0]) + 1}: unknown family code")
    return node_idx, tables
