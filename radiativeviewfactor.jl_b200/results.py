"""Result container and post-processing checks (src/Results.jl)."""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from .mesh import MeshData


@dataclass
class ViewFactorResult:
    """src/Results.jl:35-42.  F_elem[i, j] is the view factor from element i to j."""

    F_elem: np.ndarray
    A_elem: np.ndarray
    F_group: np.ndarray
    A_group: np.ndarray
    group_tags: List[int]
    group_names: List[str]
    stats: dict | None = None


def _aggregate(mesh: MeshData, F_elem: np.ndarray, A_elem: np.ndarray):
    """src/Results.jl:56-82: A_g F_{g->h} = sum_{i in g} A_i sum_{j in h} F_ij."""
    tags = sorted(mesh.group_tags)
    names = [mesh.group_tags[t] for t in tags]
    G = len(tags)
    members = [np.nonzero(mesh.elem_group == t)[0] for t in tags]
    A_group = np.array([A_elem[m].sum() if len(m) else 0.0 for m in members])
    F_group = np.zeros((G, G))
    for gj, mj in enumerate(members):
        colsum = F_elem[:, mj].sum(axis=1) if len(mj) else np.zeros(F_elem.shape[0])
        for gi, mi in enumerate(members):
            F_group[gi, gj] = np.dot(A_elem[mi], colsum[mi])
    with np.errstate(invalid="ignore", divide="ignore"):
        F_group = F_group / A_group[:, None]
    return tags, names, F_group, A_group


def aggregate_by_group(result: ViewFactorResult, mesh: MeshData):
    """src/Results.jl:90-93 -> (F_group, A_group, tags, names)."""
    tags, names, Fg, Ag = _aggregate(mesh, result.F_elem, result.A_elem)
    return Fg, Ag, tags, names


def reciprocity_error(result: ViewFactorResult, block: int = 4096) -> float:
    """max_{i<j} |A_i F_ij - A_j F_ji| / max(A_i F_ij, 1e-30) (src/Results.jl:105-114)."""
    F, A = result.F_elem, result.A_elem
    N = F.shape[0]
    worst = 0.0
    for r0 in range(0, N, block):
        r1 = min(N, r0 + block)
        for c0 in range(r0, N, block):
            c1 = min(N, c0 + block)
            P = A[r0:r1, None] * F[r0:r1, c0:c1]
            Q = (A[c0:c1, None] * F[c0:c1, r0:r1]).T
            err = np.abs(P - Q) / np.maximum(P, 1e-30)
            ii = np.arange(r0, r1)[:, None]
            jj = np.arange(c0, c1)[None, :]
            err = np.where(jj > ii, err, 0.0)
            worst = max(worst, float(np.max(err)) if err.size else 0.0)
    return worst


def check_reciprocity(result: ViewFactorResult, tol: float = 1e-4) -> bool:
    """src/Results.jl:105-114."""
    err = reciprocity_error(result)
    print(f"Reciprocity max relative error: {err}")
    return err < tol


def check_closure(result: ViewFactorResult, tol: float = 1e-3) -> bool:
    """src/Results.jl:122-127."""
    row_sums = result.F_elem.sum(axis=1)
    print(f"Row sums: min={round(float(row_sums.min()), 6)}, max={round(float(row_sums.max()), 6)}")
    return float(row_sums.max()) <= 1.0 + tol
