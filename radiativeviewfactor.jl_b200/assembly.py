"""compute_view_factors and the GPU hook registry (src/Assembly.jl:64-96,
229-260), with the B200 backend registered as the hook target the way
GPUAssembly registers compute_view_factors_gpu (src/GPUAssembly.jl:111).
"""
from __future__ import annotations

import threading
import warnings
from typing import Sequence

import numpy as np

from . import _abi
from .mesh import MeshData, flatten, merged_obstruction
from .results import ViewFactorResult


class CPU:
    """Stand-in for KernelAbstractions.CPU(): the reference's own Julia CPU path."""


class B200Backend:
    """The B200 backend (one device).  Sessions are created lazily per device."""

    _sessions: dict = {}
    _lock = threading.Lock()

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.device = device
        self.hbm_budget_bytes = hbm_budget_bytes

    @property
    def session(self) -> _abi.Session:
        with B200Backend._lock:
            s = B200Backend._sessions.get(self.device)
            if s is None:
                s = _abi.Session(self.device, self.hbm_budget_bytes)
                B200Backend._sessions[self.device] = s
            return s


# backend capability registry (src/Assembly.jl:234-238, ext/RadiativeViewFactorCUDAExt.jl:11-12)
def _gpu_array_type(backend):
    if isinstance(backend, B200Backend):
        return np.ndarray
    raise RuntimeError(f"No GPU array type registered for {type(backend).__name__}. "
                       "Load CUDA.jl (for CUDABackend) or Metal.jl (for MetalBackend).")


def _gpu_float_type(backend):
    if isinstance(backend, B200Backend):
        return np.float64
    raise RuntimeError(f"No GPU float type registered for {type(backend).__name__}.")


def _gpu_supports(backend, feature: str) -> bool:
    """Capabilities beyond the reference's GPU path: Duffy pairs, curve meshes
    and self view factors (quadrature)."""
    return isinstance(backend, B200Backend) and feature in ("duffy", "curves", "self_vf")


_GPU_HOOK_REF = [None]


def register_gpu_hook(f):
    """src/Assembly.jl:260 -- the last registration wins."""
    _GPU_HOOK_REF[0] = f


def _gpu_compute_hook(mesh, nquad, backend, FloatT, ArrayT, obstruction_groups, verbose, monte_carlo, n_samples,
                      **extra):
    if _GPU_HOOK_REF[0] is None:
        raise RuntimeError("GPU compute hook not registered. Ensure GPUAssembly is loaded.")
    return _GPU_HOOK_REF[0](mesh, nquad, backend, FloatT, ArrayT, obstruction_groups=obstruction_groups,
                            verbose=verbose, monte_carlo=monte_carlo, n_samples=n_samples, **extra)


def compute_view_factors(mesh: MeshData, *, nquad: int = 4, obstruction_groups: Sequence[int] = (),
                         backend=None, self_vf: bool = False, monte_carlo: bool = False, n_samples: int = 10000,
                         rng=None, use_duffy: bool = False, verbose: bool = True, seed: int | None = None,
                         precision: str = "fp64", geometric_soup: bool = False,
                         mc_exclude_groups: bool = False) -> ViewFactorResult:
    """src/Assembly.jl:64-96.  backend defaults to B200Backend().

    Extra keywords of this backend: seed (Monte Carlo; the reference draws
    rand(UInt64)), precision ("fp64" | "mixed"), geometric_soup (read soup
    triangles by their true vertices instead of the reference's read),
    mc_exclude_groups (skip source/destination groups in MC occlusion).
    self_vf, CPU-only in the reference (its GPU hook never receives it), is
    computed on the device for quadrature solves (plain and Duffy) and, as
    the reference's GPU path does, left out for Monte Carlo (with a warning).
    """
    if backend is None:
        backend = B200Backend()
    if isinstance(backend, type):
        backend = backend()
    if use_duffy and not isinstance(backend, CPU) and not _gpu_supports(backend, "duffy"):
        warnings.warn("use_duffy is CPU-only; ignored for GPU backends.")
        use_duffy = False
    if use_duffy and monte_carlo:
        raise ValueError("use_duffy and monte_carlo cannot both be true.")
    if not isinstance(backend, CPU):
        if self_vf and (monte_carlo or not _gpu_supports(backend, "self_vf")):
            if monte_carlo and _gpu_supports(backend, "self_vf"):
                warnings.warn("self_vf with monte_carlo is CPU-only; ignored for GPU backends.")
            self_vf = False
        if mesh.mesh_dim == 1 and not _gpu_supports(backend, "curves"):
            raise ValueError("GPU backend does not support curve meshes (mesh_dim=1). "
                             "Use the CPU backend for 2D per-unit-depth view factors.")
        ArrayT = _gpu_array_type(backend)
        FloatT = _gpu_float_type(backend)
        extra = {"self_vf": True} if self_vf else {}
        return _gpu_compute_hook(mesh, nquad, backend, FloatT, ArrayT, list(obstruction_groups), verbose,
                                 monte_carlo, n_samples, use_duffy=use_duffy, seed=seed, precision=precision,
                                 geometric_soup=geometric_soup, mc_exclude_groups=mc_exclude_groups, **extra)
    raise NotImplementedError("The CPU path is the reference's own Julia implementation; this package "
                              "provides the B200 backend only.")


def mesh_desc_arrays(mesh: MeshData, obstruction_groups: Sequence[int]):
    """Arrays of rvf_mesh_desc: build_gpu_arrays + the merged obstruction soup."""
    node_idx, tables = flatten(mesh)
    soup, sgroup = merged_obstruction(mesh, obstruction_groups) if len(obstruction_groups) else (None, None)
    d = {
        "mesh_dim": int(mesh.mesh_dim),
        "coords": np.asfortranarray(mesh.coords, dtype=np.float64),
        "elem_family": np.ascontiguousarray(mesh.elem_family, dtype=np.int8),
        "elem_node_idx": np.ascontiguousarray(node_idx, dtype=np.int32),
        "elem_group": np.ascontiguousarray(mesh.elem_group, dtype=np.int32),
        "nodes": tables,
        "group_tags": np.ascontiguousarray(np.array(sorted(mesh.group_tags), dtype=np.int32)),
    }
    if soup is not None:
        d["obs_soup"] = soup
        d["obs_group"] = sgroup
    return d


def make_options(nquad=4, monte_carlo=False, n_samples=10000, use_duffy=False, seed=None, precision="fp64",
                 occlusion=True, geometric_soup=False, mc_exclude_groups=False, self_vf=False) -> _abi.Options:
    o = _abi.default_options()
    o.nquad = int(nquad)
    o.method = _abi.METHOD_MONTE_CARLO if monte_carlo else _abi.METHOD_QUADRATURE
    o.n_samples = int(n_samples)
    o.use_duffy = int(bool(use_duffy))
    if seed is None:
        seed = int(np.random.default_rng().integers(0, 2**63))
    o.seed = int(seed) & (2**64 - 1)
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")
    o.precision = _abi.PREC_FP64 if precision == "fp64" else _abi.PREC_MIXED
    o.occlusion = int(bool(occlusion))
    o.geometric_soup = int(bool(geometric_soup))
    o.mc_exclude_groups = int(bool(mc_exclude_groups))
    o.self_vf = int(bool(self_vf))
    return o


def compute_view_factors_b200(mesh: MeshData, nquad: int, backend: B200Backend, FloatT, ArrayT, *,
                              obstruction_groups=(), verbose=True, monte_carlo=False, n_samples=10000,
                              use_duffy=False, seed=None, precision="fp64", geometric_soup=False,
                              mc_exclude_groups=False, self_vf=False) -> ViewFactorResult:
    """The hook target: compute_view_factors_gpu (src/GPUAssembly.jl:32-105) on the B200 library."""
    N = mesh.n_elems
    if verbose:
        what = f"n_samples={n_samples} (Monte Carlo)" if monte_carlo else f"nquad={nquad}"
        print(f"GPU compute_view_factors: {N} elements, {what}, FloatT=Float64, backend=B200Backend")
    d = mesh_desc_arrays(mesh, obstruction_groups)
    if len(obstruction_groups) and "obs_soup" not in d:
        warnings.warn("obstruction_groups specified but no triangle geometry found for those groups; "
                      "proceeding without obstruction checking.")
    sess = backend.session
    dm = _abi.DeviceMesh(sess, d)
    try:
        tags = [int(t) for t in sorted(mesh.group_tags)]
        G = len(tags)
        F = np.empty((N, N), dtype=np.float64, order="F")
        A = np.empty(N, dtype=np.float64)
        Fg = np.empty((G, G), dtype=np.float64, order="F")
        Ag = np.empty(G, dtype=np.float64)
        rs = np.empty(N, dtype=np.float64)
        o = make_options(nquad, monte_carlo, n_samples, use_duffy, seed, precision, True, geometric_soup,
                         mc_exclude_groups, self_vf)
        st = dm.solve(o, F, A, Fg if G else None, Ag if G else None, rs if N else None)
    finally:
        dm.release()
    if verbose and N:
        print(f"  Row-sum check (element level) — max |Σⱼ Fᵢⱼ - 1| : {np.max(np.abs(rs - 1.0))}")
        if G:
            print(f"  Row-sum check (group level)   — max |Σⱼ Fᵢⱼ - 1| : {np.max(np.abs(Fg.sum(axis=1) - 1.0))}")
    return ViewFactorResult(F, A, Fg, Ag, tags, [mesh.group_tags[t] for t in tags], st.as_dict())


register_gpu_hook(compute_view_factors_b200)
