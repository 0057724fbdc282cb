"""ctypes front-end of liboracle.so, the CPU restatement of the reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_p = C.c_void_p
_pd = C.POINTER(C.c_double)
_pi32 = C.POINTER(C.c_int32)
_pi64 = C.POINTER(C.c_int64)
_pi8 = C.POINTER(C.c_int8)
_pu8 = C.POINTER(C.c_uint8)


class OrcMesh(C.Structure):
    _fields_ = [("mesh_dim", C.c_int32), ("n_nodes", C.c_int64), ("coords", _pd), ("n_elems", C.c_int64),
                ("family", _pi8), ("elem_nodes", _pi32), ("elem_group", _pi32), ("n_obs", C.c_int64),
                ("obs_nv", C.c_int32), ("obs_soup", _pd), ("obs_group", _pi32)]


_SIG = {
    "orc_gl_1d": (C.c_int, [C.c_int, _pd, _pd]),
    "orc_gl_2d": (C.c_int, [C.c_int, _pd, _pd]),
    "orc_tri_rule": (C.c_int, [C.c_int, _pd, _pd]),
    "orc_quad8_shape": (None, [C.c_double, C.c_double, _pd, _pd, _pd]),
    "orc_quad4_shape": (None, [C.c_double, C.c_double, _pd, _pd, _pd]),
    "orc_tri6_shape": (None, [C.c_double, C.c_double, _pd, _pd, _pd]),
    "orc_tri3_shape": (None, [C.c_double, C.c_double, _pd, _pd, _pd]),
    "orc_line3_shape": (None, [C.c_double, _pd, _pd]),
    "orc_line2_shape": (None, [C.c_double, _pd, _pd]),
    "orc_eval_point": (None, [C.POINTER(OrcMesh), C.c_int64, C.c_double, C.c_double, C.c_int, _pd, _pd, _pd]),
    "orc_vf_kernel": (C.c_double, [_pd, _pd, _pd, _pd]),
    "orc_vf_kernel_2d": (C.c_double, [_pd, _pd, _pd, _pd]),
    "orc_bvh_build": (_p, [_pd, C.c_int32, C.c_int64]),
    "orc_bvh_free": (None, [_p]),
    "orc_bvh_n_nodes": (C.c_int64, [_p]),
    "orc_bvh_export": (None, [_p, _pd, _pd, _pi32, _pi32]),
    "orc_intersect_flat": (C.c_int, [_p, _pi32, _pd, _pd, C.c_double, C.c_int32, C.c_int32, C.c_int, _pi64]),
    "orc_intersect_ray_cpu": (C.c_int, [_p, _pd, _pd, C.c_double]),
    "orc_intersect_seg": (C.c_int, [_p, _pi32, _pd, _pd, C.c_int32, C.c_int32]),
    "orc_is_visible_cpu": (C.c_int, [_p, _pd, _pd, C.c_int]),
    "orc_solve_plain": (C.c_int, [C.POINTER(OrcMesh), C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                  _pd, _pd, _pu8, C.c_int32, _pi64]),
    "orc_solve_rows": (C.c_int, [C.POINTER(OrcMesh), C.c_int, C.c_int, _pi64, C.c_int64, C.c_int, _pd, _pd, _pi64]),
    "orc_self_gpu": (C.c_int, [C.POINTER(OrcMesh), C.c_int, C.c_int, _pd, _pd]),
    "orc_solve_mc": (C.c_int, [C.POINTER(OrcMesh), C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int64, C.c_int64,
                               C.c_int64, C.c_int, _pd, _pd, _pu8, _pi64]),
    "orc_singularity_type": (C.c_int, [C.POINTER(OrcMesh), C.c_int64, C.c_int64, _pi32, _pi32]),
    "orc_pair_duffy": (C.c_double, [C.POINTER(OrcMesh), _p, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int, _pd,
                                    C.POINTER(C.c_int)]),
    "orc_solve_cpu": (C.c_int, [C.POINTER(OrcMesh), C.c_int, C.c_int, C.c_int, _pi32, C.c_int32, C.c_int64,
                                C.c_int64, C.c_int64, C.c_int, _pd, _pd, _pi64]),
    "orc_aggregate": (None, [C.c_int64, _pd, _pd, _pi32, C.c_int32, _pi32, _pd, _pd]),
    "orc_reciprocity_error": (C.c_double, [C.c_int64, _pd, _pd]),
    "orc_row_sums": (None, [C.c_int64, _pd, _pd]),
    "orc_init_rng": (C.c_uint64, [C.c_uint64, C.c_uint64]),
    "orc_xorshift64": (C.c_double, [C.POINTER(C.c_uint64)]),
}

_lib = None
_lock = threading.Lock()


def build():
    src = [HERE / "rvf_oracle.cpp", HERE / "rvf_oracle.h", HERE / "Makefile"]
    if not LIB.exists() or LIB.stat().st_mtime < max(p.stat().st_mtime for p in src):
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return LIB


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(str(LIB))
            for k, (r, a) in _SIG.items():
                f = getattr(L, k)
                f.restype = r
                f.argtypes = a
            _lib = L
        return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _i32(a):
    return None if a is None else a.ctypes.data_as(_pi32)


class Mesh:
    """orc_mesh built from a MeshData (+ merged obstruction soup)."""

    def __init__(self, md, obstruction_groups=()):
        self.md = md
        self.coords = np.asfortranarray(md.coords, dtype=np.float64)
        self.fam = np.ascontiguousarray(md.elem_family, dtype=np.int8)
        self.en = np.ascontiguousarray(md.elem_nodes, dtype=np.int32)
        self.grp = np.ascontiguousarray(md.elem_group, dtype=np.int32)
        parts, tags = [], []
        for g in obstruction_groups:
            s = md.group_tri_soup.get(int(g))
            if s is None or s.shape[0] == 0:
                continue
            parts.append(s)
            tags.append(np.full(s.shape[0], int(g), dtype=np.int32))
        self.soup = np.ascontiguousarray(np.concatenate(parts)) if parts else None
        self.sgrp = np.ascontiguousarray(np.concatenate(tags)) if tags else None
        self.obstruction_groups = np.ascontiguousarray(np.asarray(list(obstruction_groups), dtype=np.int32))
        m = OrcMesh()
        m.mesh_dim = md.mesh_dim
        m.n_nodes = self.coords.shape[1]
        m.coords = _d(self.coords)
        m.n_elems = self.fam.shape[0]
        m.family = self.fam.ctypes.data_as(_pi8)
        m.elem_nodes = _i32(self.en)
        m.elem_group = _i32(self.grp)
        if self.soup is not None:
            m.n_obs = self.soup.shape[0]
            m.obs_nv = self.soup.shape[1]
            m.obs_soup = _d(self.soup)
            m.obs_group = _i32(self.sgrp)
        self.s = m
        self.N = int(m.n_elems)

    def ref(self):
        return C.byref(self.s)


def gl_1d(n):
    p, w = np.zeros(n), np.zeros(n)
    lib().orc_gl_1d(n, _d(p), _d(w))
    return p, w


def gl_2d(n):
    p, w = np.zeros(2 * n * n), np.zeros(n * n)
    lib().orc_gl_2d(n, _d(p), _d(w))
    return p.reshape(-1, 2).T.copy(), w


def tri_rule(nquad):
    p, w = np.zeros(2 * 13), np.zeros(13)
    k = lib().orc_tri_rule(nquad, _d(p), _d(w))
    return p[:2 * k].reshape(-1, 2).T.copy(), w[:k]


def shape(fam, xi, eta=0.0):
    N, a, b = np.zeros(8), np.zeros(8), np.zeros(8)
    L = lib()
    if fam in ("line3", "line2"):
        getattr(L, f"orc_{fam}_shape")(xi, _d(N), _d(a))
        k = 3 if fam == "line3" else 2
        return N[:k], a[:k]
    getattr(L, f"orc_{fam}_shape")(xi, eta, _d(N), _d(a), _d(b))
    k = {"quad8": 8, "quad4": 4, "tri6": 6, "tri3": 3}[fam]
    return N[:k], a[:k], b[:k]


def eval_point(mesh: Mesh, e, xi, eta=0.0):
    x, n, dA = np.zeros(3), np.zeros(3), np.zeros(1)
    lib().orc_eval_point(mesh.ref(), e, xi, eta, 0, _d(x), _d(n), _d(dA))
    return x, n, float(dA[0])


def vf_kernel(xi, ni, xj, nj, dim3=True):
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (xi, ni, xj, nj)]
    f = lib().orc_vf_kernel if dim3 else lib().orc_vf_kernel_2d
    return f(*[_d(v) for v in a])


class BVH:
    def __init__(self, soup: np.ndarray):
        self.soup = np.ascontiguousarray(soup, dtype=np.float64)
        self.h = lib().orc_bvh_build(_d(self.soup), self.soup.shape[1], self.soup.shape[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_free(self.h)
            self.h = None

    def export(self):
        M = lib().orc_bvh_n_nodes(self.h)
        lo, hi = np.zeros((M, 3)), np.zeros((M, 3))
        meta = np.zeros((M, 5), dtype=np.int32)
        idx = np.zeros(self.soup.shape[0], dtype=np.int32)
        lib().orc_bvh_export(self.h, _d(lo), _d(hi), _i32(meta), _i32(idx))
        return lo, hi, meta, idx

    def intersect_flat(self, groups, o, d, tmax, gi=0, gj=0, geometric=False):
        g = np.ascontiguousarray(groups, dtype=np.int32)
        o = np.ascontiguousarray(o, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        return bool(lib().orc_intersect_flat(self.h, _i32(g), _d(o), _d(d), tmax, gi, gj, int(geometric), None))

    def intersect_ray_cpu(self, o, d, tmax):
        o = np.ascontiguousarray(o, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        return bool(lib().orc_intersect_ray_cpu(self.h, _d(o), _d(d), tmax))

    def is_visible_cpu(self, xi, xj, mesh_dim=2):
        xi = np.ascontiguousarray(xi, dtype=np.float64)
        xj = np.ascontiguousarray(xj, dtype=np.float64)
        return bool(lib().orc_is_visible_cpu(self.h, _d(xi), _d(xj), mesh_dim))


def solve_plain(mesh: Mesh, nquad, geometric=False, row_begin=0, row_end=None, row_stride=1, threads=0,
                ray_log_pm=None):
    N = mesh.N
    raw = np.zeros((N, N), order="F")
    area = np.zeros(N)
    log = None
    pm = 0
    if ray_log_pm:
        pm = int(ray_log_pm)
        log = np.zeros(N * N * pm * pm, dtype=np.uint8)
    cnt = np.zeros(4, dtype=np.int64)
    lib().orc_solve_plain(mesh.ref(), nquad, int(geometric), row_begin, N if row_end is None else row_end,
                          row_stride, threads, _d(raw), _d(area),
                          None if log is None else log.ctypes.data_as(_pu8), pm, cnt.ctypes.data_as(_pi64))
    return raw, area, log, cnt


def solve_rows(mesh: Mesh, nquad, rows, geometric=False, threads=0):
    """raw[i, :] for each sampled element i (both i < j and j < i pairs, as
    solve_plain integrates them) without the N x N matrix: (rows x N, area)."""
    rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64))
    N = mesh.N
    out = np.zeros((rows.size, N))
    area = np.zeros(N)
    cnt = np.zeros(4, dtype=np.int64)
    lib().orc_solve_rows(mesh.ref(), nquad, int(geometric), rows.ctypes.data_as(_pi64), rows.size, threads,
                         _d(out), _d(area), cnt.ctypes.data_as(_pi64))
    return out, area, cnt


def self_gpu(mesh: Mesh, nquad, geometric=False):
    """raw[i,i] and areas of the self pairs with the GPU path's arithmetic."""
    raw = np.zeros(mesh.N)
    area = np.zeros(mesh.N)
    lib().orc_self_gpu(mesh.ref(), nquad, int(geometric), _d(raw), _d(area))
    return raw, area


def solve_mc(mesh: Mesh, n_samples, seed, exclude_groups=False, geometric=False, row_begin=0, row_end=None,
             row_stride=1, threads=0, ray_log=False):
    N = mesh.N
    raw = np.zeros((N, N), order="F")
    area = np.zeros(N)
    log = np.zeros(N * N * n_samples, dtype=np.uint8) if ray_log else None
    cnt = np.zeros(4, dtype=np.int64)
    lib().orc_solve_mc(mesh.ref(), n_samples, C.c_uint64(seed), int(exclude_groups), int(geometric), row_begin,
                       N if row_end is None else row_end, row_stride, threads, _d(raw), _d(area),
                       None if log is None else log.ctypes.data_as(_pu8), cnt.ctypes.data_as(_pi64))
    return raw, area, log, cnt


def singularity_type(mesh: Mesh, i, j):
    ci, cj = np.zeros(2, dtype=np.int32), np.zeros(2, dtype=np.int32)
    t = lib().orc_singularity_type(mesh.ref(), i, j, _i32(ci), _i32(cj))
    return t, ci, cj


def pair_duffy(mesh: Mesh, i, j, nquad, bvh: BVH | None = None, gpu_semantics=True, geometric=False):
    Ai = np.zeros(1)
    st = C.c_int()
    raw = lib().orc_pair_duffy(mesh.ref(), bvh.h if bvh else None, int(gpu_semantics), int(geometric), i, j, nquad,
                               _d(Ai), C.byref(st))
    return raw, float(Ai[0]), st.value


def solve_cpu(mesh: Mesh, nquad, use_duffy=False, self_vf=False, row_begin=0, row_end=None, row_stride=1,
              threads=0):
    N = mesh.N
    raw = np.zeros((N, N), order="F")
    area = np.zeros(N)
    cnt = np.zeros(4, dtype=np.int64)
    og = mesh.obstruction_groups
    lib().orc_solve_cpu(mesh.ref(), nquad, int(use_duffy), int(self_vf), _i32(og) if og.size else None, og.size,
                        row_begin, N if row_end is None else row_end, row_stride, threads, _d(raw), _d(area),
                        cnt.ctypes.data_as(_pi64))
    return raw, area, cnt


def aggregate(F, A, elem_group, tags):
    N = F.shape[0]
    F = np.asfortranarray(F, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    eg = np.ascontiguousarray(elem_group, dtype=np.int32)
    t = np.ascontiguousarray(tags, dtype=np.int32)
    G = t.size
    Fg = np.zeros((G, G), order="F")
    Ag = np.zeros(G)
    lib().orc_aggregate(N, _d(F), _d(A), _i32(eg), G, _i32(t), _d(Fg), _d(Ag))
    return Fg, Ag


def reciprocity_error(F, A):
    F = np.asfortranarray(F, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    return lib().orc_reciprocity_error(F.shape[0], _d(F), _d(A))


def f_from_raw(raw, area):
    """F = raw ./ A (src/GPUAssembly.jl:91)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        return raw / area[:, None]


def init_rng(seed, tid):
    return int(lib().orc_init_rng(C.c_uint64(seed), C.c_uint64(tid)))


def xorshift_stream(state, n):
    s = C.c_uint64(state)
    out = [lib().orc_xorshift64(C.byref(s)) for _ in range(n)]
    return out, int(s.value)
