"""ctypes binding of librvf_b200.so (include/rvf_b200.h).

This is the only way the Python host reaches the device: there is no CPU
fallback.  A missing or unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

import numpy as np

# the in-tree build; RVF_B200_LIB names another build of the same library
LIB_PATH = Path(os.environ.get("RVF_B200_LIB") or Path(__file__).resolve().parent / "lib" / "librvf_b200.so")

RVF_OK = 0
STATUS_NAMES = {0: "RVF_OK", -1: "RVF_EINVAL", -2: "RVF_ENOMEM", -3: "RVF_EBUDGET", -4: "RVF_ECUDA",
                -5: "RVF_ETIMEDOUT", -6: "RVF_ECANCELED", -7: "RVF_EUNSUPPORTED", -8: "RVF_ENODEV",
                -9: "RVF_EBUSY", -10: "RVF_ECLOSED", -11: "RVF_EINTERNAL"}
globals().update({name: code for code, name in STATUS_NAMES.items()})  # RVF_EINVAL, ...

METHOD_QUADRATURE, METHOD_MONTE_CARLO = 0, 1
FAULT_CLAIM, FAULT_ALLOC = 1, 2  # rvf_options.fault_inject test hooks
PREC_FP64, PREC_MIXED = 0, 1

_p = C.c_void_p
_pd = C.POINTER(C.c_double)
_pi32 = C.POINTER(C.c_int32)
_pi8 = C.POINTER(C.c_int8)
_pu8 = C.POINTER(C.c_uint8)


class SessionOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("n_host_threads", C.c_int32),
                ("reserved", C.c_int32 * 8)]


class MeshDesc(C.Structure):
    _fields_ = [("mesh_dim", C.c_int32), ("n_nodes", C.c_int64), ("coords", _pd), ("n_elems", C.c_int64),
                ("elem_family", _pi8), ("elem_node_idx", _pi32), ("elem_group", _pi32),
                ("nodes", _pi32 * 6), ("n_family", C.c_int64 * 6), ("n_obs", C.c_int64), ("obs_nv", C.c_int32),
                ("obs_soup", _pd), ("obs_group", _pi32), ("n_groups", C.c_int32), ("group_tags", _pi32)]


class Options(C.Structure):
    _fields_ = [("nquad", C.c_int32), ("method", C.c_int32), ("use_duffy", C.c_int32), ("n_samples", C.c_int32),
                ("seed", C.c_uint64), ("precision", C.c_int32), ("occlusion", C.c_int32),
                ("geometric_soup", C.c_int32), ("mc_exclude_groups", C.c_int32), ("near_field_factor", C.c_double),
                ("ray_log", _pu8), ("ray_log_pm", C.c_int32), ("disable_pair_lists", C.c_int32),
                ("self_vf", C.c_int32), ("disable_tile_cull", C.c_int32), ("fault_inject", C.c_int32),
                ("fast_points", C.c_int32), ("fast_row_groups", C.c_int32), ("reserved", C.c_int32 * 2)]


class Stats(C.Structure):
    _fields_ = [("ms_upload", C.c_double), ("ms_prep", C.c_double), ("ms_pairs", C.c_double),
                ("ms_duffy", C.c_double), ("ms_reduce", C.c_double), ("ms_download", C.c_double),
                ("ms_total", C.c_double), ("n_pairs", C.c_int64), ("n_point_pairs", C.c_int64),
                ("n_rays", C.c_int64), ("n_rays_fp64", C.c_int64), ("n_pairs_fp64", C.c_int64),
                ("n_duffy_pairs", C.c_int64), ("max_row_sum_dev", C.c_double),
                ("n_node_visits", C.c_int64), ("n_prim_tests", C.c_int64), ("n_kernels", C.c_int64),
                ("n_graze_fp64", C.c_int64), ("n_unsure_rays", C.c_int64), ("n_unsure_slab", C.c_int64),
                ("n_unsure_prim", C.c_int64), ("n_unsure_dir", C.c_int64), ("n_rays_traced", C.c_int64),
                ("n_chunks", C.c_int64), ("ms_gen", C.c_double), ("ms_trace", C.c_double),
                ("ms_trace_fp64", C.c_double), ("ms_resolve", C.c_double), ("n_list_pairs", C.c_int64),
                ("n_walk_pairs", C.c_int64), ("ms_lists", C.c_double), ("n_tiles_culled", C.c_int64),
                ("n_pairs_masked", C.c_int64), ("ms_cull", C.c_double),
                ("n_tiles_unclassified", C.c_int64), ("reserved", C.c_int64 * 1)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        # short names used by the bench line
        d["node_visits"] = int(self.n_node_visits)
        d["prim_tests"] = int(self.n_prim_tests)
        d["gpu_kernels"] = int(self.n_kernels)
        d["graze_point_pairs"] = int(self.n_graze_fp64)
        d["unsure_rays"] = int(self.n_unsure_rays)
        d["unsure_slab"] = int(self.n_unsure_slab)
        d["unsure_prim"] = int(self.n_unsure_prim)
        d["unsure_direction"] = int(self.n_unsure_dir)
        return d


class ServerOpts(C.Structure):
    _fields_ = [("admit_bytes", C.c_uint64), ("max_batch", C.c_int32), ("use_graphs", C.c_int32),
                ("autotune", C.c_int32), ("reserved", C.c_int32 * 8)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("n_elems", C.c_int64),
                ("footprint_bytes", C.c_uint64), ("t_submit_ms", C.c_double), ("t_admit_ms", C.c_double),
                ("t_done_ms", C.c_double), ("n_chunks", C.c_int64), ("reserved", C.c_int32 * 8)]


class TunedShape(C.Structure):
    _fields_ = [("mixed", C.c_int32), ("occlusion", C.c_int32), ("dim3", C.c_int32), ("size_class", C.c_int32),
                ("gen_blocks_per_sm", C.c_int32), ("trace_blocks_per_sm", C.c_int32), ("fast_points", C.c_int32),
                ("fast_row_groups", C.c_int32), ("rule_points", C.c_int32), ("reserved", C.c_int32),
                ("fast_ms_per_gpp", C.c_double),
                ("fast_ms_per_gpp_default", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("canceled", C.c_int64), ("in_flight", C.c_int64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("wall_ms", C.c_double),
                ("pairs_done", C.c_int64), ("chunks", C.c_int64), ("graph_replays", C.c_int64),
                ("batched_requests", C.c_int64), ("admitted_bytes_peak", C.c_uint64), ("n_tuned", C.c_int32),
                ("reserved", C.c_int32), ("ms_admit", C.c_double), ("ms_quad_chunks", C.c_double),
                ("ms_mc_chunks", C.c_double), ("ms_free", C.c_double), ("ms_idle", C.c_double),
                ("tuned", TunedShape * 8)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("reserved", "tuned")}
        d["tuned"] = [self.tuned[k].as_dict() for k in range(min(self.n_tuned, 8))]
        return d


REQ_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "canceled"}

# exported symbols and their signatures (checked by the CPU test-suite)
SIGNATURES = {
    "rvf_version": (C.c_char_p, []),
    "rvf_abi_version": (C.c_int, []),
    "rvf_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "rvf_default_options": (None, [C.POINTER(Options)]),
    "rvf_session_create": (C.c_int, [C.POINTER(SessionOpts), C.POINTER(_p)]),
    "rvf_session_destroy": (C.c_int, [_p]),
    "rvf_device_info": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "rvf_mesh_upload": (C.c_int, [_p, C.POINTER(MeshDesc), C.POINTER(_p)]),
    "rvf_mesh_release": (C.c_int, [_p, _p]),
    "rvf_mesh_n_elems": (C.c_int, [_p, C.POINTER(C.c_int64)]),
    "rvf_solve": (C.c_int, [_p, _p, C.POINTER(Options), _pd, _pd, _pd, _pd, _pd, C.POINTER(Stats)]),
    "rvf_result_copy": (C.c_int, [_p, _p, _pd, _pd]),
    "rvf_result_device": (C.c_int, [_p, C.POINTER(_pd), C.POINTER(_pd)]),
    "rvf_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_p)]),
    "rvf_host_free": (C.c_int, [_p]),
    "rvf_quadrature_rule": (C.c_int, [C.c_int32, C.c_int32, _pd, _pd, _pi32]),
    "rvf_bvh_build_host": (C.c_int, [_pd, C.c_int32, C.c_int64, _pd, _pd, _pi32, _pi32, C.POINTER(C.c_int64)]),
    "rvf_fma_peak": (C.c_int, [C.c_int32, C.c_int32, _pd]),
    "rvf_max_abs_diff": (C.c_int, [_pd, _pd, C.c_int64, _pd]),
    "rvf_solve_fp64_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                         C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rvf_server_create": (C.c_int, [_p, C.POINTER(ServerOpts), C.POINTER(_p)]),
    "rvf_server_destroy": (C.c_int, [_p]),
    "rvf_submit": (C.c_int, [_p, C.POINTER(MeshDesc), C.POINTER(Options), C.POINTER(C.c_int64)]),
    "rvf_poll": (C.c_int, [_p, C.c_int64, C.POINTER(RequestInfo)]),
    "rvf_wait": (C.c_int, [_p, C.c_int64, C.c_int64, C.POINTER(RequestInfo)]),
    "rvf_cancel": (C.c_int, [_p, C.c_int64]),
    "rvf_request_result": (C.c_int, [_p, C.c_int64, _pd, _pd, _pd, _pd, _pd]),
    "rvf_request_result_device": (C.c_int, [_p, C.c_int64, C.POINTER(_pd), C.POINTER(_pd)]),
    "rvf_wait_any": (C.c_int, [_p, C.c_int64, C.POINTER(C.c_int64)]),
    "rvf_release": (C.c_int, [_p, C.c_int64]),
    "rvf_server_stats_get": (C.c_int, [_p, C.POINTER(ServerStats)]),
}


class RVFError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None
_lib_lock = threading.Lock()


def load_library(path: str | os.PathLike | None = None):
    """Load librvf_b200.so (built in-tree by build.py) and bind its signatures."""
    global _lib
    with _lib_lock:
        if _lib is not None and path is None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise RuntimeError(f"librvf_b200.so not found at {p}; build it with radiativeviewfactor.jl_b200/build.py")
        lib = C.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if path is None:
            _lib = lib
        return lib


def last_error(lib=None) -> str:
    lib = lib or load_library()
    buf = C.create_string_buffer(4096)
    lib.rvf_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, lib=None):
    if status != RVF_OK:
        raise RVFError(status, last_error(lib))


def ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class Session:
    """One GPU, one stream (rvf_session)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = load_library()
        opts = SessionOpts(device=device, hbm_budget_bytes=hbm_budget_bytes, n_host_threads=0)
        h = _p()
        check(self.lib.rvf_session_create(C.byref(opts), C.byref(h)), self.lib)
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.rvf_session_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_info(self):
        sm = C.c_int()
        tot = C.c_uint64()
        fr = C.c_uint64()
        check(self.lib.rvf_device_info(self.handle, C.byref(sm), C.byref(tot), C.byref(fr)), self.lib)
        return {"sm_count": sm.value, "hbm_total": tot.value, "hbm_free": fr.value}


def mesh_desc(desc_arrays: dict) -> MeshDesc:
    """rvf_mesh_desc over the arrays of mesh_desc_arrays (kept alive by the caller)."""
    d = MeshDesc()
    d.mesh_dim = desc_arrays["mesh_dim"]
    d.n_nodes = desc_arrays["coords"].shape[1]
    d.coords = ptr(desc_arrays["coords"], C.c_double)
    d.n_elems = desc_arrays["elem_family"].shape[0]
    d.elem_family = ptr(desc_arrays["elem_family"], C.c_int8)
    d.elem_node_idx = ptr(desc_arrays["elem_node_idx"], C.c_int32)
    d.elem_group = ptr(desc_arrays["elem_group"], C.c_int32)
    for f in range(6):
        t = desc_arrays["nodes"][f]
        d.nodes[f] = ptr(t, C.c_int32) if t.size else None
        d.n_family[f] = t.shape[0]
    soup = desc_arrays.get("obs_soup")
    if soup is not None:
        d.n_obs = soup.shape[0]
        d.obs_nv = soup.shape[1]
        d.obs_soup = ptr(soup, C.c_double)
        d.obs_group = ptr(desc_arrays["obs_group"], C.c_int32)
    tags = desc_arrays["group_tags"]
    d.n_groups = tags.shape[0]
    d.group_tags = ptr(tags, C.c_int32)
    return d


class DeviceMesh:
    """A mesh resident on the device (rvf_mesh)."""

    def __init__(self, session: Session, desc_arrays: dict):
        self.session = session
        self.lib = session.lib
        self._keep = desc_arrays  # the library copies, but keep inputs alive during the call
        d = mesh_desc(desc_arrays)
        h = _p()
        check(self.lib.rvf_mesh_upload(session.handle, C.byref(d), C.byref(h)), self.lib)
        self.handle = h
        self.n_elems = int(d.n_elems)
        self.n_groups = int(d.n_groups)
        self._keep = None

    def release(self):
        if getattr(self, "handle", None) and self.session.handle:
            self.lib.rvf_mesh_release(self.session.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def solve(self, opts: Options, F_elem=None, A_elem=None, F_group=None, A_group=None, row_sums=None):
        st = Stats()
        check(self.lib.rvf_solve(self.session.handle, self.handle, C.byref(opts), ptr(F_elem, C.c_double),
                                 ptr(A_elem, C.c_double), ptr(F_group, C.c_double), ptr(A_group, C.c_double),
                                 ptr(row_sums, C.c_double), C.byref(st)), self.lib)
        return st

    def result_device(self):
        """Device address of the last solve's F (column-major N x N)."""
        F = _pd()
        check(self.lib.rvf_result_device(self.handle, C.byref(F), None), self.lib)
        return F

    def result_copy(self, F_elem=None, A_elem=None):
        check(self.lib.rvf_result_copy(self.session.handle, self.handle, ptr(F_elem, C.c_double),
                                       ptr(A_elem, C.c_double)), self.lib)


def bvh_build_host(soup: np.ndarray):
    """The library's host BVH build (no GPU needed): (lo, hi, meta, tri_idx)."""
    lib = load_library()
    soup = np.ascontiguousarray(soup, dtype=np.float64)
    M = C.c_int64()
    check(lib.rvf_bvh_build_host(ptr(soup, C.c_double), soup.shape[1], soup.shape[0], None, None, None, None,
                                 C.byref(M)), lib)
    lo = np.zeros((M.value, 3))
    hi = np.zeros((M.value, 3))
    meta = np.zeros((M.value, 5), dtype=np.int32)
    idx = np.zeros(soup.shape[0], dtype=np.int32)
    check(lib.rvf_bvh_build_host(ptr(soup, C.c_double), soup.shape[1], soup.shape[0], ptr(lo, C.c_double),
                                 ptr(hi, C.c_double), ptr(meta, C.c_int32), ptr(idx, C.c_int32), C.byref(M)), lib)
    return lo, hi, meta, idx


def fma_peak(device: int = 0, fp64: bool = True) -> float:
    """Measured FMA throughput of the device in TFLOP/s."""
    lib = load_library()
    t = C.c_double()
    check(lib.rvf_fma_peak(device, int(fp64), C.byref(t)), lib)
    return t.value


def max_abs_diff(a_dev, b_dev, n: int) -> float:
    """max |a - b| over n doubles at two device addresses."""
    lib = load_library()
    out = C.c_double()
    check(lib.rvf_max_abs_diff(a_dev, b_dev, n, C.byref(out)), lib)
    return out.value


def quadrature_rule(family: int, nquad: int):
    lib = load_library()
    n = C.c_int32()
    check(lib.rvf_quadrature_rule(family, nquad, None, None, C.byref(n)), lib)
    pts = np.zeros(2 * n.value)
    wts = np.zeros(n.value)
    check(lib.rvf_quadrature_rule(family, nquad, ptr(pts, C.c_double), ptr(wts, C.c_double), C.byref(n)), lib)
    return pts.reshape(-1, 2).T.copy(), wts


def default_options() -> Options:
    o = Options()
    load_library().rvf_default_options(C.byref(o))
    return o


class PinnedArray:
    """Page-locked host buffer from rvf_host_alloc, viewed as a numpy array."""

    def __init__(self, shape, dtype=np.float64, order="C"):
        self.lib = load_library()
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = _p()
        check(self.lib.rvf_host_alloc(max(self.nbytes, 1), C.byref(p)), self.lib)
        self._p = p
        buf = (C.c_char * max(self.nbytes, 1)).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape, order=order)

    def free(self):
        if self._p:
            self.array = None
            self.lib.rvf_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop on a session (rvf_server): submit
    solves as they arrive, poll / wait, copy results, release."""

    def __init__(self, session: Session, admit_bytes: int = 0, max_batch: int = 0, use_graphs: bool = True,
                 autotune: bool = True):
        self.session = session
        self.lib = session.lib
        o = ServerOpts(admit_bytes=admit_bytes, max_batch=max_batch, use_graphs=0 if use_graphs else -1,
                       autotune=0 if autotune else -1)
        h = _p()
        check(self.lib.rvf_server_create(session.handle, C.byref(o), C.byref(h)), self.lib)
        self.handle = h
        self.n_elems = {}

    def submit(self, desc_arrays: dict, opts: Options) -> int:
        d = mesh_desc(desc_arrays)
        rid = C.c_int64()
        check(self.lib.rvf_submit(self.handle, C.byref(d), C.byref(opts), C.byref(rid)), self.lib)
        self.n_elems[rid.value] = (int(d.n_elems), int(d.n_groups))
        return rid.value

    def poll(self, rid: int):
        """(state name, status, RequestInfo)."""
        info = RequestInfo()
        st = self.lib.rvf_poll(self.handle, rid, C.byref(info))
        return REQ_STATES.get(info.state, info.state), st, info

    def wait(self, rid: int, timeout_ms: int = -1) -> RequestInfo:
        info = RequestInfo()
        check(self.lib.rvf_wait(self.handle, rid, timeout_ms, C.byref(info)), self.lib)
        return info

    def wait_any(self, timeout_ms: int = -1):
        """The id of the next request to finish (in finishing order), or None at the time limit."""
        rid = C.c_int64(0)
        st = self.lib.rvf_wait_any(self.handle, timeout_ms, C.byref(rid))
        if st == RVF_ETIMEDOUT:
            return None
        check(st, self.lib)
        return int(rid.value)

    def cancel(self, rid: int):
        check(self.lib.rvf_cancel(self.handle, rid), self.lib)

    def result(self, rid: int, F=None, A=None, Fg=None, Ag=None, row_sums=None):
        N, G = self.n_elems[rid]
        F = np.empty((N, N), order="F") if F is None else F
        A = np.empty(N) if A is None else A
        Fg = np.empty((G, G), order="F") if Fg is None else Fg
        Ag = np.empty(G) if Ag is None else Ag
        check(self.lib.rvf_request_result(self.handle, rid, ptr(F, C.c_double), ptr(A, C.c_double),
                                          ptr(Fg, C.c_double), ptr(Ag, C.c_double), ptr(row_sums, C.c_double)),
              self.lib)
        return F, A, Fg, Ag

    def result_device(self, rid: int):
        """Device address of a done request's F (column-major N x N), valid until release."""
        F = _pd()
        check(self.lib.rvf_request_result_device(self.handle, rid, C.byref(F), None), self.lib)
        return F

    def release(self, rid: int):
        check(self.lib.rvf_release(self.handle, rid), self.lib)
        self.n_elems.pop(rid, None)

    def stats(self) -> dict:
        st = ServerStats()
        check(self.lib.rvf_server_stats_get(self.handle, C.byref(st)), self.lib)
        return st.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            self.lib.rvf_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
