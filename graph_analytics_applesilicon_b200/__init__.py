"""graph_analytics_applesilicon_b200 -- B200 (sm_100a) BFS and PageRank.

Python access to libgraphb200.so (the C ABI of include/graph_b200.h).  The
classes mirror the reference's host interface (gpu::GpuBfs,
src/metal/bfs_gpu.hpp:35-105; gpu::GpuPageRank, src/metal/pagerank_gpu.hpp:46-127):
same method names, argument meaning and error behaviour (invalid options raise
RuntimeError, as the reference throws std::runtime_error).

There is no CPU fallback: importing works without a GPU (graph building runs
on the host), but every GPU call goes through the CUDA library and raises if it
cannot run.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgraphb200.so")
UNREACHED = 0xFFFFFFFF
FLAG_DIRECTED, FLAG_SORTED, FLAG_DEDUP = 1, 2, 4

# gb_bfs_variant / gb_strategy / gb_pr_variant (include/graph_b200.h)
BFS_VARIANTS = {"gpu_vertex": 0, "gpu_naive": 1, "gpu_binned": 2, "gpu_edge": 3, "gpu_do": 4,
                "gpu_do_persistent": 5, "hybrid": 5, "batch": 6}
STRATEGIES = ["td_ept1", "td_ept2", "td_ept4", "td_warp", "bu"]
PR_VARIANTS = {"gpu_push": 0, "gpu_pull_scalar": 1, "gpu_pull_vector": 2, "gpu_pull_adaptive": 3,
               "gpu_pull_gs": 4, "gpu_pull_f64": 5, "gpu_pull_blocked": 6}
ERRORS = {1: "invalid argument", 2: "CUDA failure", 3: "out of memory", 4: "device wait timed out",
          5: "bad state", 6: "I/O error", 7: "capacity"}


class GraphError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} [{ERRORS.get(status, status)}]")
        self.status = status


class _Csr(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("flags", C.c_uint32),
                ("row_ptr", C.POINTER(C.c_uint32)), ("col_idx", C.POINTER(C.c_uint32))]


class _ConvertStats(C.Structure):
    _fields_ = [("lines", C.c_uint64), ("raw_max_id", C.c_uint64), ("n", C.c_uint64),
                ("m_before", C.c_uint64), ("m", C.c_uint64), ("seconds", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BfsOptions(C.Structure):
    """gb_bfs_options: GpuBfsOptions (src/metal/bfs_gpu.hpp:23-33) + new fields."""
    _fields_ = [("tg", C.c_uint32), ("small_max", C.c_uint32), ("large_min", C.c_uint32),
                ("ept", C.c_uint32), ("alpha", C.c_double), ("beta", C.c_double),
                ("selector", C.c_uint32), ("force_strategy", C.c_int32), ("hub_min", C.c_uint32),
                ("block", C.c_uint32), ("spin_limit", C.c_uint64), ("grid_blocks", C.c_uint32),
                ("sel_margin", C.c_float), ("in_flight", C.c_uint32)]

    def __init__(self, **kw):
        super().__init__()
        lib().gb_bfs_default_options(C.byref(self))
        for k, v in kw.items():
            if k == "selector" and isinstance(v, str):
                v = {"rule": 0, "learned": 1}[v]
            if k == "force_strategy" and isinstance(v, str):
                v = STRATEGIES.index(v)
            setattr(self, k, v)


class Level(C.Structure):
    """gb_level: util::BfsLevel (src/util/trace.hpp:7-14) + the strategy run."""
    _fields_ = [("level", C.c_uint32), ("direction", C.c_char), ("device", C.c_char),
                ("strategy", C.c_uint8), ("pad", C.c_uint8), ("frontier", C.c_uint64),
                ("edges", C.c_uint64), ("time_ms", C.c_double)]


class PrOptions(C.Structure):
    """gb_pr_options: GpuPrOptions (src/metal/pagerank_gpu.hpp:27-36)."""
    _fields_ = [("damping", C.c_float), ("iters", C.c_int32), ("tol", C.c_double),
                ("tol_rel", C.c_double), ("tg", C.c_uint32), ("small_max", C.c_uint32),
                ("large_min", C.c_uint32), ("inplace", C.c_uint32)]

    def __init__(self, **kw):
        super().__init__()
        lib().gb_pr_default_options(C.byref(self))
        for k, v in kw.items():
            setattr(self, k, v)


class PrResult(C.Structure):
    """gb_pr_result: GpuPrResult (src/metal/pagerank_gpu.hpp:38-44)."""
    _fields_ = [("iters", C.c_int32), ("floor_stop", C.c_int32), ("last_delta", C.c_double),
                ("last_max_rel", C.c_double), ("gpu_ms", C.c_double)]


_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lib = None


def lib():
    """The CUDA library; raises (never falls back) when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run python -m graph_analytics_applesilicon_b200.build")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(_Csr)
        vp = C.c_void_p
        sig = {
            "gb_last_error": (C.c_char_p, []),
            "gb_device_info": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
            "gb_csr_free": (None, [P]),
            "gb_csr_load": (C.c_int, [C.c_char_p, P]),
            "gb_csr_save": (C.c_int, [P, C.c_char_p]),
            "gb_csr_load_pinned": (C.c_int, [C.c_char_p, P]),
            "gb_bfs_create_from_file": (C.c_int, [C.c_char_p, vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "gb_csr_validate": (C.c_int, [P, C.c_char_p, C.c_size_t]),
            "gb_csr_from_edges": (C.c_int, [C.c_uint64, _u32p, _u32p, C.c_uint64, C.c_int, P]),
            "gb_csr_transpose": (C.c_int, [P, P]),
            "gb_csr_symmetrize": (C.c_int, [P, P]),
            "gb_csr_permute": (C.c_int, [P, _u32p, P]),
            "gb_csr_from_edges_gpu": (C.c_int, [C.c_uint64, _u32p, _u32p, C.c_uint64, C.c_int, P]),
            "gb_csr_transpose_gpu": (C.c_int, [P, P]),
            "gb_csr_symmetrize_gpu": (C.c_int, [P, P]),
            "gb_csr_permute_gpu": (C.c_int, [P, _u32p, P]),
            "gb_pick_sources_gpu": (C.c_int, [P, C.c_int, C.c_uint64, C.c_int, _u32p, C.POINTER(C.c_int)]),
            "gb_csr_from_snap_gpu": (C.c_int, [C.c_char_p, C.c_int, C.c_uint64, P, C.POINTER(_ConvertStats)]),
            "gb_convert_snap_gpu": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(_ConvertStats)]),
            "gb_random_perm": (C.c_int, [C.c_uint64, C.c_uint64, _u32p]),
            "gb_reorder": (C.c_int, [P, C.c_char_p, C.c_uint64, _u32p]),
            "gb_reorder_gpu": (C.c_int, [P, C.c_char_p, C.c_uint64, _u32p]),
            "gb_csr_hub_first_gpu": (C.c_int, [P, P]),
            "gb_locality": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "gb_gen_path": (C.c_int, [C.c_uint32, P]),
            "gb_gen_star": (C.c_int, [C.c_uint32, P]),
            "gb_gen_complete": (C.c_int, [C.c_uint32, P]),
            "gb_gen_two_components": (C.c_int, [P]),
            "gb_gen_empty": (C.c_int, [C.c_uint32, P]),
            "gb_gen_grid2d": (C.c_int, [C.c_uint32, C.c_uint32, P]),
            "gb_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint64, C.c_int, C.c_uint64, P]),
            "gb_gen_road": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint64, P]),
            "gb_gen_web": (C.c_int, [C.c_uint32, C.c_double, C.c_double, C.c_uint64, P]),
            "gb_gen_chung_lu": (C.c_int, [C.c_uint32, C.c_double, C.c_double, C.c_uint64, P]),
            "gb_pick_sources": (C.c_int, [P, C.c_int, C.c_uint64, C.c_int, _u32p, C.POINTER(C.c_int)]),
            "gb_bfs_default_options": (None, [C.POINTER(BfsOptions)]),
            "gb_bfs_create": (C.c_int, [_u32p, _u32p, C.c_uint64, C.c_uint64, C.POINTER(vp)]),
            "gb_bfs_destroy": (C.c_int, [vp]),
            "gb_bfs_run": (C.c_int, [vp, C.c_int, C.c_uint32, vp, C.POINTER(BfsOptions), vp, C.c_size_t,
                                     C.POINTER(C.c_size_t)]),
            "gb_bfs_run_batch": (C.c_int, [vp, _u32p, C.c_int, vp, C.POINTER(BfsOptions), vp, C.c_size_t,
                                           C.POINTER(C.c_size_t)]),
            "gb_bfs_run_many": (C.c_int, [vp, C.c_int, _u32p, C.c_uint32, vp, C.c_uint64, C.POINTER(BfsOptions),
                                          vp, vp]),
            "gb_bfs_last_gpu_ms": (C.c_double, [vp]),
            "gb_bfs_last_levels": (C.c_uint32, [vp]),
            "gb_bfs_device_dist": (vp, [vp]),
            "gb_bfs_stream": (vp, [vp]),
            "gb_selector_shape": (C.c_int, [C.POINTER(C.c_int)] * 3),
            "gb_selector_param_count": (C.c_size_t, []),
            "gb_bfs_set_selector": (C.c_int, [vp, C.c_int, vp, C.c_size_t]),
            "gb_bfs_hub_first": (C.c_int, [vp]),
            "gb_bfs_graph": (C.c_int, [vp, P]),
            "gb_bfs_profile_levels": (C.c_int, [vp, C.c_uint32, C.POINTER(BfsOptions), C.c_int, _f32p, _f32p,
                                                C.c_size_t, C.POINTER(C.c_size_t)]),
            "gb_bfs_profile_batch_levels": (C.c_int, [vp, _u32p, C.c_int, C.POINTER(BfsOptions), C.c_int, _f32p,
                                                      _f32p, C.c_size_t, C.POINTER(C.c_size_t)]),
            "gb_bfs_autotune": (C.c_int, [vp, C.c_int, _u32p, C.c_int, C.POINTER(BfsOptions)]),
            "gb_mlp_loss_grad": (C.c_int, [_f32p, C.c_int, _f32p, _f32p, _f32p, _f32p, C.POINTER(C.c_double)]),
            "gb_mlp_forward": (C.c_int, [_f32p, C.c_int, _f32p, _f32p]),
            "gb_mlp_train": (C.c_int, [_f32p, C.c_int, _f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_float,
                                       C.c_uint64, C.POINTER(C.c_float)]),
            "gb_pr_default_options": (None, [C.POINTER(PrOptions)]),
            "gb_pr_create": (C.c_int, [C.c_uint64, vp, vp, C.c_uint64, vp, vp, C.c_uint64, _u32p, C.POINTER(vp)]),
            "gb_pr_destroy": (C.c_int, [vp]),
            "gb_pr_prepare_adaptive": (C.c_int, [vp, C.c_uint32, C.c_uint32]),
            "gb_pr_prepare_gs": (C.c_int, [vp, C.c_uint32]),
            "gb_pr_gs_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "gb_pr_run": (C.c_int, [vp, C.c_int, C.POINTER(PrOptions), C.POINTER(PrResult)]),
            "gb_pr_ranks": (C.c_int, [vp, _f32p]),
            "gb_pr_ranks_f64": (C.c_int, [vp, _f64p]),
            "gb_pr_autotune": (C.c_int, [vp, C.POINTER(PrOptions)]),
            "gb_pr_stream": (vp, [vp]),
            "gb_prim_scan": (C.c_int, [_u32p, C.c_uint64, _u32p, C.POINTER(C.c_uint32)]),
            "gb_prim_scan_device_noalloc": (C.c_int, [vp, C.c_uint64, vp, vp, vp, vp]),
            "gb_prim_reduce": (C.c_int, [_u32p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "gb_prim_queue_bitmap": (C.c_int, [_u32p, C.c_uint64, C.c_uint64, _u32p, _u32p,
                                               C.POINTER(C.c_uint64)]),
            "gb_debug_barrier_timeout": (C.c_int, [C.c_uint64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise GraphError(status, lib().gb_last_error().decode(errors="replace"))


# ------------------------------------------------------------------ graphs

@dataclass
class Graph:
    """Host CSR (graph::CSR, src/graph/csr.hpp:29-45) as numpy arrays."""
    n: int
    m: int
    flags: int
    row_ptr: np.ndarray
    col_idx: np.ndarray

    @property
    def directed(self) -> bool:
        return bool(self.flags & FLAG_DIRECTED)

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr).astype(np.uint32)

    def degree(self, v: int) -> int:
        return int(self.row_ptr[v + 1] - self.row_ptr[v])

    def _c(self) -> _Csr:
        self._rp = np.ascontiguousarray(self.row_ptr, dtype=np.uint32)
        self._ci = np.ascontiguousarray(self.col_idx if self.m else np.zeros(1, np.uint32), dtype=np.uint32)
        return _Csr(self.n, self.m, self.flags, self._rp.ctypes.data_as(C.POINTER(C.c_uint32)),
                    self._ci.ctypes.data_as(C.POINTER(C.c_uint32)))

    def equal(self, o) -> bool:
        return (self.n == o.n and self.m == o.m and self.flags == o.flags
                and np.array_equal(self.row_ptr, o.row_ptr) and np.array_equal(self.col_idx[: self.m], o.col_idx[: o.m]))


def _take(c: _Csr) -> Graph:
    n, m = int(c.n), int(c.m)
    rp = np.ctypeslib.as_array(c.row_ptr, shape=(n + 1,)).copy()
    ci = np.ctypeslib.as_array(c.col_idx, shape=(m,)).copy() if m else np.zeros(0, np.uint32)
    g = Graph(n, m, int(c.flags), rp, ci)
    lib().gb_csr_free(C.byref(c))
    return g


def _make(fn, *args) -> Graph:
    out = _Csr()
    check(fn(*args, C.byref(out)))
    return _take(out)


class gen:
    """Generators (src/graph/generators.cpp) plus the benchmark-shaped graphs."""

    @staticmethod
    def path(n): return _make(lib().gb_gen_path, n)

    @staticmethod
    def star(leaves): return _make(lib().gb_gen_star, leaves)

    @staticmethod
    def complete(n): return _make(lib().gb_gen_complete, n)

    @staticmethod
    def two_components(): return _make(lib().gb_gen_two_components)

    @staticmethod
    def empty(n): return _make(lib().gb_gen_empty, n)

    @staticmethod
    def grid2d(rows, cols): return _make(lib().gb_gen_grid2d, rows, cols)

    @staticmethod
    def rmat(scale, edgefactor=None, directed=False, seed=1, edges=None):
        e = edges if edges is not None else (edgefactor << scale)
        return _make(lib().gb_gen_rmat, scale, e, int(directed), seed)

    @staticmethod
    def road(rows, cols, drop_frac=0.04, diag_frac=0.005, seed=1400):
        return _make(lib().gb_gen_road, rows, cols, drop_frac, diag_frac, seed)

    @staticmethod
    def web(n, out_mean=5.8, zipf_s=2.1, seed=875):
        return _make(lib().gb_gen_web, n, out_mean, zipf_s, seed)

    @staticmethod
    def chung_lu(n, gamma=2.2, mean_deg=76.0, seed=307):
        return _make(lib().gb_gen_chung_lu, n, gamma, mean_deg, seed)

    @staticmethod
    def suite() -> list:
        """The reference's eight test graphs (src/graph/generators.cpp:77-88)."""
        return [("path1000", gen.path(1000)), ("star100k", gen.star(100000)),
                ("complete200", gen.complete(200)), ("two_components", gen.two_components()),
                ("empty1000", gen.empty(1000)), ("grid100x100", gen.grid2d(100, 100)),
                ("rmat12", gen.rmat(12, 16, False, 42)), ("rmat12_directed", gen.rmat(12, 16, True, 43))]


def from_edges(n, eu, ev, directed=False) -> Graph:
    eu = np.ascontiguousarray(eu, np.uint32)
    ev = np.ascontiguousarray(ev, np.uint32)
    k = eu.size
    if k == 0:
        eu = ev = np.zeros(1, np.uint32)
    return _make(lib().gb_csr_from_edges, n, eu, ev, k, int(directed))


def transpose(g: Graph) -> Graph:
    return _make(lib().gb_csr_transpose, C.byref(g._c()))


def symmetrize(g: Graph) -> Graph:
    return _make(lib().gb_csr_symmetrize, C.byref(g._c()))


def permute(g: Graph, perm) -> Graph:
    return _make(lib().gb_csr_permute, C.byref(g._c()), np.ascontiguousarray(perm, np.uint32))


# The same operations on the GPU (gb_csr_*_gpu): identical results.
def from_edges_gpu(n, eu, ev, directed=False) -> Graph:
    eu = np.ascontiguousarray(eu, np.uint32)
    ev = np.ascontiguousarray(ev, np.uint32)
    k = eu.size
    if k == 0:
        eu = ev = np.zeros(1, np.uint32)
    return _make(lib().gb_csr_from_edges_gpu, n, eu, ev, k, int(directed))


def transpose_gpu(g: Graph) -> Graph:
    return _make(lib().gb_csr_transpose_gpu, C.byref(g._c()))


def symmetrize_gpu(g: Graph) -> Graph:
    return _make(lib().gb_csr_symmetrize_gpu, C.byref(g._c()))


def permute_gpu(g: Graph, perm) -> Graph:
    return _make(lib().gb_csr_permute_gpu, C.byref(g._c()), np.ascontiguousarray(perm, np.uint32))


def from_snap_gpu(path: str, directed: bool, chunk_bytes: int = 0) -> tuple[Graph, dict]:
    """SNAP edge-list text (plain or gzip) -> (CSR, stats), parsed on the GPU
    (graph::convertSnap without the file write, src/graph/snap.cpp:85-149)."""
    st, out = _ConvertStats(), _Csr()
    check(lib().gb_csr_from_snap_gpu(os.fsencode(path), int(directed), chunk_bytes, C.byref(out), C.byref(st)))
    return _take(out), st.as_dict()


def convert_snap_gpu(in_path: str, out_path: str, directed: bool) -> dict:
    """gconvert: SNAP text -> .bin (src/graph/convert.cpp:11-45); returns the stats."""
    st = _ConvertStats()
    check(lib().gb_convert_snap_gpu(os.fsencode(in_path), os.fsencode(out_path), int(directed), C.byref(st)))
    return st.as_dict()


def reorder(g: Graph, ordering: str, seed: int = 1) -> np.ndarray:
    """reorder::compute on a symmetric graph (host): perm[old] = new."""
    p = np.zeros(max(g.n, 1), np.uint32)
    check(lib().gb_reorder(C.byref(g._c()), ordering.encode(), seed, p))
    return p[: g.n]


def reorder_gpu(g: Graph, ordering: str, seed: int = 1) -> np.ndarray:
    """reorder with "degree" / "rcm" computed on the GPU (same permutation)."""
    p = np.zeros(max(g.n, 1), np.uint32)
    check(lib().gb_reorder_gpu(C.byref(g._c()), ordering.encode(), seed, p))
    return p[: g.n]


def hub_first_gpu(g: Graph) -> Graph:
    """Adjacency lists by descending neighbour degree, ties by id (GPU)."""
    return _make(lib().gb_csr_hub_first_gpu, C.byref(g._c()))


def locality(g: Graph) -> tuple[float, float]:
    """(mean |u - v|, fraction of entries within one 64-vertex block)."""
    a, b = C.c_double(0), C.c_double(0)
    check(lib().gb_locality(C.byref(g._c()), C.byref(a), C.byref(b)))
    return a.value, b.value


def random_perm(n: int, seed: int = 1) -> np.ndarray:
    p = np.zeros(max(n, 1), np.uint32)
    check(lib().gb_random_perm(n, seed, p))
    return p[:n]


def load(path: str) -> Graph:
    return _make(lib().gb_csr_load, path.encode())


def load_pinned(path: str) -> Graph:
    """graph::load into page-locked memory (returned here as numpy copies; C
    callers keep the pinned arrays and upload them at full PCIe speed)."""
    return _make(lib().gb_csr_load_pinned, path.encode())


def save(g: Graph, path: str) -> None:
    check(lib().gb_csr_save(C.byref(g._c()), path.encode()))


def validate(g: Graph) -> str:
    buf = C.create_string_buffer(256)
    check(lib().gb_csr_validate(C.byref(g._c()), buf, 256))
    return buf.value.decode()


def pick_sources(g: Graph, count=64, seed=1, any_component=False) -> np.ndarray:
    out = np.zeros(max(count, 1), np.uint32)
    k = C.c_int(0)
    check(lib().gb_pick_sources(C.byref(g._c()), count, seed, int(any_component), out, C.byref(k)))
    return out[: k.value]


def pick_sources_gpu(g: Graph, count=64, seed=1, any_component=False) -> np.ndarray:
    """pick_sources with the largest component found on the GPU (same result)."""
    out = np.zeros(max(count, 1), np.uint32)
    k = C.c_int(0)
    check(lib().gb_pick_sources_gpu(C.byref(g._c()), count, seed, int(any_component), out, C.byref(k)))
    return out[: k.value]


# --------------------------------------------------------------------- BFS

def _levels(buf, k):
    return [{"level": buf[i].level, "direction": buf[i].direction.decode(), "device": buf[i].device.decode(),
             "strategy": STRATEGIES[buf[i].strategy] if buf[i].strategy < len(STRATEGIES) else "?",
             "frontier": buf[i].frontier, "edges": buf[i].edges, "time_ms": buf[i].time_ms} for i in range(k)]


class GpuBfs:
    """gpu::GpuBfs (src/metal/bfs_gpu.hpp:35-105): one upload of a symmetric CSR."""

    @classmethod
    def from_file(cls, path: str) -> "GpuBfs":
        """A handle whose graph streams from a symmetric .bin file straight
        into GPU memory (gb_bfs_create_from_file)."""
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        n, m = C.c_uint64(0), C.c_uint64(0)
        check(lib().gb_bfs_create_from_file(os.fsencode(path), C.byref(self._h), C.byref(n), C.byref(m)))
        self.n, self.m = n.value, m.value
        return self

    def __init__(self, g: Graph):
        self.n, self.m = g.n, g.m
        self._h = C.c_void_p()
        ci = g.col_idx if g.m else np.zeros(1, np.uint32)
        check(lib().gb_bfs_create(np.ascontiguousarray(g.row_ptr, np.uint32), np.ascontiguousarray(ci, np.uint32),
                                  g.n, g.m, C.byref(self._h)))

    def close(self):
        if self._h:
            lib().gb_bfs_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, variant, source: int, out=None, opts: BfsOptions | None = None, trace=False):
        """Runs one variant; returns dist (uint32[n]) or (dist, levels) when trace."""
        v = BFS_VARIANTS[variant] if isinstance(variant, str) else int(variant)
        o = opts if opts is not None else BfsOptions()
        if out is None:
            out = np.empty(self.n, np.uint32)
        cap = self.n + 8 if trace else 0
        buf = (Level * cap)() if trace else None
        nlev = C.c_size_t(0)
        check(lib().gb_bfs_run(self._h, v, source, out.ctypes.data, C.byref(o), C.cast(buf, C.c_void_p) if trace else None,
                               cap, C.byref(nlev)))
        return (out, _levels(buf, nlev.value)) if trace else out

    # reference names (src/metal/bfs_gpu.hpp:43-66)
    def runVertex(self, s, out=None, opts=None, trace=False): return self.run("gpu_vertex", s, out, opts, trace)
    def runNaive(self, s, out=None, opts=None, trace=False): return self.run("gpu_naive", s, out, opts, trace)
    def runBinned(self, s, out=None, opts=None, trace=False): return self.run("gpu_binned", s, out, opts, trace)
    def runEdge(self, s, out=None, opts=None, trace=False): return self.run("gpu_edge", s, out, opts, trace)
    def runDO(self, s, out=None, opts=None, trace=False): return self.run("gpu_do", s, out, opts, trace)
    def runPersistent(self, s, out=None, opts=None, trace=False): return self.run("gpu_do_persistent", s, out, opts, trace)
    def runHybrid(self, s, out=None, opts=None, trace=False): return self.run("hybrid", s, out, opts, trace)

    def run_batch(self, sources, out=None, opts: BfsOptions | None = None, trace=False):
        """64-source batched BFS in one launch; returns uint32[k, n] (source-major)."""
        src = np.ascontiguousarray(sources, np.uint32)
        o = opts if opts is not None else BfsOptions()
        if out is None:
            out = np.empty((src.size, self.n), np.uint32)
        cap = 4 * self.n + 8 if trace else 0
        buf = (Level * cap)() if trace else None
        nlev = C.c_size_t(0)
        check(lib().gb_bfs_run_batch(self._h, src, src.size, out.ctypes.data, C.byref(o),
                                     C.cast(buf, C.c_void_p) if trace else None, cap, C.byref(nlev)))
        return (out, _levels(buf, nlev.value)) if trace else out

    def run_many(self, variant, sources, out=None, stride=None, opts: BfsOptions | None = None, device=False):
        """One traversal per source in one call (gb_bfs_run_many); returns
        (depths, gpu_ms[k], levels[k]).  depths: uint32[k, n] (out, or a new
        array), or out itself when stride is 0 (it ends with the last source's
        depths); device=True keeps every result on the GPU (depths None)."""
        v = BFS_VARIANTS[variant] if isinstance(variant, str) else int(variant)
        src = np.ascontiguousarray(sources, np.uint32)
        o = opts if opts is not None else BfsOptions()
        ms = np.zeros(src.size, np.float32)
        lv = np.zeros(src.size, np.uint32)
        if device:
            out, stride, ptr = None, 0, None
        else:
            if out is None:
                out = np.empty((src.size, self.n), np.uint32)
            if stride is None:
                stride = self.n if out.size >= src.size * self.n else 0
            need = (src.size - 1) * stride + self.n if src.size else 0
            if out.dtype != np.uint32 or not out.flags.c_contiguous or out.size < need:
                raise ValueError(f"out must be a contiguous uint32 array of at least {need} entries")
            ptr = out.ctypes.data
        check(lib().gb_bfs_run_many(self._h, v, src, src.size, ptr, stride, C.byref(o), ms.ctypes.data,
                                    lv.ctypes.data))
        return out, ms, lv

    def lastGpuMs(self) -> float:
        return lib().gb_bfs_last_gpu_ms(self._h)

    def lastLevels(self) -> int:
        return lib().gb_bfs_last_levels(self._h)

    def graph(self) -> Graph:
        """GpuBfs::graph(): the traversed graph, copied back from the device."""
        return _make(lib().gb_bfs_graph, self._h)

    def hub_first(self):
        """Hub-first adjacency order on the device: same depths, bottom-up
        levels exit earlier (trace edges of bottom-up levels follow it)."""
        check(lib().gb_bfs_hub_first(self._h))
        return self

    def set_selector(self, params, which: int = 0):
        if params is None:
            check(lib().gb_bfs_set_selector(self._h, which, None, 0))
            return
        p = np.ascontiguousarray(params, np.float32)
        check(lib().gb_bfs_set_selector(self._h, which, p.ctypes.data, p.size))

    def profile_levels(self, source: int, opts: BfsOptions | None = None, repeats: int = 3):
        nf = selector_shape()[0]
        cap = 4096
        feats = np.zeros((cap, nf), np.float32)
        times = np.zeros((cap, len(STRATEGIES)), np.float32)
        rows = C.c_size_t(0)
        o = opts if opts is not None else BfsOptions()
        check(lib().gb_bfs_profile_levels(self._h, source, C.byref(o), repeats, feats, times, cap, C.byref(rows)))
        return feats[: rows.value], times[: rows.value]

    def profile_batch_levels(self, sources, opts: BfsOptions | None = None, repeats: int = 3):
        nf = selector_shape()[0]
        cap = 1 << 16
        feats = np.zeros((cap, nf), np.float32)
        times = np.zeros((cap, len(STRATEGIES)), np.float32)
        rows = C.c_size_t(0)
        src = np.ascontiguousarray(sources, np.uint32)
        o = opts if opts is not None else BfsOptions()
        check(lib().gb_bfs_profile_batch_levels(self._h, src, src.size, C.byref(o), repeats, feats, times, cap,
                                                C.byref(rows)))
        return feats[: rows.value], times[: rows.value]

    def autotune(self, variant, sources, opts: BfsOptions | None = None) -> BfsOptions:
        o = opts if opts is not None else BfsOptions()
        v = BFS_VARIANTS[variant] if isinstance(variant, str) else int(variant)
        src = np.ascontiguousarray(sources, np.uint32)
        check(lib().gb_bfs_autotune(self._h, v, src, src.size, C.byref(o)))
        return o


def selector_shape():
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    lib().gb_selector_shape(C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def selector_param_count() -> int:
    return int(lib().gb_selector_param_count())


def default_selector_params(which: str = "single") -> np.ndarray | None:
    """Trained selector weights shipped with the package (None if absent)."""
    path = os.path.join(PKG, f"selector_{which}.npy")
    return np.load(path).astype(np.float32) if os.path.exists(path) else None


# ---------------------------------------------------------------- PageRank

class GpuPageRank:
    """gpu::GpuPageRank (src/metal/pagerank_gpu.hpp:46-127)."""

    def __init__(self, n: int, out_graph: Graph | None, in_graph: Graph | None, outdeg: np.ndarray):
        self.n = n
        self._h = C.c_void_p()
        self._keep = []

        def arr(g, which):
            if g is None:
                return None, 0
            a = np.ascontiguousarray(g.row_ptr if which == 0 else (g.col_idx if g.m else np.zeros(1, np.uint32)),
                                     np.uint32)
            self._keep.append(a)
            return a.ctypes.data, g.m

        orp, om = arr(out_graph, 0)
        oci, _ = arr(out_graph, 1)
        irp, im = arr(in_graph, 0)
        ici, _ = arr(in_graph, 1)
        od = np.ascontiguousarray(outdeg, np.uint32)
        check(lib().gb_pr_create(n, orp, oci, om, irp, ici, im, od if od.size else np.zeros(1, np.uint32),
                                 C.byref(self._h)))
        self._keep = []

    def close(self):
        if self._h:
            lib().gb_pr_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prepareAdaptive(self, small_max=16, large_min=256):
        check(lib().gb_pr_prepare_adaptive(self._h, small_max, large_min))

    def prepareGS(self, pair_max_outdeg=2):
        check(lib().gb_pr_prepare_gs(self._h, pair_max_outdeg))

    def gs_info(self):
        c, s, d = C.c_int(), C.c_uint64(), C.c_uint64()
        check(lib().gb_pr_gs_info(self._h, C.byref(c), C.byref(s), C.byref(d)))
        return bool(c.value), s.value, d.value

    def gsColored(self): return self.gs_info()[0]
    def gsSets(self): return self.gs_info()[1]
    def gsDeferred(self): return self.gs_info()[2]

    def run(self, variant, opts: PrOptions | None = None) -> PrResult:
        v = PR_VARIANTS[variant] if isinstance(variant, str) else int(variant)
        o = opts if opts is not None else PrOptions()
        r = PrResult()
        check(lib().gb_pr_run(self._h, v, C.byref(o), C.byref(r)))
        return r

    def ranks(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.float32)
        check(lib().gb_pr_ranks(self._h, out))
        return out[: self.n]

    def ranks_f64(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.float64)
        check(lib().gb_pr_ranks_f64(self._h, out))
        return out[: self.n]

    def autotune(self, opts: PrOptions | None = None) -> PrOptions:
        o = opts if opts is not None else PrOptions()
        check(lib().gb_pr_autotune(self._h, C.byref(o)))
        return o


def pagerank_handle(g: Graph, need_out=True, need_in=True) -> GpuPageRank:
    """Builds the handle the way gbench's runPr does (src/bench/main.cpp:499-511)."""
    gin = (transpose(g) if g.directed else g) if need_in else None
    return GpuPageRank(g.n, g if need_out else None, gin, g.degrees())


# -------------------------------------------------------- primitives / misc

def prim_scan(x: np.ndarray):
    x = np.ascontiguousarray(x, np.uint32)
    out = np.zeros(max(x.size, 1), np.uint32)
    tot = C.c_uint32(0)
    check(lib().gb_prim_scan(x if x.size else np.zeros(1, np.uint32), x.size, out, C.byref(tot)))
    return out[: x.size], tot.value


def prim_scan_device_noalloc(in_ptr: int, n: int, out_ptr: int, total_ptr: int = 0, flag_ptr: int = 0,
                             stream: int = 0):
    """Exclusive scan of n uint32 at device address in_ptr into out_ptr, with
    no device allocation (gb_prim_scan_device_noalloc); only enqueues on
    stream.  Pointers are plain device addresses (0 = none)."""
    check(lib().gb_prim_scan_device_noalloc(in_ptr or None, n, out_ptr or None, total_ptr or None,
                                            flag_ptr or None, stream or None))


def prim_reduce(x: np.ndarray):
    x = np.ascontiguousarray(x, np.uint32)
    s, m = C.c_uint32(0), C.c_uint32(0)
    check(lib().gb_prim_reduce(x if x.size else np.zeros(1, np.uint32), x.size, C.byref(s), C.byref(m)))
    return s.value, m.value


def prim_queue_bitmap(queue: np.ndarray, n: int):
    q = np.ascontiguousarray(queue, np.uint32)
    words = (n + 31) // 32
    bm = np.zeros(max(words, 1), np.uint32)
    q2 = np.zeros(max(n, 1), np.uint32)
    cnt = C.c_uint64(0)
    check(lib().gb_prim_queue_bitmap(q if q.size else np.zeros(1, np.uint32), q.size, n, bm, q2, C.byref(cnt)))
    return bm[:words], q2[: cnt.value]


def barrier_timeout_selftest(spin_limit: int = 1000) -> int:
    """Status of a grid barrier that cannot complete (expected: 4, timeout)."""
    return lib().gb_debug_barrier_timeout(spin_limit)


def device_info():
    name = C.create_string_buffer(256)
    sms, ma, mi = C.c_int(), C.c_int(), C.c_int()
    check(lib().gb_device_info(name, 256, C.byref(sms), C.byref(ma), C.byref(mi)))
    return name.value.decode(), sms.value, (ma.value, mi.value)
