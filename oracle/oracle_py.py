"""ctypes access to the test oracle (oracle/liboracle.so) and to the reference's
own CPU code (oracle/_ref/libgref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker or as the timed CPU
baseline, never as the product path.

Graphs cross this boundary as ``HostGraph`` (numpy uint32 row_ptr / col_idx
plus n, m, flags), the same layout as the reference's graph::CSR
(src/graph/csr.hpp:29-45).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
UNREACHED = 0xFFFFFFFF
FLAG_DIRECTED, FLAG_SORTED, FLAG_DEDUP = 1, 2, 4


@dataclass
class HostGraph:
    n: int
    m: int
    flags: int
    row_ptr: np.ndarray  # uint32[n+1]
    col_idx: np.ndarray  # uint32[m]

    @property
    def directed(self) -> bool:
        return bool(self.flags & FLAG_DIRECTED)

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_ptr).astype(np.uint32)

    def equal(self, other: "HostGraph") -> bool:
        return (self.n == other.n and self.m == other.m and self.flags == other.flags
                and np.array_equal(self.row_ptr, other.row_ptr)
                and np.array_equal(self.col_idx[: self.m], other.col_idx[: other.m]))


class _Csr(C.Structure):
    _fields_ = [("n", C.c_uint64), ("m", C.c_uint64), ("flags", C.c_uint32),
                ("row_ptr", C.POINTER(C.c_uint32)), ("col_idx", C.POINTER(C.c_uint32))]


class _ConvertStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("lines", "raw_max_id", "n", "m_before", "m")]


class _Level(C.Structure):
    _fields_ = [("level", C.c_uint32), ("direction", C.c_uint32),
                ("frontier", C.c_uint64), ("edges", C.c_uint64)]


_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def _ensure_built(path: str, target: str) -> None:
    if os.path.exists(path):
        return
    subprocess.run(["make", "-C", HERE, target], check=True, capture_output=True)


# ------------------------------------------------------------------ oracle

_orc = None


def lib():
    global _orc
    if _orc is None:
        path = os.path.join(HERE, "liboracle.so")
        _ensure_built(path, "oracle")
        L = C.CDLL(path)
        P = C.POINTER(_Csr)
        for name, args in {
            "orc_gen_path": [C.c_uint32], "orc_gen_star": [C.c_uint32],
            "orc_gen_complete": [C.c_uint32], "orc_gen_two_components": [],
            "orc_gen_empty": [C.c_uint32], "orc_gen_grid2d": [C.c_uint32, C.c_uint32],
            "orc_gen_rmat": [C.c_uint32, C.c_uint32, C.c_int, C.c_uint64],
            "orc_gen_rmat_edges": [C.c_uint32, C.c_uint64, C.c_int, C.c_uint64],
            "orc_from_edge_list": [C.c_uint64, _u32p, _u32p, C.c_uint64, C.c_int],
            "orc_transpose": [P], "orc_symmetrize": [P], "orc_permute": [P, _u32p],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = P
        L.orc_csr_free.argtypes = [P]
        L.orc_random_perm.argtypes = [C.c_uint64, C.c_uint64, _u32p]
        L.orc_rmat_draw.argtypes = [C.c_uint32, C.c_uint64, C.c_uint64, _u32p, _u32p]
        L.orc_validate.argtypes = [P]
        L.orc_validate.restype = C.c_int
        L.orc_bfs_serial.argtypes = [P, C.c_uint32, _u32p]
        L.orc_bfs_do.argtypes = [P, C.c_uint32, _u32p, C.c_double, C.c_double,
                                 C.POINTER(_Level), C.c_int]
        L.orc_bfs_do.restype = C.c_int
        L.orc_pick_sources.argtypes = [P, C.c_int, C.c_uint64, C.c_int, _u32p]
        L.orc_pick_sources.restype = C.c_int
        L.orc_component_edges.argtypes = [P, _u32p]
        L.orc_component_edges.restype = C.c_uint64
        L.orc_out_degrees.argtypes = [P, _u32p]
        L.orc_pagerank_serial.argtypes = [P, _u32p, _f64p, C.c_double, C.c_int, C.c_double,
                                          C.POINTER(C.c_double)]
        L.orc_pagerank_serial.restype = C.c_int
        for nm, gp in (("orc_check_ranks_f32", _f32p), ("orc_check_ranks_f64", _f64p)):
            f = getattr(L, nm)
            f.argtypes = [_f64p, gp, C.c_uint64] + [C.POINTER(C.c_double)] * 3
        L.orc_gs_no_worse.argtypes = [C.c_double] * 5
        L.orc_gs_no_worse.restype = C.c_int
        L.orc_mlp_loss_grad.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_int, _f32p, _f32p,
                                        _f32p, _f32p]
        L.orc_mlp_loss_grad.restype = C.c_double
        L.orc_mlp_forward.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, C.c_int, _f32p, _f32p]
        L.orc_reorder_degree.argtypes = [P, _u32p]
        L.orc_reorder_rcm.argtypes = [P, _u32p]
        L.orc_locality.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_convert_snap.argtypes = [C.c_char_p, C.c_int, C.POINTER(P), C.POINTER(_ConvertStats),
                                       C.c_char_p, C.c_size_t]
        L.orc_convert_snap.restype = C.c_int
        _orc = L
    return _orc


def _take(p) -> HostGraph:
    c = p.contents
    n, m = int(c.n), int(c.m)
    rp = np.ctypeslib.as_array(c.row_ptr, shape=(n + 1,)).copy()
    ci = (np.ctypeslib.as_array(c.col_idx, shape=(m,)).copy() if m
          else np.zeros(0, dtype=np.uint32))
    g = HostGraph(n, m, int(c.flags), rp, ci)
    lib().orc_csr_free(p)
    return g


class _View:
    """Borrowed oracle CSR over a HostGraph's numpy arrays (no copy)."""

    def __init__(self, g: HostGraph):
        self.g = g
        self.rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
        self.ci = np.ascontiguousarray(g.col_idx, dtype=np.uint32)
        if self.ci.size == 0:
            self.ci = np.zeros(1, dtype=np.uint32)
        self.s = _Csr(g.n, g.m, g.flags, self.rp.ctypes.data_as(C.POINTER(C.c_uint32)),
                      self.ci.ctypes.data_as(C.POINTER(C.c_uint32)))

    @property
    def ptr(self):
        return C.byref(self.s)


def gen(name: str, *args) -> HostGraph:
    return _take(getattr(lib(), "orc_gen_" + name)(*args))


def suite() -> list[tuple[str, HostGraph]]:
    """The reference's eight test graphs (src/graph/generators.cpp:77-88)."""
    return [
        ("path1000", gen("path", 1000)),
        ("star100k", gen("star", 100000)),
        ("complete200", gen("complete", 200)),
        ("two_components", gen("two_components")),
        ("empty1000", gen("empty", 1000)),
        ("grid100x100", gen("grid2d", 100, 100)),
        ("rmat12", gen("rmat", 12, 16, 0, 42)),
        ("rmat12_directed", gen("rmat", 12, 16, 1, 43)),
    ]


def from_edges(n: int, eu, ev, directed: bool) -> HostGraph:
    eu = np.ascontiguousarray(eu, dtype=np.uint32)
    ev = np.ascontiguousarray(ev, dtype=np.uint32)
    if eu.size == 0:
        eu = np.zeros(1, np.uint32)
        ev = np.zeros(1, np.uint32)
        return _take(lib().orc_from_edge_list(n, eu, ev, 0, int(directed)))
    return _take(lib().orc_from_edge_list(n, eu, ev, eu.size, int(directed)))


def transpose(g: HostGraph) -> HostGraph:
    return _take(lib().orc_transpose(_View(g).ptr))


def symmetrize(g: HostGraph) -> HostGraph:
    return _take(lib().orc_symmetrize(_View(g).ptr))


def permute(g: HostGraph, perm: np.ndarray) -> HostGraph:
    return _take(lib().orc_permute(_View(g).ptr, np.ascontiguousarray(perm, np.uint32)))


def rmat_draw(scale: int, edges: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """The raw R-MAT endpoint pairs (src/graph/generators.cpp:51-75 quadrant
    draws, any edge count), before fromEdgeList."""
    eu = np.zeros(max(edges, 1), dtype=np.uint32)
    ev = np.zeros(max(edges, 1), dtype=np.uint32)
    lib().orc_rmat_draw(scale, edges, seed, eu, ev)
    return eu[:edges], ev[:edges]


def random_perm(n: int, seed: int) -> np.ndarray:
    p = np.zeros(max(n, 1), dtype=np.uint32)
    lib().orc_random_perm(n, seed, p)
    return p[:n]


def validate(g: HostGraph) -> int:
    return lib().orc_validate(_View(g).ptr)


def bfs_serial(g: HostGraph, source: int) -> np.ndarray:
    d = np.zeros(max(g.n, 1), dtype=np.uint32)
    lib().orc_bfs_serial(_View(g).ptr, source, d)
    return d[: g.n]


def bfs_do(g: HostGraph, source: int, alpha=15.0, beta=18.0):
    """Returns (dist, [(level, 'T'|'B', frontier, edges), ...])."""
    d = np.zeros(max(g.n, 1), dtype=np.uint32)
    cap = 4 * (g.n + 2)
    tr = (_Level * cap)()
    k = lib().orc_bfs_do(_View(g).ptr, source, d, alpha, beta, tr, cap)
    levels = [(tr[i].level, chr(tr[i].direction), tr[i].frontier, tr[i].edges) for i in range(k)]
    return d[: g.n], levels


def pick_sources(g: HostGraph, count=64, seed=1, any_component=False) -> np.ndarray:
    out = np.zeros(max(count, 1), dtype=np.uint32)
    k = lib().orc_pick_sources(_View(g).ptr, count, seed, int(any_component), out)
    return out[:k]


def component_edges(g: HostGraph, dist: np.ndarray) -> int:
    return int(lib().orc_component_edges(_View(g).ptr, np.ascontiguousarray(dist, np.uint32)))


def out_degrees(g: HostGraph) -> np.ndarray:
    return g.degrees()


def pagerank_serial(g_in: HostGraph, outdeg: np.ndarray, iters=20, tol=0.0, damping=0.85):
    """Returns (ranks float64[n], iterations, last L1 change)."""
    r = np.zeros(max(g_in.n, 1), dtype=np.float64)
    last = C.c_double(0)
    it = lib().orc_pagerank_serial(_View(g_in).ptr, np.ascontiguousarray(outdeg, np.uint32), r,
                                   damping, iters, tol, C.byref(last))
    return r[: g_in.n], it, last.value


@dataclass
class PrCheck:
    l1: float
    max_rel_top: float
    sum: float

    def ok(self) -> bool:  # src/cpu/pagerank_cpu.hpp:37-40
        return self.l1 < 1e-4 and self.max_rel_top < 1e-3 and abs(self.sum - 1.0) < 1e-4


def check_ranks(ref: np.ndarray, got: np.ndarray) -> PrCheck:
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    ref = np.ascontiguousarray(ref, np.float64)
    if got.dtype == np.float32:
        lib().orc_check_ranks_f32(ref, np.ascontiguousarray(got), ref.size, C.byref(a), C.byref(b), C.byref(c))
    else:
        lib().orc_check_ranks_f64(ref, np.ascontiguousarray(got, np.float64), ref.size, C.byref(a),
                                  C.byref(b), C.byref(c))
    return PrCheck(a.value, b.value, c.value)


def gs_no_worse(gs: PrCheck, jacobi: PrCheck) -> bool:
    return bool(lib().orc_gs_no_worse(gs.l1, gs.max_rel_top, gs.sum, jacobi.l1, jacobi.max_rel_top))


def mlp_loss_grad(nf, nh, no, params, x, y, mask):
    params = np.ascontiguousarray(params, np.float32)
    g = np.zeros_like(params)
    loss = lib().orc_mlp_loss_grad(nf, nh, no, params, x.shape[0], np.ascontiguousarray(x, np.float32),
                                   np.ascontiguousarray(y, np.float32),
                                   np.ascontiguousarray(mask, np.float32), g)
    return loss, g


def mlp_forward(nf, nh, no, params, x):
    out = np.zeros((x.shape[0], no), dtype=np.float32)
    lib().orc_mlp_forward(nf, nh, no, np.ascontiguousarray(params, np.float32), x.shape[0],
                          np.ascontiguousarray(x, np.float32), out)
    return out


def reorder(g: HostGraph, ordering: str, seed: int = 1) -> np.ndarray:
    """reorder::compute (src/graph/reorder.cpp:94-100): perm[old] = new."""
    if ordering == "original":
        return np.arange(g.n, dtype=np.uint32)
    if ordering == "random":
        return random_perm(g.n, seed)
    p = np.zeros(max(g.n, 1), np.uint32)
    fn = {"degree": lib().orc_reorder_degree, "rcm": lib().orc_reorder_rcm}[ordering]
    v = _View(g)
    fn(v.ptr, p)
    return p[: g.n]


def locality(g: HostGraph) -> tuple[float, float]:
    """(mean |u - v|, fraction of entries within one 64-vertex block)."""
    a, b, v = C.c_double(0), C.c_double(0), _View(g)
    lib().orc_locality(v.ptr, C.byref(a), C.byref(b))
    return a.value, b.value


class ConvertError(RuntimeError):
    """A converter failure; str() is the reference's message."""


def convert_snap(path: str, directed: bool) -> tuple[HostGraph, dict]:
    """SNAP text (plain or gzip) -> (CSR, stats) by the oracle; raises
    ConvertError with the reference's message on bad input."""
    out = C.POINTER(_Csr)()
    st = _ConvertStats()
    msg = C.create_string_buffer(1024)
    if lib().orc_convert_snap(path.encode(), int(directed), C.byref(out), C.byref(st), msg, 1024):
        raise ConvertError(msg.value.decode())
    return _take(out), {k: int(getattr(st, k)) for k, _ in _ConvertStats._fields_}


# --------------------------------------------------- the reference's own code

_ref = None
REF_PATH = os.path.join(HERE, "_ref", "libgref.so")


def ref_available() -> bool:
    """True when the reference build exists; otherwise tries `make ref` once
    (the Makefile knows where the reference sources are and skips when they
    are absent)."""
    if not os.path.exists(REF_PATH):
        subprocess.run(["make", "-C", HERE, "ref"], check=False, capture_output=True)
    return os.path.exists(REF_PATH)


def ref():
    """The reference's CPU code compiled from its sources (None if absent)."""
    global _ref
    if _ref is None and ref_available():
        L = C.CDLL(REF_PATH)
        vp = C.c_void_p
        for name, args in {
            "gref_suite": [C.c_char_p], "gref_path": [C.c_uint32], "gref_star": [C.c_uint32],
            "gref_complete": [C.c_uint32], "gref_grid2d": [C.c_uint32, C.c_uint32],
            "gref_rmat": [C.c_uint32, C.c_uint32, C.c_int, C.c_uint64],
            "gref_from_arrays": [C.c_uint64, C.c_uint64, C.c_uint32, _u32p, _u32p],
            "gref_from_edges": [C.c_uint64, _u32p, _u32p, C.c_uint64, C.c_int],
            "gref_symmetrize": [vp], "gref_transpose": [vp], "gref_permute": [vp, _u32p],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = vp
        L.gref_ordering.argtypes = [vp, C.c_char_p, C.c_uint64, _u32p]
        for name, rt in (("gref_n", C.c_uint64), ("gref_m", C.c_uint64), ("gref_flags", C.c_uint32)):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = rt
        L.gref_copy.argtypes = [vp, _u32p, _u32p]
        L.gref_validate.argtypes = [vp]
        L.gref_free.argtypes = [vp]
        L.gref_bfs_serial.argtypes = [vp, C.c_uint32, _u32p]
        L.gref_bfs_omp.argtypes = [vp, C.c_uint32, _u32p, C.c_int]
        L.gref_bfs_do.argtypes = [vp, C.c_uint32, _u32p, C.c_double, C.c_double, C.c_int,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.gref_bfs_do.restype = C.c_int
        L.gref_pagerank.argtypes = [vp, _u32p, _f64p, C.c_int, C.c_double, C.c_int,
                                    C.POINTER(C.c_double)]
        L.gref_pagerank.restype = C.c_int
        L.gref_check_ranks_f32.argtypes = [_f64p, _f32p, C.c_uint64] + [C.POINTER(C.c_double)] * 3
        L.gref_max_threads.restype = C.c_int
        L.gref_locality.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.gref_convert_snap.argtypes = [C.c_char_p, C.c_char_p, C.c_int, _u64p, C.c_char_p, C.c_size_t]
        L.gref_convert_snap.restype = vp
        _ref = L
    return _ref


class RefGraph:
    """A graph::CSR held by the reference build."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("reference call returned no graph")
        self.h = C.c_void_p(handle)

    def __del__(self):
        if _ref is not None and self.h:
            _ref.gref_free(self.h)

    @staticmethod
    def of(g: HostGraph) -> "RefGraph":
        ci = g.col_idx if g.m else np.zeros(1, np.uint32)
        return RefGraph(ref().gref_from_arrays(g.n, g.m, g.flags,
                                               np.ascontiguousarray(g.row_ptr, np.uint32),
                                               np.ascontiguousarray(ci, np.uint32)))

    def host(self) -> HostGraph:
        L = ref()
        n, m = int(L.gref_n(self.h)), int(L.gref_m(self.h))
        rp = np.zeros(n + 1, np.uint32)
        ci = np.zeros(max(m, 1), np.uint32)
        L.gref_copy(self.h, rp, ci)
        return HostGraph(n, m, int(L.gref_flags(self.h)), rp, ci[:m])

    def symmetrize(self) -> "RefGraph":
        return RefGraph(ref().gref_symmetrize(self.h))

    def transpose(self) -> "RefGraph":
        return RefGraph(ref().gref_transpose(self.h))

    def permute(self, perm) -> "RefGraph":
        return RefGraph(ref().gref_permute(self.h, np.ascontiguousarray(perm, np.uint32)))

    def ordering(self, name: str, seed: int = 1) -> np.ndarray:
        n = int(ref().gref_n(self.h))
        p = np.zeros(max(n, 1), np.uint32)
        ref().gref_ordering(self.h, name.encode(), seed, p)
        return p[:n]

    def locality(self) -> tuple[float, float]:
        a, b = C.c_double(0), C.c_double(0)
        ref().gref_locality(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def bfs_serial(self, src: int) -> np.ndarray:
        n = int(ref().gref_n(self.h))
        d = np.zeros(max(n, 1), np.uint32)
        ref().gref_bfs_serial(self.h, src, d)
        return d[:n]

    def bfs_do(self, src: int, alpha=15.0, beta=18.0, threads=0, trace=True):
        n = int(ref().gref_n(self.h))
        d = np.zeros(max(n, 1), np.uint32)
        if not trace:
            ref().gref_bfs_do(self.h, src, d, alpha, beta, threads, None, None, None, None, 0)
            return d[:n], []
        cap = 4 * (n + 2)
        lv = np.zeros(cap, np.uint32)
        dr = np.zeros(cap, np.uint8)
        fr = np.zeros(cap, np.uint64)
        ed = np.zeros(cap, np.uint64)
        k = ref().gref_bfs_do(self.h, src, d, alpha, beta, threads, lv.ctypes.data, dr.ctypes.data,
                              fr.ctypes.data, ed.ctypes.data, cap)
        return d[:n], [(int(lv[i]), chr(dr[i]), int(fr[i]), int(ed[i])) for i in range(k)]

    def pagerank(self, outdeg, iters=20, tol=0.0, threads=-1):
        n = int(ref().gref_n(self.h))
        r = np.zeros(max(n, 1), np.float64)
        last = C.c_double(0)
        it = ref().gref_pagerank(self.h, np.ascontiguousarray(outdeg, np.uint32), r, iters, tol,
                                 threads, C.byref(last))
        return r[:n], it, last.value


def ref_rmat_graph(scale: int, edges: int, seed: int, perm_seed: int) -> RefGraph:
    """An undirected R-MAT graph built by the reference's own code: the restated
    quadrant draw (rmat_draw), then graph::fromEdgeList, reorder "random"
    (perm_seed) and graph::permute -- how the benchmark graph of 2^22 vertices
    and 8.5 * 2^22 drawn edges is defined."""
    eu, ev = rmat_draw(scale, edges, seed)
    r = RefGraph(ref().gref_from_edges(1 << scale, eu, ev, eu.size, 0))
    del eu, ev
    return r.permute(r.ordering("random", perm_seed))


def ref_check_ranks(ref_ranks: np.ndarray, got: np.ndarray) -> PrCheck:
    """The reference's own cpu::checkRanks (src/cpu/pagerank_cpu.hpp:37-60)."""
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    ref().gref_check_ranks_f32(np.ascontiguousarray(ref_ranks, np.float64),
                               np.ascontiguousarray(got, np.float32), ref_ranks.size,
                               C.byref(a), C.byref(b), C.byref(c))
    return PrCheck(a.value, b.value, c.value)


def ref_suite(name: str) -> RefGraph:
    return RefGraph(ref().gref_suite(name.encode()))


def ref_convert_snap(path: str, out_path: str, directed: bool) -> tuple[RefGraph, dict]:
    """graph::convertSnap(path, out_path, directed), then graph::load(out_path);
    raises ConvertError with the reference's exception text."""
    st = np.zeros(5, np.uint64)
    msg = C.create_string_buffer(1024)
    h = ref().gref_convert_snap(path.encode(), out_path.encode(), int(directed), st, msg, 1024)
    if not h:
        raise ConvertError(msg.value.decode())
    keys = ("lines", "raw_max_id", "n", "m_before", "m")
    return RefGraph(h), {k: int(v) for k, v in zip(keys, st)}
