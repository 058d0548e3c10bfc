"""Writes tests/golden/golden.json and golden_ranks.npz from the reference's
own CPU code (oracle/_ref/libgref.so, compiled from the reference sources by
oracle/Makefile).  Run in a tree where the reference sources exist:

    make -C oracle && python tests/golden/make_golden.py

What is recorded (all produced by the reference's functions, nothing by this
repository's code):
  * the eight suite graphs of src/graph/generators.cpp:77-88 -- n, m, flags and
    SHA-256 of row_ptr / col_idx, of the stored graph, its symmetrization and
    its transpose;
  * star(100000), grid2d(1400, 1400) and rmat(16, 16, undirected, 1) the same way;
  * the R-MAT scale-22 config graph: the reference's quadrant draw is
    restated to produce 8.5 * 2^22 edges (its gen::rmat only takes an integer
    edge factor), then the reference's fromEdgeList, reorder "random" (seed 1)
    and permute build the graph whose hashes are stored;
  * BFS: for every suite graph and the reference test sources
    (tests/test_main.cpp:286-291, plus the max-degree vertex), the SHA-256 of
    cpu_serial's distance array, the reached count, the TEPS denominator and
    cpu_do's per-level (direction, frontier, edges) trace under the four
    alpha/beta modes of tests/test_main.cpp:322-350;
  * PageRank: cpu_serial ranks (float64) after 20 iterations and at tol 1e-6
    (iteration count and last L1 change recorded), plus the converged
    (tol 1e-10) ranks, for every suite graph.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle_py as O  # noqa: E402

SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]
DO_MODES = {"default": (15.0, 18.0), "all_td": (1e-12, 18.0), "all_bu": (1e12, 1e12),
            "flip_flop": (2.0, 4.0)}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def graph_record(g: O.HostGraph) -> dict:
    return {"n": g.n, "m": g.m, "flags": g.flags, "row_ptr": sha(g.row_ptr), "col_idx": sha(g.col_idx)}


def trace_record(tr) -> dict:
    """Per-level (direction, frontier, edges) of a cpu_do trace, compactly."""
    return {"levels": len(tr), "dirs": "".join(t[1] for t in tr),
            "frontier": sha(np.array([t[2] for t in tr], dtype=np.uint64)),
            "edges": sha(np.array([t[3] for t in tr], dtype=np.uint64))}


def test_sources(n: int) -> list:
    """tests/test_main.cpp:286-291."""
    s = [0, n // 2, n - 1]
    x = 12345
    for _ in range(3):
        x = (x * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        s.append((x >> 33) % n)
    return s


def rmat_edges_c2(scale=22, edges=35651584, seed=22):
    """The reference's quadrant draw (src/graph/generators.cpp:51-75) for a
    non-integer edge factor; vectorised over edges (stream position i*scale+bit)."""
    n_draw = edges * scale
    golden = np.uint64(0x9E3779B97F4A7C15)
    k = np.arange(1, n_draw + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * golden
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    r = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    del z, k
    r = r.reshape(edges, scale)
    a, b, c = 0.57, 0.19, 0.19
    ub = (r >= a + b).astype(np.uint32)
    vb = (((r >= a) & (r < a + b)) | (r >= a + b + c)).astype(np.uint32)
    del r
    w = (np.uint32(1) << np.arange(scale - 1, -1, -1, dtype=np.uint32))
    u = (ub * w).sum(axis=1, dtype=np.uint64).astype(np.uint32)
    v = (vb * w).sum(axis=1, dtype=np.uint64).astype(np.uint32)
    return u, v


def main():
    if O.ref() is None:
        raise SystemExit("reference build oracle/_ref/libgref.so is missing")
    out = {"generator": "tests/golden/make_golden.py", "graphs": {}, "bfs": {}, "pagerank": {}}
    ranks = {}
    for name in SUITE:
        r = O.ref_suite(name)
        g = r.host()
        rs = r.symmetrize()
        out["graphs"][name] = {"stored": graph_record(g), "sym": graph_record(rs.host()),
                               "transpose": graph_record(r.transpose().host())}
        s = rs.host()
        srcs = test_sources(s.n)
        deg = s.degrees()
        srcs.append(int(np.argmax(deg)) if s.n else 0)
        recs = []
        for src in srcs:
            d = rs.bfs_serial(src)
            rec = {"source": int(src), "dist": sha(d), "reached": int((d != O.UNREACHED).sum()),
                   "max_depth": int(d[d != O.UNREACHED].max()),
                   "comp_edges": int(deg[d != O.UNREACHED].sum(dtype=np.uint64) // 2), "do": {}}
            for mode, (a, b) in DO_MODES.items():
                dd, tr = rs.bfs_do(src, a, b, threads=1)
                assert np.array_equal(dd, d)
                rec["do"][mode] = trace_record(tr)
            recs.append(rec)
        out["bfs"][name] = recs
        rin = r.transpose() if g.directed else r
        od = g.degrees()
        pr = {}
        for key, iters, tol in (("fixed20", 20, 0.0), ("tol1e-6", 1000, 1e-6), ("conv1e-10", 1000, 1e-10)):
            rk, it, last = rin.pagerank(od, iters, tol, threads=-1)
            pr[key] = {"iters": it, "last_delta": last, "sum": float(rk.sum())}
            ranks[f"{name}/{key}"] = rk
        out["pagerank"][name] = pr

    extra = {"star100000": O.RefGraph(O.ref().gref_star(100000)),
             "grid1400x1400": O.RefGraph(O.ref().gref_grid2d(1400, 1400)),
             "rmat16_ef16_s1": O.RefGraph(O.ref().gref_rmat(16, 16, 0, 1))}
    for name, r in extra.items():
        out["graphs"][name] = {"stored": graph_record(r.host())}

    u, v = rmat_edges_c2()
    n = 1 << 22
    # The restated draw must agree with the reference's own gen::rmat on a case
    # it can express (same stream layout, integer edge factor).
    us, vs = rmat_edges_c2(scale=12, edges=16 << 12, seed=42)
    chk = O.RefGraph(O.ref().gref_from_edges(1 << 12, us, vs, us.size, 0)).host()
    assert chk.equal(O.ref_suite("rmat12").host())
    r = O.RefGraph(O.ref().gref_from_edges(n, u, v, u.size, 0))
    del u, v
    perm = r.ordering("random", 1)
    rp = r.permute(perm)
    out["graphs"]["rmat22_c2"] = {"stored": graph_record(rp.host()), "edges_drawn": 35651584,
                                  "gen_seed": 22, "perm_seed": 1, "perm": sha(perm)}

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"), sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "golden_ranks.npz"), **ranks)
    print("wrote golden.json and golden_ranks.npz")


if __name__ == "__main__":
    main()
