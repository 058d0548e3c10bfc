"""Writes tests/golden/order_golden.json: the reference's own vertex orderings
(reorder::compute "degree" and "rcm", src/graph/reorder.cpp:27-100) and
locality metrics (:111-125), computed by the reference build
(oracle/_ref/libgref.so, compiled from the reference sources by
oracle/Makefile) on symmetric graphs it generates itself.  Run where the
reference sources exist:

    make -C oracle && python tests/golden/make_order_golden.py

Per graph: n, m_sym, SHA-256 of each permutation (uint32 perm[old] = new)
and (mean |u - v|, same 64-block fraction) of the graph under each ordering
(original included).
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


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def graphs():
    for name in SUITE:
        r = O.ref_suite(name)
        yield name, (r.symmetrize() if O.ref().gref_flags(r.h) & 1 else r)
    yield "grid1400x1400", O.RefGraph(O.ref().gref_grid2d(1400, 1400))
    yield "rmat16_ef16_s1", O.RefGraph(O.ref().gref_rmat(16, 16, 0, 1))
    yield "rmat18_ef8_s5_directed_sym", O.RefGraph(O.ref().gref_rmat(18, 8, 1, 5)).symmetrize()


def main() -> None:
    if not O.ref_available():
        sys.exit("oracle/_ref/libgref.so is not built (needs the reference sources)")
    out = {}
    for name, sym in graphs():
        h = sym.host()
        rec = {"n": h.n, "m": h.m, "orderings": {}}
        for ordering in ("original", "degree", "rcm"):
            perm = sym.ordering(ordering) if ordering != "original" else np.arange(h.n, dtype=np.uint32)
            relabeled = sym.permute(perm) if ordering != "original" else sym
            gap, same = relabeled.locality()
            rec["orderings"][ordering] = {"perm": sha(perm), "mean_gap": gap, "same_block64": same}
        out[name] = rec
        print(name, h.n, h.m)
    with open(os.path.join(HERE, "order_golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
