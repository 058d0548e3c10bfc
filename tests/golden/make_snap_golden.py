"""Writes tests/golden/snap_golden.json: what the reference's own converter
(graph::convertSnap + graph::load, src/graph/snap.cpp:85-149 and
src/graph/csr.cpp:54-84, compiled from the reference sources into
oracle/_ref/libgref.so by oracle/Makefile) produces for every input of
snap_cases.py, plain and gzip, directed and undirected.  Run where the
reference sources exist:

    make -C oracle && python tests/golden/make_snap_golden.py

Per case: either {"error": message} (the input path replaced by "{path}") or
the ConvertStats fields plus n, m, flags and SHA-256 of row_ptr / col_idx.
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, HERE)
import oracle_py as O  # noqa: E402
import snap_cases as S  # noqa: E402

RANDOM = {"random_200k": (200_000, 7)}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def record(path: str, directed: bool, tmp: str) -> dict:
    try:
        r, st = O.ref_convert_snap(path, os.path.join(tmp, "out.bin"), directed)
    except O.ConvertError as e:
        return {"error": str(e).replace(path, "{path}")}
    g = r.host()
    return {**st, "flags": g.flags, "row_ptr": sha(g.row_ptr), "col_idx": sha(g.col_idx)}


def all_cases() -> dict[str, bytes]:
    cases = dict(S.SMALL)
    cases.update(S.long_cases())
    for name, (lines, seed) in RANDOM.items():
        cases[name] = S.random_text(lines, seed)
    return cases


def main() -> None:
    if not O.ref_available():
        sys.exit("oracle/_ref/libgref.so is not built (needs the reference sources)")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, data in all_cases().items():
            for gz in (False, True):
                path = S.write_case(data, tmp, name, gz)
                for directed in (True, False):
                    out[f"{name}|{'gz' if gz else 'txt'}|{'dir' if directed else 'undir'}"] = record(path, directed, tmp)
                os.unlink(path)
    with open(os.path.join(HERE, "snap_golden.json"), "w") as f:
        json.dump({"random": RANDOM, "cases": out}, f, indent=1, sort_keys=True)
    print(f"{len(out)} records")


if __name__ == "__main__":
    main()
