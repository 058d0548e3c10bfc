"""SNAP edge-list inputs for the converter tests (graph::convertSnap,
src/graph/snap.cpp:17-149): the line rules, every error the reference raises,
the 4 MiB line limit on both sides, and larger seeded texts.

Each case is bytes built here (no files are committed); ``write_case`` puts
one on disk, gzip-compressed when asked.  make_snap_golden.py records what the
reference's own converter does with each of them in snap_golden.json.
"""
from __future__ import annotations

import gzip
import os

import numpy as np

LONG = 4 << 20  # the reference rejects a line of this many bytes before its newline

QUIRKS = (
    b"% sample network, tab separated\n"
    b"#  src\tdst\n"
    b"  # indented comment\n"
    b"3\t9\n"
    b"9 27\r\n"
    b"\t\r\n"                # whitespace only
    b"\n"
    b"3 9\n"                 # duplicate
    b"27\t27\n"              # self-loop
    b"  27 \t 3 \n"          # padding around the ids
    b"81\t9\t0.5\n"          # weight column, ignored
    b"9\t243 extra text\n"   # trailing text, ignored
    b"\r 81 3\n"             # carriage return before the ids
    b"9\t729"                # 729 only ever a target; no final newline
)


def _pad(prefix: bytes, length: int) -> bytes:
    """prefix followed by spaces up to `length` bytes (no newline)."""
    return prefix + b" " * (length - len(prefix))


SMALL = {
    "quirks": QUIRKS,
    "empty": b"",
    "comments_only": b"# a\n% b\n\n  \n",
    "self_loop_only": b"7 7\n",
    "max_id": b"4294967294 0\n",
    "wrap_2_64": b"18446744073709551626 5\n",  # 2^64 + 10: the reference's uint64 wraps to 10
    "leading_zeros": b"007 0008\n",
    "single_no_newline": b"1 2",
    "crlf": b"1 2\r\n2 3\r\n3 1\r\n",
    "dup_both_ways": b"1 2\n2 1\n1 2\n",
    # errors
    "one_field": b"1 2\n3\n",
    "cr_between": b"1\r2\n",
    "minus": b"-1 2\n",
    "plus_second": b"1 +2\n",
    "letter_after_first": b"5a 6\n",
    "nul_line": b"1 2\n\x00\n",
    "too_large_first": b"1 2\n4294967295 3\n",
    "too_large_second": b"0 4294967295\n",
    "first_error_wins": b"1 2\n#\n3\n7 99999999999\n",
    "too_large_then_bad": b"99999999999 x\n",
    "bad_then_too_large": b"x 99999999999\n",
}


def long_cases() -> dict[str, bytes]:
    """Lines at and around the 4 MiB limit (built on demand: ~4-9 MB each)."""
    return {
        "long_ok": _pad(b"1 2", LONG - 1) + b"\n3 4\n",
        "long_bad": b"1 2\n" + _pad(b"5 6", LONG) + b"\n7 8\n",
        "long_bad_last": b"1 2\n" + _pad(b"5 6", LONG),
        "long_ok_last": b"1 2\n" + _pad(b"5 6", LONG - 1),
        "bad_then_long": b"x\n" + _pad(b"5 6", LONG) + b"\n",
        "long_then_bad": _pad(b"5 6", LONG) + b"\nx\n",
        "long_comment_9mib": b"1 2\n#" + b"-" * (9 << 20) + b"\n3 4\n",
    }


def random_text(lines: int, seed: int, max_id: int = 1 << 20) -> bytes:
    """A SNAP-style text: random ids (duplicates and self-loops included), mixed
    separators, CRLF endings, comments, blank lines and weight columns."""
    rng = np.random.default_rng(seed)
    u = rng.integers(0, max_id, size=lines)
    v = rng.integers(0, max_id, size=lines)
    kind = rng.integers(0, 16, size=lines)
    seps = [b"\t", b" ", b"  ", b" \t"]
    out = [b"# random SNAP text\n"]
    for i in range(lines):
        k = int(kind[i])
        if k == 0:
            out.append(b"% comment line\n")
            continue
        if k == 1:
            out.append(b"\n")
            continue
        a, b = int(u[i]), int(v[i])
        if k == 2:
            b = a  # self-loop
        line = str(a).encode() + seps[k % 4] + str(b).encode()
        if k == 3:
            line += b"\t1.0"
        out.append(line + (b"\r\n" if k == 4 else b"\n"))
    return b"".join(out)


def rmat_dump(g, one_based: bool = True) -> bytes:
    """Every stored entry u v of a CSR as a text line (ids + 1 when one_based)."""
    rows = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(g.row_ptr.astype(np.int64)))
    off = 1 if one_based else 0
    body = "\n".join(f"{a + off}\t{b + off}" for a, b in zip(rows.tolist(), g.col_idx[: g.m].tolist()))
    return ("# rmat dump\n" + body + "\n").encode()


def write_case(data: bytes, directory: str, name: str, gz: bool = False) -> str:
    path = os.path.join(directory, name + (".txt.gz" if gz else ".txt"))
    if gz:
        with gzip.open(path, "wb") as f:
            f.write(data)
    else:
        with open(path, "wb") as f:
            f.write(data)
    return path
