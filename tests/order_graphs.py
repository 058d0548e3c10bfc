"""The symmetric graphs of tests/golden/order_golden.json, rebuilt with the
oracle's generators (pinned to the reference's by test_oracle.py)."""
import oracle_py as O

SUITE = ["path1000", "star100k", "complete200", "two_components", "empty1000", "grid100x100",
         "rmat12", "rmat12_directed"]


def order_graphs():
    suite = dict(O.suite())
    for name in SUITE:
        g = suite[name]
        yield name, (O.symmetrize(g) if g.directed else g)
    yield "grid1400x1400", O.gen("grid2d", 1400, 1400)
    yield "rmat16_ef16_s1", O.gen("rmat", 16, 16, 0, 1)
    yield "rmat18_ef8_s5_directed_sym", O.symmetrize(O.gen("rmat", 18, 8, 1, 5))
