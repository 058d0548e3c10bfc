"""GPU PageRank parity through the C ABI against the oracle, following the
reference's tests/test_main.cpp:665-783.  Tolerances are the reference's
checkRanks (src/cpu/pagerank_cpu.hpp:37-40): L1 < 1e-4, max relative error on
the top-1000 vertices < 1e-3, |sum - 1| < 1e-4; Gauss-Seidel runs use
gsNoWorseThanJacobi (:80-84) against the tol-1e-10 reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFGS = [("gpu_push", 16, 256), ("gpu_pull_scalar", 16, 256), ("gpu_pull_vector", 16, 256),
        ("gpu_pull_blocked", 16, 256),
        ("gpu_pull_adaptive", 16, 256), ("gpu_pull_adaptive", 1 << 30, 1 << 31),
        ("gpu_pull_adaptive", 0, 0), ("gpu_pull_adaptive", 0, 1 << 30), ("gpu_pull_adaptive", 2, 3)]


@pytest.fixture(scope="module")
def prcases(gb, oracle):
    out = []
    for name, g in gb.gen.suite():
        gin = gb.transpose(g) if g.directed else g
        od = g.degrees()
        h = gb.GpuPageRank(g.n, g, gin, od)
        out.append((name, g, gin, od, h))
    return out


@pytest.mark.parametrize("tol", [0.0, 1e-6])
def test_variants_match_reference(prcases, gb, oracle, tol):
    failures = []
    for name, g, gin, od, h in prcases:
        iters = 1000 if tol > 0 else 20
        ref, ref_iters, _ = oracle.pagerank_serial(gin, od, iters, tol)
        for variant, sm, lm in CFGS:
            for tg in (32, 256, 1024):
                r = h.run(variant, gb.PrOptions(tol=tol, iters=iters, tg=tg, small_max=sm, large_min=lm))
                chk = oracle.check_ranks(ref, h.ranks())
                if not chk.ok():
                    failures.append((name, variant, sm, lm, tol, tg, chk))
                    continue
                if tol == 0:
                    assert r.iters == 20
                    continue
                if r.floor_stop or (variant == "gpu_push" and name == "star100k"):
                    continue
                if abs(r.iters - ref_iters) > 3:
                    failures.append((name, variant, tg, "iters", r.iters, ref_iters, r.last_delta))
    assert not failures, failures[:10]


def test_inplace_option_converges(prcases, gb, oracle):
    for name, g, gin, od, h in prcases:
        conv, _, _ = oracle.pagerank_serial(gin, od, 1000, 1e-10)
        for variant in ("gpu_pull_scalar", "gpu_pull_vector", "gpu_pull_adaptive"):
            h.run(variant, gb.PrOptions(iters=200, inplace=1))
            c = oracle.check_ranks(conv, h.ranks())
            assert c.ok(), (name, variant, c)


def test_gs_converges_to_reference(gb, oracle):
    colored = natural = deferred_graphs = 0
    failures = []
    for name, g in gb.gen.suite():
        gin = gb.transpose(g) if g.directed else g
        od = g.degrees()
        conv, _, _ = oracle.pagerank_serial(gin, od, 1000, 1e-10)
        jac, _, _ = oracle.pagerank_serial(gin, od, 1000, 1e-6)
        jerr = oracle.check_ranks(conv, jac)
        for K in (0, 2):
            h = gb.GpuPageRank(g.n, None, gin, od)
            h.prepareGS(K)
            is_colored, sets, deferred = h.gs_info()
            if is_colored:
                colored += 1
            else:
                natural += 1
            deferred_graphs += deferred > 0
            for tg in (32, 256, 1024):
                for what, tol, tol_rel, iters in (("20 sweeps", 0.0, 0.0, 20), ("200 sweeps", 0.0, 0.0, 200),
                                                  ("tol 2.5e-7", 2.5e-7, 0.0, 1000),
                                                  ("tol 1e-6 + rel 2.5e-5", 1e-6, 2.5e-5, 1000)):
                    r = h.run("gpu_pull_gs", gb.PrOptions(tol=tol, tol_rel=tol_rel, iters=iters, tg=tg))
                    c = oracle.check_ranks(conv, h.ranks())
                    if iters == 20:
                        ok = abs(c.sum - 1.0) < 1e-4
                    elif iters == 200:
                        ok = c.ok()
                    else:
                        ok = oracle.gs_no_worse(c, jerr)
                    if not ok:
                        failures.append((name, K, is_colored, what, tg, c, r.iters))
    assert not failures, failures[:8]
    assert colored > 0 and natural > 0 and deferred_graphs > 0


def test_f64_oracle_kernel_matches_cpu(prcases, gb, oracle):
    for name, g, gin, od, h in prcases:
        for tol, iters in ((0.0, 20), (1e-9, 1000)):
            ref, ref_iters, _ = oracle.pagerank_serial(gin, od, iters, tol)
            r = h.run("gpu_pull_f64", gb.PrOptions(tol=tol, iters=iters))
            got = h.ranks_f64()
            # same arithmetic in a different summation order: double rounding only
            assert np.abs(got - ref).sum() < 1e-10, name
            if tol > 0:
                assert abs(r.iters - ref_iters) <= 1, (name, r.iters, ref_iters)


def test_errors(prcases, gb):
    name, g, gin, od, h = prcases[0]
    with pytest.raises(gb.GraphError):
        h.run("gpu_pull_vector", gb.PrOptions(tg=48))
    pull_only = gb.GpuPageRank(g.n, None, gin, od)
    with pytest.raises(gb.GraphError):
        pull_only.run("gpu_push")
    fresh = gb.GpuPageRank(g.n, None, gin, od)
    with pytest.raises(gb.GraphError):
        fresh.ranks()


def test_larger_graphs_fp32_vs_fp64(gb, oracle):
    """Web-shaped directed graph: FP32 variants vs the FP64 GPU oracle (itself
    checked against the CPU oracle here), fixed 20 iterations and tol 1e-6."""
    g = gb.gen.web(200000, 5.8, 2.1, 875)
    gin = gb.transpose(g)
    od = g.degrees()
    h = gb.GpuPageRank(g.n, g, gin, od)
    for tol, iters in ((0.0, 20), (1e-6, 1000)):
        ref, ref_iters, _ = oracle.pagerank_serial(gin, od, iters, tol)
        h.run("gpu_pull_f64", gb.PrOptions(tol=tol, iters=iters))
        r64 = h.ranks_f64()
        assert np.abs(r64 - ref).sum() < 1e-10
        for variant in ("gpu_pull_adaptive", "gpu_pull_blocked", "gpu_pull_vector", "gpu_pull_scalar", "gpu_push"):
            r = h.run(variant, gb.PrOptions(tol=tol, iters=iters))
            c = oracle.check_ranks(r64, h.ranks())
            assert c.ok() and c.l1 < 1e-5, (variant, tol, c)
            if tol > 0 and not r.floor_stop:
                assert abs(r.iters - ref_iters) <= 3
    for sm, lm in ((16, 256), (4, 64), (64, 100000)):
        h.run("gpu_pull_adaptive", gb.PrOptions(iters=20, small_max=sm, large_min=lm, inplace=1))
        assert abs(h.ranks().astype(np.float64).sum() - 1) < 1e-4


def test_gs_with_split_hubs(gb, oracle):
    """Gauss-Seidel where vertices with >= 4096 in-edges are split into warp
    chunks: the web graph (colored order, hub inside a colour set) and a
    directed R-MAT (natural order or colored, whichever prepareGS picks)."""
    modes = set()
    for g in (gb.gen.web(200000, 5.8, 2.1, 875), gb.gen.rmat(16, 16, True, 3), gb.gen.rmat(15, 32, True, 5)):
        gin = gb.transpose(g)
        od = g.degrees()
        assert int(np.diff(gin.row_ptr).max()) >= 4096
        conv, _, _ = oracle.pagerank_serial(gin, od, 2000, 1e-12)
        jac, _, _ = oracle.pagerank_serial(gin, od, 1000, 1e-6)
        jerr = oracle.check_ranks(conv, jac)
        h = gb.GpuPageRank(g.n, None, gin, od)
        for K in (0, 2):
            h.prepareGS(K)
            modes.add(h.gsColored())
            h.run("gpu_pull_gs", gb.PrOptions(iters=200))
            assert oracle.check_ranks(conv, h.ranks()).ok(), (g.n, K)
            h.run("gpu_pull_gs", gb.PrOptions(tol=2.5e-7, iters=1000))
            assert oracle.gs_no_worse(oracle.check_ranks(conv, h.ranks()), jerr), (g.n, K)
    assert True in modes


def test_blocked_pull_layouts(gb, oracle):
    """gpu_pull_blocked against the FP64 GPU pull and the CPU oracle on graphs
    that exercise its layout: many column parts and row blocks with split-off
    rows of >= 4096 in-edges (web-shaped, Chung-Lu), a last part that is not a
    multiple of 4 vertices, and more row blocks than SMs (a 4M-vertex path,
    so blocks loop over several row blocks)."""
    cases = [gb.gen.web(200003, 5.8, 2.1, 17), gb.gen.chung_lu(300001, 2.2, 40.0, 5), gb.gen.path(4000001)]
    for g in cases:
        gin = gb.transpose(g) if g.directed else g
        od = g.degrees()
        h = gb.GpuPageRank(g.n, None, gin, od)
        for tol, iters in ((0.0, 20), (1e-6, 1000)):
            ref, ref_iters, _ = oracle.pagerank_serial(gin, od, iters, tol)
            r = h.run("gpu_pull_blocked", gb.PrOptions(tol=tol, iters=iters))
            c = oracle.check_ranks(ref, h.ranks())
            assert c.ok() and c.l1 < 1e-5, (g.n, tol, c)
            if tol == 0:
                assert r.iters == 20
            elif not r.floor_stop:
                assert abs(r.iters - ref_iters) <= 3, (g.n, r.iters, ref_iters)
