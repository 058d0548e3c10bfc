"""The learned selector: GPU forward/backward kernels against the oracle's
double-precision MLP, training reduces the loss, and whatever the selector
picks the BFS depths stay exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def shape(gb):
    return gb.selector_shape()


def test_gpu_gradients_match_oracle(gb, oracle):
    nf, nh, no = shape(gb)
    npar = gb.selector_param_count()
    rng = np.random.default_rng(1)
    for batch in (1, 7, 256, 1000):
        p = rng.normal(0, 0.3, npar).astype(np.float32)
        x = rng.random((batch, nf), dtype=np.float32)
        y = rng.normal(3, 1, (batch, no)).astype(np.float32)
        mask = (rng.random((batch, no)) > 0.1).astype(np.float32)
        g = np.zeros(npar, np.float32)
        loss = gb.C.c_double(0)
        gb.check(gb.lib().gb_mlp_loss_grad(p, batch, x, y, mask, g, gb.C.byref(loss)))
        ref_loss, ref_g = oracle.mlp_loss_grad(nf, nh, no, p, x, y, mask)
        assert abs(loss.value - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
        scale = np.abs(ref_g).max()
        assert np.abs(g - ref_g).max() <= 1e-4 * scale + 1e-6, batch
        out = np.zeros((batch, no), np.float32)
        gb.check(gb.lib().gb_mlp_forward(p, batch, x, out))
        assert np.allclose(out, oracle.mlp_forward(nf, nh, no, p, x), rtol=1e-4, atol=1e-4)


def test_gpu_training_fits_a_known_function(gb):
    nf, nh, no = shape(gb)
    rng = np.random.default_rng(2)
    x = rng.random((2048, nf), dtype=np.float32)
    y = np.stack([x[:, 0] * 4 + 1, x[:, 1] * 3, x[:, 2] + x[:, 3], 2 - x[:, 4], x[:, 5] * x[:, 6] * 5], 1)
    y = y[:, :no].astype(np.float32)
    mask = np.ones_like(y)
    from graph_analytics_applesilicon_b200.train_selector import init_params
    p0 = init_params(0)
    g0 = np.zeros_like(p0)
    l0 = gb.C.c_double(0)
    gb.check(gb.lib().gb_mlp_loss_grad(p0, len(x), x, y, mask, g0, gb.C.byref(l0)))
    p = p0.copy()
    fl = gb.C.c_float(0)
    gb.check(gb.lib().gb_mlp_train(p, len(x), x, y, mask, 200, 128, 3e-3, 5, gb.C.byref(fl)))
    assert fl.value < 0.02 * l0.value and fl.value < 0.05


def test_selector_picks_never_change_depths(gb, oracle):
    """Random selector parameters (arbitrary strategy sequences) and the
    shipped ones give cpu_serial's depths; with an unbounded direction margin
    the directions are the alpha/beta rule's."""
    nf, nh, no = shape(gb)
    rng = np.random.default_rng(3)
    graphs = [gb.gen.rmat(15, 16, False, 7), gb.gen.road(150, 150, 0.04, 0.005, 8), gb.gen.star(50000)]
    params = [rng.normal(0, 1.0, gb.selector_param_count()).astype(np.float32) for _ in range(4)]
    shipped = gb.default_selector_params("single")
    if shipped is not None:
        params.append(shipped)
    for g in graphs:
        bfs = gb.GpuBfs(g)
        for s in gb.pick_sources(g, 3, 1):
            ref = oracle.bfs_serial(g, int(s))
            _, ctr = oracle.bfs_do(g, int(s))
            for p in params:
                bfs.set_selector(p, 0)
                for margin in (0.0, 0.5, 1e9):
                    o = gb.BfsOptions(selector="learned", sel_margin=margin)
                    d, tr = bfs.run("gpu_do_persistent", int(s), opts=o, trace=True)
                    assert np.array_equal(d, ref)
                    assert [L["frontier"] for L in tr] == [t[2] for t in ctr]
                    if margin > 1e6:  # direction left to the alpha/beta rule
                        assert [L["direction"] for L in tr] == [t[1] for t in ctr]


def test_learned_without_parameters_is_an_error(gb):
    bfs = gb.GpuBfs(gb.gen.path(10))
    with pytest.raises(gb.GraphError) as e:
        bfs.run("gpu_do_persistent", 0, opts=gb.BfsOptions(selector="learned"))
    assert e.value.status == 5
