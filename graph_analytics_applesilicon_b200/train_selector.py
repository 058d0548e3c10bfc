"""Trains the learned per-level BFS strategy selector on the GPU.

  python -m graph_analytics_applesilicon_b200.train_selector generate OUT.npz
  python -m graph_analytics_applesilicon_b200.train_selector train DATA.npz [OUT.npy] [--seed S]
  python -m graph_analytics_applesilicon_b200.train_selector evaluate [PARAMS.npy]
  python -m graph_analytics_applesilicon_b200.train_selector generate-batch OUT.npz
  python -m graph_analytics_applesilicon_b200.train_selector train-batch DATA.npz
  python -m graph_analytics_applesilicon_b200.train_selector evaluate-batch

generate: on seeded synthetic graphs (R-MAT of several scales and densities,
road-shaped grids, Chung-Lu and web-shaped graphs, a star), BFS advances level
by level with the alpha/beta rule; before every level each strategy
(gb_strategy: top-down edge-balanced with 1/2/4 edges per thread, top-down
warp per vertex, bottom-up) is run from the same device state and timed on
the device (gb_bfs_profile_levels).  Rows: the level's features and the five
times.
train: the MLP (8 features -> 32 -> 32 -> 5 predicted log2 us) is fitted with
the library's GPU training kernels (gb_mlp_train, Adam) and written to
selector_single.npy beside this file, where GpuBfs users and bench.py find it.
--seed picks the initial weights and the minibatch order (default 0); the
shipped selector_single.npy was trained with --seed 1.
evaluate: learned vs rule persistent BFS on held-out graphs (same depths).

Every handle uses the hub-first adjacency layout (GpuBfs.hub_first), the one
bench.py and gbench --hub-first run with; --natural keeps the caller's order.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(PKG))
import graph_analytics_applesilicon_b200 as G  # noqa: E402


HUB_FIRST = "--natural" not in sys.argv


def handle(g):
    """A BFS handle with the layout the selector is trained for."""
    bfs = G.GpuBfs(g)
    return bfs.hub_first() if HUB_FIRST else bfs


def training_graphs():
    """(name, graph) pairs; seeds differ from every benchmark graph's."""
    out = []
    for scale, ef, seed in ((16, 16, 101), (18, 8, 102), (18, 32, 103), (20, 4, 104), (20, 16, 105), (21, 8, 106)):
        g = G.gen.rmat(scale, ef, False, seed)
        out.append((f"rmat{scale}_ef{ef}", G.permute(g, G.random_perm(g.n, seed))))
    for rows, seed in ((300, 201), (700, 202), (1000, 203)):
        out.append((f"road{rows}", G.gen.road(rows, rows, 0.04, 0.005, seed)))
    for n, deg, seed in ((200000, 20.0, 301), (500000, 60.0, 302)):
        out.append((f"chunglu{n}_{int(deg)}", G.gen.chung_lu(n, 2.2, deg, seed)))
    out.append(("web300k_sym", G.symmetrize(G.gen.web(300000, 5.8, 2.1, 401))))
    out.append(("star200k", G.gen.star(200000)))
    out.append(("grid300", G.gen.grid2d(300, 300)))
    return out


def heldout_graphs():
    out = []
    g = G.gen.rmat(19, 16, False, 901)
    out.append(("rmat19_ef16", G.permute(g, G.random_perm(g.n, 9))))
    out.append(("road500", G.gen.road(500, 500, 0.04, 0.005, 902)))
    out.append(("chunglu300k", G.gen.chung_lu(300000, 2.2, 40.0, 903)))
    return out


def generate_batch(path, batches_per_graph=2, repeats=2, max_rows_per_batch=400):
    """Rows for the 64-source batched kernel (each strategy forced for the whole
    batch; every level's time is read from the device trace)."""
    feats, times, tags = [], [], []
    for name, g in training_graphs():
        t0 = time.time()
        bfs = handle(g)
        for b in range(batches_per_graph):
            srcs = G.pick_sources(g, 64, 11 + b)
            f, t = bfs.profile_batch_levels(srcs, repeats=repeats)
            if len(f) > max_rows_per_batch:
                keep = np.linspace(0, len(f) - 1, max_rows_per_batch).astype(int)
                f, t = f[keep], t[keep]
            feats.append(f)
            times.append(t)
            tags += [name] * len(f)
        bfs.close()
        print(f"{name}: rows so far {sum(len(x) for x in feats)} ({time.time() - t0:.1f}s)", flush=True)
    np.savez_compressed(path, feats=np.concatenate(feats), times=np.concatenate(times), tags=np.array(tags))


def save_params(p, out_path):
    np.save(out_path, p)
    p.astype(np.float32).tofile(os.path.splitext(out_path)[0] + ".bin")  # raw float32 for C++ callers


def generate(path, sources_per_graph=3, repeats=3, max_rows_per_source=400):
    feats, times, tags = [], [], []
    for name, g in training_graphs():
        t0 = time.time()
        bfs = handle(g)
        for s in G.pick_sources(g, sources_per_graph, 7):
            f, t = bfs.profile_levels(int(s), repeats=repeats)
            if len(f) > max_rows_per_source:  # long-diameter graphs: keep an even sample of levels
                keep = np.linspace(0, len(f) - 1, max_rows_per_source).astype(int)
                f, t = f[keep], t[keep]
            feats.append(f)
            times.append(t)
            tags += [name] * len(f)
        bfs.close()
        print(f"{name}: n={g.n} m={g.m} rows so far {sum(len(x) for x in feats)} ({time.time() - t0:.1f}s)",
              flush=True)
    np.savez_compressed(path, feats=np.concatenate(feats), times=np.concatenate(times), tags=np.array(tags))


def init_params(seed=0):
    nf, nh, no = G.selector_shape()
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, np.sqrt(2 / nf), (nh, nf))
    w2 = rng.normal(0, np.sqrt(2 / nh), (nh, nh))
    w3 = rng.normal(0, np.sqrt(1 / nh), (no, nh))
    p = np.concatenate([w1.ravel(), np.zeros(nh), w2.ravel(), np.zeros(nh), w3.ravel(), np.full(no, 5.0)])
    return p.astype(np.float32)


def train(data_path, out_path=None, epochs=600, batch=128, lr=3e-3, seed=0):
    d = np.load(data_path)
    x = d["feats"].astype(np.float32)
    t = np.maximum(d["times"].astype(np.float64), 0.5)
    y = np.log2(t).astype(np.float32)
    mask = np.isfinite(y).astype(np.float32) * (d["times"] < 1e20)
    y = np.where(mask > 0, y, 0).astype(np.float32)
    if "tags" in d.files:
        # every training graph weighs the same: a long-diameter graph gives
        # hundreds of levels, a power-law graph a dozen
        tags = d["tags"]
        names, inv, counts = np.unique(tags, return_inverse=True, return_counts=True)
        w = (len(tags) / len(names)) / counts[inv]
        mask = mask * w[:, None].astype(np.float32)
    p = init_params(seed)
    loss = G.C.c_float(0)
    G.check(G.lib().gb_mlp_train(p, len(x), np.ascontiguousarray(x), np.ascontiguousarray(y),
                                 np.ascontiguousarray(mask.astype(np.float32)), epochs, batch, lr, seed,
                                 G.C.byref(loss)))
    out = np.zeros((len(x), y.shape[1]), np.float32)
    G.check(G.lib().gb_mlp_forward(p, len(x), np.ascontiguousarray(x), out))
    pick = out.argmin(1)
    best = t.argmin(1)
    regret = (t[np.arange(len(t)), pick].sum() / t[np.arange(len(t)), best].sum())
    print(f"train: rows={len(x)} final mse(log2 us)={loss.value:.4f} "
          f"oracle-pick rate={np.mean(pick == best):.3f} time(picked)/time(best)={regret:.3f}")
    out_path = out_path or os.path.join(PKG, "selector_single.npy")
    save_params(p, out_path)
    return p


def evaluate(params_path=None, sources=8):
    p = np.load(params_path) if params_path else G.default_selector_params("single")
    rows = []
    for name, g in heldout_graphs():
        bfs = handle(g)
        bfs.set_selector(p, 0)
        srcs = G.pick_sources(g, sources, 3)
        tt = {}
        for sel in ("rule", "learned"):
            o = G.BfsOptions(selector=sel)
            for s in srcs:  # warm
                bfs.run("gpu_do_persistent", int(s), opts=o)
            ms = []
            for s in srcs:
                d = bfs.run("gpu_do_persistent", int(s), opts=o)
                ms.append(bfs.lastGpuMs())
            tt[sel] = sum(ms)
        rows.append((name, tt["rule"], tt["learned"], tt["rule"] / tt["learned"]))
        print(f"{name}: rule {tt['rule']:.3f} ms, learned {tt['learned']:.3f} ms, gain x{tt['rule'] / tt['learned']:.3f}",
              flush=True)
    return rows


def evaluate_batch(params_path=None, batches=2):
    p = np.load(params_path) if params_path else G.default_selector_params("batch")
    rows = []
    for name, g in heldout_graphs():
        bfs = handle(g)
        bfs.set_selector(p, 1)
        tt = {}
        for sel in ("rule", "learned"):
            o = G.BfsOptions(selector=sel)
            ms = []
            for b in range(batches):
                srcs = G.pick_sources(g, 64, 21 + b)
                bfs.run_batch(srcs, opts=o)
                bfs.run_batch(srcs, opts=o)
                ms.append(bfs.lastGpuMs())
            tt[sel] = sum(ms)
        rows.append((name, tt["rule"], tt["learned"], tt["rule"] / tt["learned"]))
        print(f"batch {name}: rule {tt['rule']:.3f} ms, learned {tt['learned']:.3f} ms, "
              f"gain x{tt['rule'] / tt['learned']:.3f}", flush=True)
    return rows


if __name__ == "__main__":
    sys.argv = [a for a in sys.argv if a != "--natural"]
    seed = 0
    if "--seed" in sys.argv:
        i = sys.argv.index("--seed")
        seed = int(sys.argv[i + 1])
        del sys.argv[i:i + 2]
    cmd = sys.argv[1] if len(sys.argv) > 1 else "evaluate"
    if cmd == "generate":
        generate(sys.argv[2])
    elif cmd == "train":
        train(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else None, seed=seed)
    elif cmd == "generate-batch":
        generate_batch(sys.argv[2])
    elif cmd == "train-batch":
        train(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else os.path.join(PKG, "selector_batch.npy"), seed=seed)
    elif cmd == "evaluate-batch":
        evaluate_batch(sys.argv[2] if len(sys.argv) > 2 else None)
    else:
        evaluate(sys.argv[2] if len(sys.argv) > 2 else None)
