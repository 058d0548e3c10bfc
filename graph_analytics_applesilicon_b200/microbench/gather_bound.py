"""Gather-rate bound of one PageRank sweep on the Chung-Lu PageRank workload
(3.07M vertices, degree exponent 2.2, mean degree 76, seed 307; 232.5M in-edges).

Times, on cuda:0, the kernels of gather_bound.cu over the graph's in-lists in the
degree-adaptive pull's order (vertices by descending in-degree, each list
sorted) and in the generator's order, beside the library's own gpu_pull_adaptive
(autotuned, as the benchmark runs it) and gpu_pull_blocked, then under four vertex
orderings (in-degree, RCM and their mixes).  Every figure is the
minimum over repeats of CUDA-event time, each run after a 256 MB buffer write
that flushes L2.  Run from the repository root on a machine with a GPU:

    python graph_analytics_applesilicon_b200/microbench/gather_bound.py

The shared library is compiled on first use next to this file with
    nvcc -shared -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a -O3 \
        -o libgather_bound.so gather_bound.cu
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import graph_analytics_applesilicon_b200 as G  # noqa: E402


def load_probe():
    so = os.path.join(HERE, "libgather_bound.so")
    src = os.path.join(HERE, "gather_bound.cu")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["nvcc", "-shared", "-Xcompiler", "-fPIC", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-O3", "-o", so, src], check=True)
    lib = C.CDLL(so)
    lib.gb_gather_probe.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32,
                                    C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    return lib


def main():
    lib = load_probe()
    g = G.gen.chung_lu(3070000, 2.2, 76.0, 307)
    n, m = g.n, g.m
    pr = G.GpuPageRank(g.n, g, g, g.degrees())
    o = pr.autotune(G.PrOptions(iters=20))
    lines = []
    for v, opts in (("gpu_pull_adaptive", o), ("gpu_pull_blocked", G.PrOptions(iters=20))):
        pr.run(v, opts)
        t = min(pr.run(v, opts).gpu_ms for _ in range(3)) / 20
        lines.append((f"library {v}", t))
    del pr

    dev = torch.device("cuda:0")
    rp = torch.from_numpy(g.row_ptr.astype(np.int64)).to(dev)
    ci = torch.from_numpy(g.col_idx.astype(np.int64)).to(dev)
    deg = rp[1:] - rp[:-1]
    order = torch.sort(-deg, stable=True).indices
    perm = torch.empty_like(order)
    perm[order] = torch.arange(n, device=dev)
    rows = torch.repeat_interleave(torch.arange(n, device=dev), deg)
    key = torch.sort((perm[rows] << 32) | perm[ci]).values
    col_sorted = (key & 0xFFFFFFFF).to(torch.int32).contiguous()
    share = {h: float((col_sorted < h).double().mean()) for h in (4096, 16384, 32768, 49152)}
    col_gen = ci.to(torch.int32).contiguous()
    del key, rows, rp, ci, perm, order
    contrib = torch.rand(n, device=dev, dtype=torch.float32)
    out = torch.zeros(1, device=dev)
    nvec = m // 4
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sms = torch.cuda.get_device_properties(0).multi_processor_count

    def run(kind, col, h=0, blocks=2 * sms, threads=1024, words=nvec):
        ts = []
        for _ in range(5):
            flush.zero_()
            out.zero_()
            e0.record()
            rc = lib.gb_gather_probe(kind, col.data_ptr(), words, contrib.data_ptr(), n, h, out.data_ptr(), blocks,
                                     threads, st)
            e1.record()
            torch.cuda.synchronize()
            if rc != 0:
                raise RuntimeError(f"probe kind {kind} failed: {rc}")
            ts.append(e0.elapsed_time(e1))
        return min(ts[2:])

    lines.append(("edge gather, adaptive-pull order", run(0, col_sorted)))
    lines.append(("edge gather, generator order", run(0, col_gen)))
    lines.append(("uniform random ids, same count", run(2, col_sorted)))
    for h in (16384, 32768, 49152):
        lines.append((f"edge gather, ids < {h} from shared memory", run(1, col_sorted, h=h, blocks=sms)))
    print(f"Chung-Lu n={n} m={m}; gathers hitting the first 4K/16K/32K/48K ids: "
          + " / ".join(f"{share[h]:.3f}" for h in sorted(share)))
    for label, t in lines:
        print(f"{label:48s} {t:.4f} ms per sweep = {4 * nvec / t / 1e6 if 'library' not in label else m / t / 1e6:7.1f}"
              f" G gathers/s")
    # the same uniform gathers as a short kernel: 2 blocks of 1024 threads per SM, 256 gathers each
    short = 2 * sms * 1024 * 256 // 4
    t = run(2, col_sorted, words=short)
    print(f"{'uniform random ids, 256 per thread (short)':48s} {t:.4f} ms = {4 * short / t / 1e6:7.1f} G gathers/s")
    del col_sorted, col_gen

    # vertex orderings: does any recover locality beyond the degree skew?
    rp = torch.from_numpy(g.row_ptr.astype(np.int64)).to(dev)
    ci = torch.from_numpy(g.col_idx.astype(np.int64)).to(dev)
    deg = rp[1:] - rp[:-1]
    rows = torch.repeat_interleave(torch.arange(n, device=dev), deg)
    rcm = torch.from_numpy(G.reorder_gpu(g, "rcm").astype(np.int64)).to(dev)  # perm[old] = new

    def rank_of(keys):
        order = torch.sort(keys, stable=True).indices
        p = torch.empty_like(order)
        p[order] = torch.arange(n, device=dev)
        return p

    cls = torch.clamp(torch.floor(torch.log2(deg.clamp(min=1).double())).long(), 0, 30)
    for label, p in (("in-degree descending", rank_of(-deg)), ("rcm", rcm),
                     ("in-degree descending, rcm within", rank_of(-deg * (1 << 23) + rcm)),
                     ("power-of-two classes, rcm within", rank_of((30 - cls) * (1 << 23) + rcm))):
        col = (torch.sort((p[rows] << 32) | p[ci]).values & 0xFFFFFFFF).to(torch.int32).contiguous()
        t0, t1 = run(0, col), run(1, col, h=32768, blocks=sms)
        print(f"order {label:36s} ideal {4 * nvec / t0 / 1e6:6.1f} G/s, ids < 32768 in shared memory "
              f"{4 * nvec / t1 / 1e6:6.1f} G/s")
        del col


if __name__ == "__main__":
    main()
