"""The multi-rank path on CPU: two gloo ranks each evaluate their program
range (with the oracle standing in for the GPU evaluator) and gather the
fitness vector; it must equal a single-process evaluation bit for bit."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from galop_b200 import workloads as W
    from sharding import evaluate_sharded
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl = W.single_generation(seed=5, n_programs=301, n_cases=200)
        o = Oracle(0, 16)
        fit = evaluate_sharded(lambda w, off: o.evaluate_csr(w, off, wl.X, wl.y, threads=1),
                               wl.words, wl.offsets, rank, world)
        if rank == 0:
            np.save(out_path, fit)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_everything():
    from sharding import shard_bounds
    for n in (0, 1, 7, 1000, 1023):
        for world in (1, 2, 3, 8):
            b = [shard_bounds(n, r, world) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            assert max(h - l for l, h in b) - min(h - l for l, h in b) <= 1


def test_two_gloo_ranks_gather_matches_single_process(tmp_path):
    from galop_b200 import workloads as W
    from oracle.oracle import Oracle
    out = tmp_path / "fit.npy"
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(out))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = np.load(out)
    wl = W.single_generation(seed=5, n_programs=301, n_cases=200)
    want = Oracle(0, 16).evaluate_csr(wl.words, wl.offsets, wl.X, wl.y, threads=1)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
