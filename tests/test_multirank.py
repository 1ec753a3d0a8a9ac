"""Multi-process plumbing of the benchmark on CPU (gloo, two ranks).

The route is replicated per GPU: every rank processes its own corpus and only
the timing crosses ranks (a barrier and a max over the measured times).  This
checks that plumbing with two CPU ranks: the max over ranks, distinct
per-rank corpora, and that only rank 0 reports.
"""
import json
import os
import socket
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    dist = bench.Dist(backend="gloo")
    dist.barrier()
    slowest = dist.max(10.0 + rank)
    images = bench.make_corpus(0, 2, bench.corpus_seed_base(rank), "cpu")
    digest = [int(im.to(dtype=torch.int64).sum()) for im in images]
    dist.barrier()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"max": slowest, "digest": digest,
                   "reports": dist.rank == 0}, f)
    dist.close()


def test_two_gloo_ranks(tmp_path):
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=worker, args=(r, 2, port, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert res[0]["max"] == res[1]["max"] == 11.0
    assert res[0]["digest"] != res[1]["digest"]
    assert res[0]["reports"] and not res[1]["reports"]
