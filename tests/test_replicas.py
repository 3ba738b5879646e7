"""Multi-GPU replica logic on CPU: two gloo ranks shard a query stream, each
answers its shard with the oracle, and the combined checksum and the
max-over-ranks time equal those of one process answering everything."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from exclucene_b200 import replicas, synth


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        w = synth.zipf_corpus(seed=13, ndocs=1 << 16, nterms=300, cap=20_000, nq=301, qmin=1, qmax=5)
        t, o, q0, q1 = replicas.shard_queries(w.terms, w.term_offsets, rank, world)
        offs, docs = oracle.answer(w.docs, w.list_offsets, t, o)
        cs = replicas.gather_checksums(oracle.checksum(offs, docs))
        slowest = replicas.max_over_ranks(1.5 + rank)
        out.put((rank, q0, q1, cs, slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_combine_to_single_run():
    from exclucene_b200 import synth as _s  # noqa: F401  (library loads in the parent too)
    import oracle

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    w = synth.zipf_corpus(seed=13, ndocs=1 << 16, nterms=300, cap=20_000, nq=301, qmin=1, qmax=5)
    offs, docs = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    want = oracle.checksum(offs, docs)
    # shards tile the stream, both ranks see the combined checksum and the slowest time
    assert res[0][1] == 0 and res[0][2] == res[1][1] and res[1][2] == w.nq
    for _, _, _, cs, slowest in res:
        assert tuple(cs) == tuple(want)
        assert slowest == 2.5


def test_shard_queries_partitions():
    terms = np.arange(20, dtype=np.uint32)
    toff = np.array([0, 2, 5, 5, 9, 14, 20], dtype=np.uint32)
    parts = [replicas.shard_queries(terms, toff, r, 4) for r in range(4)]
    assert [p[2] for p in parts] == [0, 1, 3, 4] and [p[3] for p in parts] == [1, 3, 4, 6]
    joined = np.concatenate([p[0] for p in parts])
    assert np.array_equal(joined, terms)
    for t, o, q0, q1 in parts:
        assert o[0] == 0 and len(o) == q1 - q0 + 1 and o[-1] == len(t)
    assert replicas.combine_checksums([(1, 2, 3), (4, 5, 6)]) == (5, 7, 3 ^ 6)
