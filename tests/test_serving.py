"""Serving loop (continuous batching) on the GPU: every query's result equals
the oracle's, whether it ran alone or batched with others that arrived while
earlier batches were on the device; admission keeps the working set inside
the HBM budget; invalid and oversize queries fail without stopping the rest."""
import threading

import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(gpu_ctx):
    w = synth.zipf_corpus(seed=91, ndocs=1 << 20, nterms=2000, cap=150_000, nq=1500, qmin=1, qmax=8)
    ix = ex.Index(w.docs, w.list_offsets, codec="seglrc", block=256)
    gpu_ctx.upload(ix)
    eoffs, edocs = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    want = [edocs[eoffs[q]:eoffs[q + 1]] for q in range(w.nq)]
    yield w, ix, want
    ix.close()


def _q(w, q):
    return w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]


@pytest.mark.parametrize("algo", ["hashseg", "auto"])
def test_alone_equals_mixed_equals_oracle(served, algo):
    w, ix, want = served
    srv = ex.Server(ix, slots=3, max_batch_queries=64, max_batch_keys=1 << 20, algo=algo)
    try:
        # alone: each query waited for before the next is submitted (batches of one)
        alone = [srv.wait(srv.submit(_q(w, q))) for q in range(200)]
        # mixed: four threads submit concurrently; later arrivals join batches
        # while earlier ones are still on the device
        tickets = {}
        lock = threading.Lock()

        def producer(part):
            for q in range(part, w.nq, 4):
                t = srv.submit(_q(w, q))
                with lock:
                    tickets[q] = t

        ths = [threading.Thread(target=producer, args=(i,)) for i in range(4)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        mixed = {q: srv.wait(t) for q, t in tickets.items()}
        st = srv.stats()
    finally:
        srv.close()
    for q in range(200):
        assert np.array_equal(alone[q], want[q]), q
        assert np.array_equal(mixed[q], alone[q]), q
    for q in range(w.nq):
        assert np.array_equal(mixed[q], want[q]), q
    assert st["completed"] == 200 + w.nq
    assert st["batches"] < st["completed"]  # queries were batched together
    assert st["p99_us"] >= st["p50_us"] > 0


def test_replay_poisson_checksum(served):
    w, ix, want = served
    srv = ex.Server(ix, slots=4, max_batch_queries=256)
    try:
        rng = np.random.default_rng(5)
        arrival = np.cumsum(rng.exponential(1.0 / 50_000, w.nq))  # 50k queries/s
        lat, cs, wall = srv.replay(w.terms, w.term_offsets, arrival)
        st = srv.stats()
    finally:
        srv.close()
    eoffs = np.concatenate([[0], np.cumsum([len(x) for x in want])]).astype(np.uint64)
    edocs = np.concatenate(want) if want else np.zeros(0, np.uint32)
    assert cs == oracle.checksum(eoffs, edocs)
    assert np.all(lat > 0) and wall >= arrival[-1]
    assert st["completed"] == w.nq


def test_admission_budget_and_rejection(served):
    w, ix, want = served
    lens = np.diff(w.list_offsets)
    big = int(np.argmax(lens))
    # the pool holds the longest list's docIDs (4 B each) but not that plus the
    # rest of a one-term query's working set, and only a few of the queries below
    budget = 4 * int(lens[big])
    qs = [q for q in range(w.nq) if len(_q(w, q)) and lens[_q(w, q)].min() <= 20_000][:400]
    assert len(qs) == 400
    srv = ex.Server(ix, slots=4, max_batch_queries=32, max_batch_keys=1 << 18, hbm_budget_bytes=budget)
    try:
        tb = srv.submit([big])
        ts = [srv.submit(_q(w, q)) for q in qs]
        got = [srv.wait(t) for t in ts]
        with pytest.raises(ex.ExclError) as e:
            srv.wait(tb)
        assert e.value.status == ex.api.E_CAPACITY
        st = srv.stats()
    finally:
        srv.close()
    for i, q in enumerate(qs):
        assert np.array_equal(got[i], want[q]), q
    assert st["pool_peak_bytes"] <= budget
    assert st["rejected"] == 1


def test_invalid_query_is_refused(served):
    w, ix, want = served
    srv = ex.Server(ix, slots=1)
    try:
        with pytest.raises(ex.ExclError):
            srv.submit([ix.nlists + 5])
        with pytest.raises(ex.ExclError):
            srv.submit(list(range(33)))
        assert np.array_equal(srv.wait(srv.submit(_q(w, 3))), want[3])
        assert len(srv.wait(srv.submit([]))) == 0
    finally:
        srv.close()
