"""excl_submit_into: the zero-copy host path (results written by the last
kernel straight into the caller's page-locked arrays) gives the oracle's
output, keeps each in-flight batch's error flags to itself, and rejects
output arrays that the device cannot write."""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def corpus():
    return synth.zipf_corpus(seed=91, ndocs=1 << 20, nterms=2000, cap=150_000, nq=2000, qmin=1, qmax=5)


@pytest.fixture(scope="module")
def expected(corpus):
    return oracle.answer(corpus.docs, corpus.list_offsets, corpus.terms, corpus.term_offsets)


def _pinned_copy(a):
    p = ex.pinned_empty(len(a))
    p[:] = a
    return p


@pytest.mark.parametrize("codec", ["parapfd", "seglrc", "hs_parapfd", "newpfd"])
@pytest.mark.parametrize("graphs", [False, True])
def test_matches_oracle(corpus, expected, codec, graphs):
    ctx = ex.Context(0, max_queries=8192, max_keys=1 << 23, use_graphs=graphs)
    kb = 10 if codec == "hs_parapfd" else 0
    ix = ex.Index(corpus.docs, corpus.list_offsets, codec=codec, block=128, frac=0.1, hs_bucket=256, hs_kbits=kb)
    ctx.upload(ix)
    eoffs, edocs = expected
    terms, toff = _pinned_copy(corpus.terms), _pinned_copy(corpus.term_offsets)
    offs = ex.pinned_empty(corpus.nq + 1)
    docs = ex.pinned_empty(len(edocs) + 64)
    try:
        for _ in range(3):  # uncaptured, captured, replayed when graphs are on
            offs[:] = 0xFFFFFFFF
            docs[:] = 0xFFFFFFFF
            b = ctx.submit_into(ix, terms, toff, offs, docs, "auto")
            tot = b.wait()
            b.free()
            assert tot == len(edocs)
            assert np.array_equal(offs.astype(np.uint64), eoffs)
            assert np.array_equal(docs[:tot], edocs)
            assert np.all(docs[tot:] == 0xFFFFFFFF)
    finally:
        ix.close()
        ctx.close()


def test_batches_in_flight_keep_their_own_results_and_flags(corpus, expected):
    ctx = ex.Context(0, max_queries=8192, max_keys=1 << 23)
    ix = ex.Index(corpus.docs, corpus.list_offsets, codec="seglrc", block=256)
    ctx.upload(ix)
    eoffs, edocs = expected
    toff = corpus.term_offsets
    cuts = [(0, 700), (700, 701), (701, 2000)]
    try:
        bufs, batches = [], []
        for i, (q0, q1) in enumerate(cuts):
            t = corpus.terms[toff[q0]:toff[q1]].copy()
            o = (toff[q0:q1 + 1] - toff[q0]).astype(np.uint32)
            if i == 1:
                t[:] = corpus.nlists + 3  # an unknown term id: this batch alone fails
            n = int(eoffs[q1] - eoffs[q0])
            ob, db = ex.pinned_empty(len(o)), ex.pinned_empty(n + 1)
            bufs.append((t, o, ob, db))
            batches.append(ctx.submit_into(ix, t, o, ob, db, "hashseg"))  # pageable inputs
        for i, ((q0, q1), b) in enumerate(zip(cuts, batches)):
            if i == 1:
                with pytest.raises(ex.ExclError) as e:
                    b.wait()
                assert e.value.status == ex.api.E_INVALID
            else:
                tot = b.wait()
                _, _, ob, db = bufs[i]
                assert np.array_equal(ob.astype(np.uint64), eoffs[q0:q1 + 1] - eoffs[q0])
                assert np.array_equal(db[:tot], edocs[eoffs[q0]:eoffs[q1]])
            b.free()
    finally:
        ix.close()
        ctx.close()


def test_capacity_and_rejected_outputs(corpus, expected):
    ctx = ex.Context(0, max_queries=8192, max_keys=1 << 23)
    ix = ex.Index(corpus.docs, corpus.list_offsets, codec="parapfd", block=256)
    ctx.upload(ix)
    eoffs, edocs = expected
    terms, toff = corpus.terms, corpus.term_offsets
    offs = ex.pinned_empty(corpus.nq + 1)
    try:
        # too small a result array: the first cap docIDs are written, the wait reports capacity
        cap = len(edocs) // 2
        small = ex.pinned_empty(cap)
        b = ctx.submit_into(ix, terms, toff, offs, small)
        with pytest.raises(ex.ExclError) as e:
            b.wait()
        assert e.value.status == ex.api.E_CAPACITY
        b.free()
        assert np.array_equal(small, edocs[:cap])
        # pageable output arrays are refused before any work
        with pytest.raises(ex.ExclError) as e:
            ctx.submit_into(ix, terms, toff, np.zeros(corpus.nq + 1, np.uint32), small)
        assert e.value.status == ex.api.E_INVALID
        # the context is still good
        docs = ex.pinned_empty(len(edocs))
        b = ctx.submit_into(ix, terms, toff, offs, docs)
        assert b.wait() == len(edocs)
        b.free()
        assert np.array_equal(docs, edocs)
    finally:
        ix.close()
        ctx.close()


def test_threads_share_a_context(corpus, expected):
    """Four host threads submit zero-copy batches on one context at once; each
    gets its own results. An excl_submit batch superseded by a later one is
    refused rather than answered with the later batch's results."""
    import threading

    ctx = ex.Context(0, max_queries=8192, max_keys=1 << 23)
    ix = ex.Index(corpus.docs, corpus.list_offsets, codec="seglrc", block=256)
    ctx.upload(ix)
    eoffs, edocs = expected
    toff = corpus.term_offsets
    errors = []

    def worker(k):
        try:
            rng = np.random.default_rng(k)
            for _ in range(6):
                q0 = int(rng.integers(0, corpus.nq - 50))
                q1 = q0 + int(rng.integers(1, 50))
                t = _pinned_copy(corpus.terms[toff[q0]:toff[q1]])
                o = _pinned_copy((toff[q0:q1 + 1] - toff[q0]).astype(np.uint32))
                ob = ex.pinned_empty(q1 - q0 + 1)
                db = ex.pinned_empty(int(eoffs[q1] - eoffs[q0]) + 1)
                b = ctx.submit_into(ix, t, o, ob, db, "hashseg")
                tot = b.wait()
                b.free()
                assert np.array_equal(ob.astype(np.uint64), eoffs[q0:q1 + 1] - eoffs[q0])
                assert np.array_equal(db[:tot], edocs[eoffs[q0]:eoffs[q1]])
        except Exception as e:  # reported below
            errors.append(e)

    try:
        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        assert not errors, errors
        # excl_submit: the older batch's results were replaced by the newer one's
        b1 = ctx.submit(ix, corpus.terms[:int(toff[10])], toff[:11], "hashseg")
        b2 = ctx.submit(ix, corpus.terms[:int(toff[20])], toff[:21], "hashseg")
        with pytest.raises(ex.ExclError) as e:
            b1.wait()
        assert e.value.status == ex.api.E_INVALID
        offs, docs = b2.wait()
        assert np.array_equal(docs, edocs[:int(eoffs[20])])
        b1.free()
        b2.free()
    finally:
        ix.close()
        ctx.close()
