"""GPU parity: device decode and batched AND intersection of every format and
search method against the CPU oracle, bit for bit, through the C ABI."""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth

pytestmark = pytest.mark.gpu

FORMATS = ["parapfd", "lrc", "lrcseg", "seglrc", "hs_seglrc", "hs_parapfd", "newpfd"]
DGAP = ("parapfd", "newpfd")  # exercised with FRAC 0.1 and 128-entry blocks (exceptions)
ALGOS = ["bsearch", "hashseg", "segreg", "auto"]


def _index(w, codec, block=256, frac=0.0, ubits=24):
    kb = 10 if codec == "hs_parapfd" else 0
    return ex.Index(w.docs, w.list_offsets, codec=codec, block=block, frac=frac, hs_bucket=256, hs_kbits=kb,
                    hs_ubits=ubits)


@pytest.fixture(scope="module")
def corpus():
    # Zipf-frequency corpus in the shape of the multi-term workload, scaled down
    return synth.zipf_corpus(seed=77, ndocs=1 << 20, nterms=3000, cap=200_000, nq=3000, qmin=1, qmax=6)


@pytest.fixture(scope="module")
def expected(corpus):
    return oracle.answer(corpus.docs, corpus.list_offsets, corpus.terms, corpus.term_offsets)


@pytest.mark.parametrize("codec", FORMATS)
@pytest.mark.parametrize("block,frac", [(256, 0.0), (128, 0.1)])
def test_decode_matches_source_lists(gpu_ctx, corpus, codec, block, frac):
    ix = _index(corpus, codec, block, frac)
    gpu_ctx.upload(ix)
    got = gpu_ctx.decode_lists(ix)
    assert np.array_equal(got, corpus.docs)
    # a sub-range of lists
    l0, l1 = 17, 401
    got = gpu_ctx.decode_lists(ix, l0, l1)
    assert np.array_equal(got, corpus.docs[corpus.list_offsets[l0]:corpus.list_offsets[l1]])
    ix.close()


@pytest.mark.parametrize("codec", FORMATS)
@pytest.mark.parametrize("algo", ALGOS)
def test_intersection_matches_oracle(gpu_ctx, corpus, expected, codec, algo):
    ix = _index(corpus, codec, 128 if codec in DGAP else 256, 0.1 if codec in DGAP else 0.0)
    gpu_ctx.upload(ix)
    offs, docs = gpu_ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo=algo)
    eoffs, edocs = expected
    assert np.array_equal(offs.astype(np.uint64), eoffs)
    assert np.array_equal(docs, edocs)
    assert ex.checksum(offs, docs) == oracle.checksum(eoffs, edocs)
    ix.close()


def test_edge_case_queries(gpu_ctx):
    lists = [np.array([5], np.uint32),                               # 0 single posting
             np.arange(0, 3000, 3, dtype=np.uint32),                   # 1
             np.arange(1, 3000, 3, dtype=np.uint32),                   # 2 disjoint from 1
             np.arange(0, 600000, 2, dtype=np.uint32),                 # 3 long
             np.array([0, 2 ** 31 - 1, 2 ** 32 - 8], np.uint32),       # 4 extremes (gaps < 2^31)
             np.arange(2 ** 31 - 1000, 2 ** 31 + 1000, 7, dtype=np.uint32),  # 5 around 2^31
             np.arange(0, 256, dtype=np.uint32),                       # 6 exactly one block
             np.arange(0, 257, dtype=np.uint32)]                       # 7 one block + 1
    docs = np.concatenate(lists)
    loff = np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.uint64)
    queries = [[], [0], [1], [1, 2], [1, 3], [3, 1], [3, 3], [0, 3, 1], [4, 4], [4, 3], [5], [5, 5, 5],
               [6, 7], [7, 6, 1, 3], list(range(8)), [3] * 32, [1, 3, 6, 7, 3, 1]]
    terms = np.array([t for q in queries for t in q], np.uint32)
    toff = np.concatenate([[0], np.cumsum([len(q) for q in queries])]).astype(np.uint32)
    eoffs, edocs = oracle.answer(docs, loff, terms, toff)
    for codec in FORMATS:
        if codec == "lrc":
            continue  # docIDs near 2^32 are beyond LRC's int arithmetic
        ix = ex.Index(docs, loff, codec=codec, block=256, hs_bucket=64, hs_kbits=12 if codec == "hs_parapfd" else 0,
                      hs_ubits=32)
        gpu_ctx.upload(ix)
        for algo in ALGOS:
            offs, got = gpu_ctx.intersect(ix, terms, toff, algo=algo)
            assert np.array_equal(offs.astype(np.uint64), eoffs), (codec, algo)
            assert np.array_equal(got, edocs), (codec, algo)
        ix.close()


def test_invalid_batches_raise(gpu_ctx, corpus):
    ix = _index(corpus, "parapfd")
    gpu_ctx.upload(ix)
    with pytest.raises(ex.ExclError):
        gpu_ctx.intersect(ix, np.array([corpus.nlists + 5], np.uint32), np.array([0, 1], np.uint32))
    with pytest.raises(ex.ExclError):
        gpu_ctx.intersect(ix, np.zeros(33, np.uint32), np.array([0, 33], np.uint32))
    # the context stays usable
    offs, docs = gpu_ctx.intersect(ix, corpus.terms[:10], corpus.term_offsets[:4] - corpus.term_offsets[0])
    eo, ed = oracle.answer(corpus.docs, corpus.list_offsets, corpus.terms[:10], corpus.term_offsets[:4])
    assert np.array_equal(docs, ed)
    ix.close()


def test_tile_overflow_reports_capacity(corpus):
    """A batch with more tiles (and shortest-list docIDs) than a small context
    holds fails with EXCL_E_CAPACITY: the pack phase's work order then covers
    only the tiles that fit, and nothing runs past the buffers. The context
    answers the next batch exactly."""
    ix = _index(corpus, "seglrc")
    ctx = ex.Context(0, max_queries=8, max_keys=2048)  # room for 2048/32 + 8 + 1 = 73 tiles
    try:
        ctx.upload(ix)
        lens = np.diff(corpus.list_offsets).astype(np.int64)
        order = np.argsort(lens, kind="stable")
        longest = order[::-1][:4].astype(np.uint32)  # two pairs of the longest lists: hundreds of tiles each
        assert lens[longest].min() > 256 * 80
        with pytest.raises(ex.ExclError) as e:
            ctx.intersect(ix, longest, np.array([0, 2, 4], np.uint32))
        assert e.value.status == ex.api.E_CAPACITY
        short = order[(lens[order] > 0) & (lens[order] <= 400)][:4].astype(np.uint32)
        toff = np.array([0, 2, 4], np.uint32)
        offs, docs = ctx.intersect(ix, short, toff)
        eo, ed = oracle.answer(corpus.docs, corpus.list_offsets, short, toff)
        assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(docs, ed)
    finally:
        ctx.close()
        ix.close()


def test_batching_does_not_change_results(gpu_ctx, corpus, expected):
    ix = _index(corpus, "seglrc")
    gpu_ctx.upload(ix)
    eoffs, edocs = expected
    toff = corpus.term_offsets
    for q0, q1 in [(0, 1), (5, 6), (100, 357), (1000, 3000)]:
        t = corpus.terms[toff[q0]:toff[q1]]
        o = (toff[q0:q1 + 1] - toff[q0]).astype(np.uint32)
        offs, docs = gpu_ctx.intersect(ix, t, o)
        exp = edocs[eoffs[q0]:eoffs[q1]]
        assert np.array_equal(docs, exp)
        assert np.array_equal(offs.astype(np.uint64), eoffs[q0:q1 + 1] - eoffs[q0])
    ix.close()


def test_graph_replay_matches_oracle(corpus, expected):
    """A context that replays its batches as CUDA graphs gives the same output
    on every replay, and recaptures when the batch or the method changes."""
    import torch

    gctx = ex.Context(0, max_queries=65536, max_keys=1 << 24, use_graphs=True)
    ix = _index(corpus, "seglrc")
    gctx.upload(ix)
    dev = torch.device("cuda", 0)
    eoffs, edocs = expected
    try:
        for nq, algo in [(corpus.nq, "hashseg"), (1000, "hashseg"), (corpus.nq, "bsearch"), (1000, "hashseg")]:
            n_terms = int(corpus.term_offsets[nq])
            d_terms = torch.from_numpy(corpus.terms[:n_terms].astype(np.int32)).to(dev)
            d_toff = torch.from_numpy(corpus.term_offsets[:nq + 1].astype(np.int32)).to(dev)
            cap = int(eoffs[nq]) + 16
            d_offs = torch.empty(nq + 1, dtype=torch.int32, device=dev)
            d_docs = torch.empty(cap, dtype=torch.int32, device=dev)
            for _ in range(3):  # first run uncaptured, then captured, then replayed
                d_offs.fill_(-1)
                d_docs.fill_(-1)
                torch.cuda.synchronize()  # the context's stream does not wait for torch's
                gctx.intersect_device(ix, d_terms.data_ptr(), d_toff.data_ptr(), nq, algo, d_offs.data_ptr(),
                                      d_docs.data_ptr(), cap)
                gctx.check()
                offs = d_offs.cpu().numpy().astype(np.uint64)
                assert np.array_equal(offs, eoffs[:nq + 1] - eoffs[0])
                assert np.array_equal(d_docs[:int(offs[-1])].cpu().numpy().astype(np.uint32),
                                      edocs[:int(eoffs[nq])])
                assert gctx.stats().total_ms > 0
    finally:
        ix.close()
        gctx.close()


@pytest.mark.parametrize("codec", FORMATS)
@pytest.mark.parametrize("merge", [ex.api.MERGE_OFF, 1, 4])
def test_merge_and_probe_paths_agree(corpus, expected, codec, merge):
    """The shared-memory merge path (tiles whose keys span few segments of a
    longer list) and the per-key probe path give the oracle's output."""
    ctx = ex.Context(0, max_queries=65536, max_keys=1 << 24, merge_segs=merge)
    ix = _index(corpus, codec, 128 if codec in DGAP else 256, 0.1 if codec in DGAP else 0.0)
    ctx.upload(ix)
    eoffs, edocs = expected
    try:
        for algo in ("bsearch", "hashseg"):
            offs, docs = ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo=algo)
            assert np.array_equal(offs.astype(np.uint64), eoffs)
            assert np.array_equal(docs, edocs)
            st = ctx.stats()
            if merge == ex.api.MERGE_OFF:
                assert st.merges == 0
            else:
                assert st.merges > 0
    finally:
        ix.close()
        ctx.close()


def test_autotune_keeps_output_exact(corpus, expected):
    """The autotuner picks a setting no slower than the default on its sample,
    and batches run with the tuned setting still match the oracle."""
    ctx = ex.Context(0, max_queries=65536, max_keys=1 << 24)
    ix = _index(corpus, "seglrc")
    ctx.upload(ix)
    eoffs, edocs = expected
    try:
        rep = ctx.autotune(ix, corpus.terms[:int(corpus.term_offsets[500])], corpus.term_offsets[:501])
        assert rep["tried"] > 10
        assert rep["algo"] in ("bsearch", "hashseg", "segreg", "learned", "auto")
        assert rep["warps_per_cta"] in (4, 8) and rep["ctas_per_sm"] in (4, 5, 6)
        assert 0 < rep["best_ms"] <= rep["default_ms"]
        assert rep["tile_split"] in (0, 1, 2)
        offs, docs = ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo="auto")
        assert np.array_equal(offs.astype(np.uint64), eoffs)
        assert np.array_equal(docs, edocs)
    finally:
        ix.close()
        ctx.close()


@pytest.mark.parametrize("codec", ["parapfd", "seglrc", "hs_parapfd", "newpfd"])
@pytest.mark.parametrize("split", [0, 1, 2])
def test_tile_split_keeps_output_exact(corpus, expected, codec, split):
    """Fixed segments of the shortest lists cut into 2^split tiles (the part's
    keys probed after the whole segment is decoded) give the oracle's output,
    with graphs and merges on; settings out of range are refused."""
    ctx = ex.Context(0, max_queries=65536, max_keys=1 << 24, use_graphs=True)
    ix = _index(corpus, codec, 128 if codec in DGAP else 256, 0.1 if codec in DGAP else 0.0)
    ctx.upload(ix)
    eoffs, edocs = expected
    try:
        for merge in (ex.api.MERGE_OFF, 2):
            ctx.set_tuning(algo="hashseg", warps_per_cta=8, ctas_per_sm=4, merge_segs=merge, tile_split=split)
            for _ in range(2):
                offs, docs = ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo="auto")
                assert np.array_equal(offs.astype(np.uint64), eoffs)
                assert np.array_equal(docs, edocs)
        with pytest.raises(ex.ExclError):
            ctx.set_tuning(tile_split=3)
        with pytest.raises(ex.ExclError):
            ctx.set_tuning(ctas_per_sm=7)
    finally:
        ix.close()
        ctx.close()


@pytest.mark.parametrize("codec", ["parapfd", "seglrc", "newpfd", "lrc", "lrcseg", "hs_seglrc"])
def test_reference_file_set_runs_unchanged(gpu_ctx, tmp_path, codec):
    """A file set written as the reference's compressors write it (blocks from
    its own encoder) loads without re-encoding, decodes to its lists and
    answers its .query stream as the oracle does."""
    import os

    g = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_files.npz")))
    sets = {"parapfd": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".segMedian"),
            "newpfd": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".segMedian"),
            "seglrc": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".ind2_distance_base",
                       ".regression_info", ".regression_info_list"),
            "lrc": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".regression_info"),
            "lrcseg": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".ind2_distance_base",
                       ".regression_info"),
            "hs_seglrc": (".ind1", ".ind2", ".HashSeg_offset", ".HashSeg_info", ".segNum", ".segOffset",
                          ".ind2_distance_base", ".regression_info")}
    for suffix in sets[codec]:
        g[codec + suffix].tofile(os.path.join(tmp_path, "g" + suffix))
    ix = ex.Index.load_reference(str(tmp_path), "g", codec)
    gpu_ctx.upload(ix)
    pre = "hs_" if codec == "hs_seglrc" else ""
    docs = g[pre + "docs"]
    loff = np.concatenate([[0], np.cumsum(g[pre + "lens"].astype(np.uint64))]).astype(np.uint64)
    assert np.array_equal(gpu_ctx.decode_lists(ix), docs)
    if pre:
        q = [[0, 1], [2, 0], [1, 2, 0], [3], [4, 5], [0, 1, 2, 4], [5, 5], [2, 4]]
        terms = np.array([t for x in q for t in x], np.uint32)
        toff = np.concatenate([[0], np.cumsum([len(x) for x in q])]).astype(np.uint32)
    else:
        terms, toff = ex.query_parse(g["queries"].tobytes())
    eoffs, edocs = oracle.answer(docs, loff, terms, toff)
    for algo in ("bsearch", "hashseg"):
        offs, got = gpu_ctx.intersect(ix, terms, toff, algo=algo)
        assert np.array_equal(offs.astype(np.uint64), eoffs)
        assert np.array_equal(got, edocs)
    ix.close()


@pytest.mark.parametrize("block,frac", [(32, 0.64), (128, 0.64), (256, 0.64), (128, 0.3)])
def test_newpfd_many_exceptions_decode_and_intersect(gpu_ctx, corpus, expected, block, frac):
    """NewPFD blocks with up to 64% exceptions: the group-parallel Simple-16
    exception decode (many rounds of exceptions and of stream words per block)
    in the whole-list decode and in the probe phase's tile decode."""
    ix = _index(corpus, "newpfd", block, frac)
    gpu_ctx.upload(ix)
    assert np.array_equal(gpu_ctx.decode_lists(ix), corpus.docs)
    offs, docs = gpu_ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo="hashseg")
    eoffs, edocs = expected
    assert np.array_equal(offs.astype(np.uint64), eoffs) and np.array_equal(docs, edocs)
    ix.close()
