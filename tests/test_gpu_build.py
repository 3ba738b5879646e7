"""Index build on the GPU: for the ParaPFD, NewPFD, LRC, LRCSeg, SegLRC,
HS_SegLRC and HS_ParaPFD formats the device build gives the host build's arrays bit for bit
(hash partition, fits, residual bases, medians, blocks, directories, tile
maps), rejects unordered lists, and the index it builds answers queries as the
oracle does."""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth

pytestmark = pytest.mark.gpu

FIELDS = ("word_base", "n", "seg_base", "nseg", "codec", "log2_block", "first_doc", "last_doc", "reg", "dir_shift",
          "dir_base", "ndir", "tile_base", "ntiles", "model")


def _same_index(a: ex.Index, b: ex.Index):
    ea, eb = a.export(), b.export()
    for k in ("words", "seg_head", "seg_rec", "seg_reg", "dir"):
        assert np.array_equal(getattr(ea, k), getattr(eb, k)), k
    for f in FIELDS:
        assert np.array_equal(ea.lists[f], eb.lists[f]), f


def _edge_lists():
    rng = np.random.default_rng(3)
    lists = [np.array([7], np.uint32), np.arange(1000, 1300, dtype=np.uint32),          # gaps of 1
             np.array([0, 1, 2 ** 31, 2 ** 32 - 2], np.uint32),                          # huge gaps
             np.sort(rng.choice(2 ** 32 - 1, 5000, replace=False)).astype(np.uint32),   # wide residuals
             np.arange(0, 256 * 3, 3, dtype=np.uint32), np.arange(5, 5 + 257, dtype=np.uint32)]
    docs = np.concatenate(lists)
    return docs, np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.uint64)


@pytest.fixture(scope="module")
def corpus():
    return synth.zipf_corpus(seed=21, ndocs=1 << 20, nterms=2500, cap=150_000, nq=800, qmin=2, qmax=5)


HS_BUCKET = dict(hs_bucket=256)          # the reference's bucketing: shift from the length
HS_TOP = dict(hs_kbits=12, hs_ubits=32)   # top 12 bits of the docID
CASES = [("parapfd", 256, 0.0, {}), ("parapfd", 128, 0.12, {}), ("parapfd", 256, 0.64, {}),
         ("seglrc", 256, 0.0, {}), ("seglrc", 128, 0.1, {}), ("lrc", 256, 0.0, {}), ("lrc", 128, 0.1, {}),
         ("lrcseg", 256, 0.0, {}), ("lrcseg", 128, 0.1, {}),
         ("hs_seglrc", 256, 0.0, HS_BUCKET), ("hs_seglrc", 256, 0.1, HS_BUCKET), ("hs_seglrc", 256, 0.0, HS_TOP),
         ("hs_parapfd", 128, 0.1, HS_BUCKET), ("hs_parapfd", 256, 0.0, HS_TOP),
         ("newpfd", 128, 0.1, {}), ("newpfd", 256, 0.64, {}), ("newpfd", 32, 0.3, {})]


@pytest.mark.parametrize("codec,block,frac,hs", CASES)
def test_device_build_equals_host_build(gpu_ctx, corpus, codec, block, frac, hs):
    import torch

    for docs, loff in ((corpus.docs, corpus.list_offsets), _edge_lists()):
        d = torch.from_numpy(docs.view(np.int32)).cuda()
        torch.cuda.synchronize()
        try:
            got = gpu_ctx.build_index(d.data_ptr(), loff, codec=codec, block=block, frac=frac, **hs)
        except ex.ExclError as e:
            # where the host build rejects the data (unrepresentable block), so must the device
            with pytest.raises(ex.ExclError):
                ex.Index(docs, loff, codec=codec, block=block, frac=frac, **hs)
            assert e.status == ex.api.E_FORMAT
            continue
        want = ex.Index(docs, loff, codec=codec, block=block, frac=frac, **hs)
        _same_index(got, want)
        got.close()
        want.close()


@pytest.mark.parametrize("codec,hs", [("lrc", {}), ("lrcseg", {}), ("hs_seglrc", HS_BUCKET),
                                      ("newpfd", dict(block=128, frac=0.3))])
def test_device_built_index_answers_queries(gpu_ctx, corpus, codec, hs):
    import torch

    d = torch.from_numpy(corpus.docs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ix = gpu_ctx.build_index(d.data_ptr(), corpus.list_offsets, codec=codec, **hs)
    gpu_ctx.upload(ix)
    assert np.array_equal(gpu_ctx.decode_lists(ix), corpus.docs)
    offs, got = gpu_ctx.intersect(ix, corpus.terms, corpus.term_offsets, algo="hashseg")
    eo, ed = oracle.answer(corpus.docs, corpus.list_offsets, corpus.terms, corpus.term_offsets)
    assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(got, ed)
    ix.close()


def test_device_build_of_a_list_range_and_queries(gpu_ctx, corpus):
    import torch

    # lists 100.. of the corpus, indexed through absolute offsets into the full array
    loff = corpus.list_offsets[100:]
    d = torch.from_numpy(corpus.docs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ix = gpu_ctx.build_index(d.data_ptr(), loff, codec="seglrc")
    sub_docs = corpus.docs[int(loff[0]):int(loff[-1])]
    sub_off = (loff - loff[0]).astype(np.uint64)
    _same_index(ix, ex.Index(sub_docs, sub_off, codec="seglrc"))
    gpu_ctx.upload(ix)
    rng = np.random.default_rng(8)
    nl = len(sub_off) - 1
    qs = [rng.choice(nl, size=int(rng.integers(2, 5)), replace=False) for _ in range(300)]
    terms = np.concatenate(qs).astype(np.uint32)
    toff = np.concatenate([[0], np.cumsum([len(q) for q in qs])]).astype(np.uint32)
    offs, got = gpu_ctx.intersect(ix, terms, toff, algo="hashseg")
    eo, ed = oracle.answer(sub_docs, sub_off, terms, toff)
    assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(got, ed)
    ix.close()


def test_device_build_rejects_unordered_lists(gpu_ctx):
    import torch

    docs = np.array([5, 9, 9, 12, 1, 2, 3], np.uint32)  # list 0 repeats 9
    d = torch.from_numpy(docs.view(np.int32)).cuda()
    torch.cuda.synchronize()
    for codec in ("parapfd", "seglrc", "lrc", "lrcseg", "hs_seglrc", "hs_parapfd", "newpfd"):
        with pytest.raises(ex.ExclError) as e:
            gpu_ctx.build_index(d.data_ptr(), np.array([0, 4, 7], np.uint64), codec=codec)
        assert e.value.status == ex.api.E_INVALID


def test_layout_autotuner_keeps_the_fastest_exact_layout(gpu_ctx):
    """excl_autotune_layout builds each candidate layout on the GPU, tunes and
    times the sample on it, and hands back the fastest one, uploaded; that
    index answers as the oracle does, and so would every other candidate."""
    import torch

    w = synth.skewed(seed=77, nq=300, npool=6, long_min=200_000, long_max=800_000)
    d_docs = torch.from_numpy(w.docs.view(np.int32)).to("cuda:0")
    torch.cuda.synchronize()
    cands = [dict(codec="hs_parapfd", block=128, frac=0.1, hs_kbits=k, hs_ubits=26) for k in (8, 12, 16)]
    cands += [dict(codec="seglrc", block=256), dict(codec="parapfd", block=128, frac=0.1)]
    ix, best, rep = gpu_ctx.autotune_layout(d_docs.data_ptr(), w.list_offsets, cands, w.terms, w.term_offsets)
    assert all(r["status"] == 0 and r["best_ms"] > 0 for r in rep), rep
    assert rep[best]["best_ms"] == min(r["best_ms"] for r in rep)
    eo, ed = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    offs, docs = gpu_ctx.intersect(ix, w.terms, w.term_offsets, algo="auto")
    assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(docs, ed)
    # the same layout built on the host is the same index
    host = ex.Index(w.docs, w.list_offsets, **{k: v for k, v in cands[best].items()})
    _same_index(ix, host)
    ix.close()
    host.close()
    # a layout that cannot be built (blocks of 512 are beyond the tile size) is
    # recorded as skipped, the others still run
    ix, best, rep = gpu_ctx.autotune_layout(d_docs.data_ptr(), w.list_offsets,
                                            [dict(codec="parapfd", block=512), dict(codec="newpfd", block=128,
                                                                                    frac=0.1)],
                                            w.terms, w.term_offsets)
    assert rep[0]["status"] != 0 and rep[1]["status"] == 0 and best == 1
    ix.close()
