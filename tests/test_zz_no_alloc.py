"""The allocation-free entry point, excl_intersect_device_noalloc.

It serves callers that cannot call cudaMalloc when they query (a host that
fixes its device memory at start-up, or an embedding without an excl_ctx,
whose creation allocates). This file is collected last so that a run stopping
at the first failure has already run every other test; it also passes alone.
The entry point's results must equal excl_intersect_device's on the same
batch, bit for bit (integer docIDs), on two calls in a row — the second call
finds the first call's data in the shared scratch array — and both must equal
the CPU oracle's exact AND of the batch.
"""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    # 2,000 queries of 1-6 terms whose shortest lists sum to ~636k docIDs,
    # inside the entry point's limits (4,096 queries, 2^20 keys)
    w = synth.zipf_corpus(seed=4242, ndocs=1 << 20, nterms=3000, cap=60_000, nq=2000, qmin=1, qmax=6)
    lens = np.diff(w.list_offsets).astype(np.int64)
    keys = sum(int(min(lens[w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]])) for q in range(w.nq))
    assert w.nq <= api.NOALLOC_MAX_QUERIES and keys <= api.NOALLOC_MAX_KEYS
    ctx = ex.Context(0, max_queries=4096, max_keys=1 << 22)
    yield torch, w, ctx
    ctx.close()


def _run_both(torch, w, ctx, ix, algo):
    dev = torch.device("cuda", 0)
    lens = np.diff(w.list_offsets).astype(np.int64)
    cap = max(1, sum(int(min(lens[w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]], default=0))
                     for q in range(w.nq)))
    d_terms = torch.from_numpy(w.terms.astype(np.int32)).to(dev)
    d_toff = torch.from_numpy(w.term_offsets.astype(np.int32)).to(dev)
    ref_offs = torch.zeros(w.nq + 1, dtype=torch.int32, device=dev)
    ref_docs = torch.zeros(cap, dtype=torch.int32, device=dev)
    ctx.intersect_device(ix, d_terms.data_ptr(), d_toff.data_ptr(), w.nq, algo, ref_offs.data_ptr(),
                         ref_docs.data_ptr(), cap)
    ctx.check()
    ro = ref_offs.cpu().numpy()
    rd = ref_docs.cpu().numpy()[: int(ro[-1])]
    # the allocating path against the CPU oracle's exact AND on the same batch
    eo, ed = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    assert np.array_equal(ro.astype(np.uint64), eo) and np.array_equal(rd.view(np.uint32), ed)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        offs = torch.full((w.nq + 1,), -1, dtype=torch.int32, device=dev)
        docs = torch.full((cap,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        api.intersect_device_noalloc(ix, d_terms.data_ptr(), d_toff.data_ptr(), w.nq, algo, offs.data_ptr(),
                                     docs.data_ptr(), cap, stream.cuda_stream)
        o = offs.cpu().numpy()
        assert np.array_equal(o, ro), f"offsets differ on call {call}"
        assert np.array_equal(docs.cpu().numpy()[: int(o[-1])], rd), f"docIDs differ on call {call}"
        # and the no-alloc result itself against the oracle
        assert np.array_equal(o.astype(np.uint64), eo), f"offsets differ from the oracle on call {call}"
        assert np.array_equal(docs.cpu().numpy()[: int(o[-1])].view(np.uint32), ed), \
            f"docIDs differ from the oracle on call {call}"


@pytest.mark.parametrize("codec,algo", [("seglrc", "auto"), ("parapfd", "bsearch"), ("hs_parapfd", "hashseg")])
def test_noalloc_matches_allocating_entry_point(setup, codec, algo):
    torch, w, ctx = setup
    ix = ex.Index(w.docs, w.list_offsets, codec=codec, block=128 if codec != "seglrc" else 256, hs_kbits=10,
                  hs_ubits=20)
    ctx.upload(ix)
    _run_both(torch, w, ctx, ix, algo)
    ix.close()


def test_noalloc_rejects_oversized_batches(setup):
    torch, w, ctx = setup
    dev = torch.device("cuda", 0)
    # one list of 600,000 postings; two single-term queries on it need 1.2M keys > 2^20
    docs = np.arange(0, 1_200_000, 2, dtype=np.uint32)
    ix = ex.Index(docs, np.array([0, len(docs)], np.uint64), codec="parapfd")
    ctx.upload(ix)
    terms = torch.zeros(2, dtype=torch.int32, device=dev)
    toff = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    offs = torch.zeros(3, dtype=torch.int32, device=dev)
    out = torch.zeros(1_200_000, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    with pytest.raises(ex.ExclError) as e:
        api.intersect_device_noalloc(ix, terms.data_ptr(), toff.data_ptr(), 2, "auto", offs.data_ptr(),
                                     out.data_ptr(), len(out), s)
    assert e.value.status == api.E_CAPACITY
    # too many queries is refused before any work
    big = torch.zeros(api.NOALLOC_MAX_QUERIES + 2, dtype=torch.int32, device=dev)
    with pytest.raises(ex.ExclError) as e:
        api.intersect_device_noalloc(ix, terms.data_ptr(), big.data_ptr(), api.NOALLOC_MAX_QUERIES + 1, "auto",
                                     offs.data_ptr(), out.data_ptr(), len(out), s)
    assert e.value.status == api.E_CAPACITY
    # a batch within the limits still works afterwards
    offs1 = torch.zeros(2, dtype=torch.int32, device=dev)
    api.intersect_device_noalloc(ix, terms.data_ptr(), toff.data_ptr(), 1, "auto", offs1.data_ptr(),
                                 out.data_ptr(), len(out), s)
    assert int(offs1[1]) == len(docs)
    assert np.array_equal(out[: len(docs)].cpu().numpy().astype(np.uint32), docs)
    ix.close()
