"""Device failure path without a GPU fault.

Every cross-CTA wait of the batch kernel is bounded: when it gives up it sets
an error bit and the kernel finishes. excl_ctx_set_wait_check makes each batch
run one more bounded wait on a flag that nothing sets, so that wait always
gives up; the test checks that the host sees EXCL_E_DEVICE_FLAG on every path
that reports a batch (excl_ctx_check after excl_intersect_device, excl_wait
after excl_submit and excl_submit_into, a CUDA-graph replay), that the batch
itself still completes exactly, and that the context answers the next batch as
the oracle does once the check is off. Nothing traps, faults or hangs.
"""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def work():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = synth.zipf_corpus(seed=4711, ndocs=1 << 19, nterms=800, cap=30_000, nq=600, qmin=2, qmax=5)
    eo, ed = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    return torch, w, eo, ed


def _expect_flag(fn):
    with pytest.raises(ex.ExclError) as e:
        fn()
    assert e.value.status == api.E_DEVICE_FLAG
    assert "scan wait expired" in str(e.value)


@pytest.mark.parametrize("graphs", [False, True])
def test_expired_wait_is_reported_and_the_context_recovers(work, graphs):
    torch, w, eo, ed = work
    dev = torch.device("cuda", 0)
    ctx = ex.Context(0, max_queries=4096, max_keys=1 << 22, use_graphs=graphs)
    ix = ex.Index(w.docs, w.list_offsets, codec="seglrc")
    ctx.upload(ix)
    cap = 1 << 22
    d_terms = torch.from_numpy(w.terms.astype(np.int32)).to(dev)
    d_toff = torch.from_numpy(w.term_offsets.astype(np.int32)).to(dev)
    d_offs = torch.zeros(w.nq + 1, dtype=torch.int32, device=dev)
    d_docs = torch.zeros(cap, dtype=torch.int32, device=dev)

    def device_batch():
        ctx.intersect_device(ix, d_terms.data_ptr(), d_toff.data_ptr(), w.nq, "auto", d_offs.data_ptr(),
                             d_docs.data_ptr(), cap)
        ctx.check()

    def device_exact():
        o = d_offs.cpu().numpy().astype(np.uint64)
        return np.array_equal(o, eo) and np.array_equal(d_docs[: int(o[-1])].cpu().numpy().view(np.uint32), ed)

    device_batch()  # a clean batch first (and, with graphs, the uncaptured first sighting)
    assert device_exact()
    ctx.set_wait_check(32)
    for _ in range(3):  # stream launch, then capture and replays when graphs are on
        _expect_flag(device_batch)
        assert device_exact()  # the batch itself completed exactly
    # excl_submit + excl_wait and excl_submit_into + excl_wait report it per batch
    b = ctx.submit(ix, w.terms, w.term_offsets, "auto")
    _expect_flag(b.wait)
    b.free()
    p_off, p_docs = ex.pinned_empty(w.nq + 1), ex.pinned_empty(cap)
    b = ctx.submit_into(ix, w.terms, w.term_offsets, p_off, p_docs, "auto")
    _expect_flag(b.wait)
    b.free()
    # off again: the same context answers exactly and reports nothing
    ctx.set_wait_check(0)
    device_batch()
    assert device_exact()
    offs, docs = ctx.intersect(ix, w.terms, w.term_offsets, algo="auto")
    assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(docs, ed)
    ix.close()
    ctx.close()
