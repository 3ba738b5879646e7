"""include/excl_scorer.hpp: a batch's AND results walked with CLucene's Scorer
protocol give the documents and scores of CLucene's leapfrog
ConjunctionScorer over the same term scorers (C++ driver
tests/scorer/scorer_check.cpp, compiled with g++). The CPU test feeds the
oracle's results; the GPU test feeds the results of a real device batch
(excl_submit + excl_wait), as a CLucene host would."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from exclucene_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _driver(tmp_path) -> str:
    exe = str(tmp_path / "scorer_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT}/include",
                    os.path.join(HERE, "scorer", "scorer_check.cpp"), "-o", exe], check=True)
    return exe


def _walk(tmp_path, exe, w, eoffs, edocs):
    parts = [np.array([w.nlists], np.uint32)]
    for l in range(w.nlists):
        d = w.docs[w.list_offsets[l]:w.list_offsets[l + 1]]
        parts += [np.array([len(d)], np.uint32), d.astype(np.uint32)]
    parts.append(np.array([w.nq], np.uint32))
    for q in range(w.nq):
        t = w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]
        parts += [np.array([len(t)], np.uint32), t.astype(np.uint32)]
    parts += [eoffs.astype(np.uint32), edocs.astype(np.uint32)]
    inp = tmp_path / "batch.bin"
    np.concatenate(parts).tofile(inp)
    r = subprocess.run([exe, str(inp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK") and int(r.stdout.split()[1]) > 100


def test_gpu_conjunction_walks_like_conjunction_scorer(tmp_path):
    exe = _driver(tmp_path)
    w = synth.zipf_corpus(seed=31, ndocs=1 << 18, nterms=400, cap=40_000, nq=300, qmin=1, qmax=5)
    eoffs, edocs = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    _walk(tmp_path, exe, w, eoffs, edocs)


@pytest.mark.gpu
@pytest.mark.parametrize("codec", ["seglrc", "parapfd"])
def test_scorer_over_a_device_batch(tmp_path, gpu_ctx, codec):
    """The results of one device batch, taken through excl_submit and
    excl_wait, drive GpuConjunction; every query visits the leapfrog's
    documents with its scores."""
    import exclucene_b200 as ex

    exe = _driver(tmp_path)
    w = synth.zipf_corpus(seed=32, ndocs=1 << 18, nterms=400, cap=40_000, nq=300, qmin=1, qmax=5)
    ix = ex.Index(w.docs, w.list_offsets, codec=codec, block=256 if codec == "seglrc" else 128)
    gpu_ctx.upload(ix)
    b = gpu_ctx.submit(ix, w.terms, w.term_offsets, "auto")
    offs, docs = b.wait()
    b.free()
    eoffs, edocs = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    assert np.array_equal(offs.astype(np.uint64), eoffs) and np.array_equal(docs, edocs)
    _walk(tmp_path, exe, w, offs.astype(np.uint64), docs)
    ix.close()
