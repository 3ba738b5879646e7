"""include/excl_scorer.hpp: a batch's AND results walked with CLucene's Scorer
protocol give the documents and scores of CLucene's leapfrog
ConjunctionScorer over the same term scorers (C++ driver
tests/scorer/scorer_check.cpp, compiled with g++; results from the oracle,
which the GPU path matches bit for bit in the parity tests)."""
import os
import subprocess

import numpy as np

import oracle
from exclucene_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_gpu_conjunction_walks_like_conjunction_scorer(tmp_path):
    exe = str(tmp_path / "scorer_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT}/include",
                    os.path.join(HERE, "scorer", "scorer_check.cpp"), "-o", exe], check=True)
    w = synth.zipf_corpus(seed=31, ndocs=1 << 18, nterms=400, cap=40_000, nq=300, qmin=1, qmax=5)
    eoffs, edocs = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
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
