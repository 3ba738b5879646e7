"""The oracle's restatement of the benchmark workloads and encoders (CPU only).

bench.py's CPU reference arm builds its inputs with the oracle alone, so that
arm loads no library of the package. These tests pin that restatement to the
package: the seeded generators give the same lists and queries bit for bit,
the oracle's whole-corpus encoder writes the same compressed image as the
package's index build, and the threaded batch answer equals the per-query
exact AND.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GEN_CASES = [
    ("pairs", dict(npairs=6, long_len=1 << 16)),
    ("zipf_corpus", dict(ndocs=1 << 20, nterms=3000, cap=60_000, nq=500)),
    ("skewed", dict(nq=40, npool=4, long_min=100_000, long_max=300_000)),
    ("learned", dict(lmin=100_000, lmax=600_000, nq=30, nclust=3, nzipf=3)),
    ("serving", dict(total=2_000_000, nterms=5000, nq=300)),
]


@pytest.mark.parametrize("name,kw", GEN_CASES, ids=[c[0] for c in GEN_CASES])
def test_oracle_generators_match_the_package(name, kw):
    a = getattr(synth, name)(**kw)
    b = getattr(oracle, "wl_" + name)(**kw)
    for k in ("docs", "list_offsets", "terms", "term_offsets", "info"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert (a.codecs is None and b.codecs is None) or np.array_equal(a.codecs, b.codecs)


def test_query_stream_prefix_is_the_single_batch():
    """--gpus N draws N batches from one stream; rank 0's batch is the N=1 batch."""
    one = oracle.wl_zipf_corpus(ndocs=1 << 18, nterms=800, cap=20_000, nq=100)
    two = oracle.wl_zipf_corpus(ndocs=1 << 18, nterms=800, cap=20_000, nq=200)
    assert np.array_equal(one.docs, two.docs)
    n = int(one.term_offsets[-1])
    assert np.array_equal(one.term_offsets, two.term_offsets[:101]) and np.array_equal(one.terms, two.terms[:n])


ENC_CASES = [("parapfd", 128, 0.1, {}), ("seglrc", 256, 0.0, {}), ("lrc", 256, 0.0, {}), ("lrcseg", 256, 0.1, {}),
             ("newpfd", 128, 0.1, {}), ("hs_seglrc", 256, 0.0, {}),
             ("hs_parapfd", 128, 0.1, dict(hs_kbits=10, hs_ubits=20))]


@pytest.mark.parametrize("cname,block,frac,hs", ENC_CASES, ids=[c[0] for c in ENC_CASES])
def test_oracle_corpus_encoder_matches_the_index_build(cname, block, frac, hs):
    w = synth.zipf_corpus(seed=77, ndocs=1 << 20, nterms=400, cap=50_000, nq=200, qmin=2, qmax=4)
    codec = {"newpfd": 6, **oracle.CODECS}[cname]
    img = oracle.encode_corpus(w.docs, w.list_offsets, codec, block=block, frac=frac,
                               kbits=hs.get("hs_kbits", 0), ubits=hs.get("hs_ubits", 32))
    arr = ex.Index(w.docs, w.list_offsets, codec=cname, block=block, frac=frac, **hs).export()
    assert np.array_equal(img.words[: len(arr.words) - 8], arr.words[:-8])
    assert np.array_equal(img.head, arr.seg_head)
    assert np.array_equal(img.rec.reshape(-1, 4), arr.seg_rec)
    if codec in (3, 4):
        assert np.array_equal(img.sreg.reshape(-1, 4), np.asarray(arr.seg_reg).view(np.uint32).reshape(-1, 4))
    # the CPU path on the oracle's image answers as the exact AND
    _, counts = oracle.run_queries_compressed(img, w.terms, w.term_offsets, 2)
    eo, _ = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    assert np.array_equal(counts, np.diff(eo))


def test_answer_batch_equals_answer():
    w = synth.zipf_corpus(seed=78, ndocs=1 << 19, nterms=600, cap=40_000, nq=700, qmin=1, qmax=6)
    o1, d1 = oracle.answer(w.docs, w.list_offsets, w.terms, w.term_offsets)
    o2, d2 = oracle.answer_batch(w.docs, w.list_offsets, w.terms, w.term_offsets, threads=3)
    assert np.array_equal(o1, o2) and np.array_equal(d1, d2)


def test_reference_arm_loads_no_package_library():
    code = (
        "import io, contextlib, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--cpu-sample-s', '0.2',"
        " '--scale', '0.01']\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "bad = [l for l in maps.splitlines() if 'exclucene_b200' in l]\n"
        "assert not bad, bad\n"
        "import json\n"
        "line = json.loads(buf.getvalue().strip().splitlines()[-1])\n"
        "assert line['impl'] == 'reference' and line['cpu_baseline']['kind'] == 'port'\n"
        "print('ok', line['config']['queries_per_step'])\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok")
