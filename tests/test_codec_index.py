"""Host-side product code against the oracle: the ParaPFD codec calls, the
index builder of every format (blocks, segment metadata, regressions, hash
buckets) and the C ABI surface."""
import os
import re

import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import api, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_codec_matches_oracle_random():
    rng = np.random.default_rng(11)
    for _ in range(500):
        n = int(rng.integers(1, 300))
        bits = int(rng.integers(0, 31))
        v = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32) if bits else np.zeros(n, np.uint32)
        k = int(rng.integers(0, max(1, n // 5)))
        v[rng.integers(0, n, size=k)] = rng.integers(0, 1 << 30, size=k).astype(np.uint32)
        frac = float(rng.choice([0.0, 0.04, 0.1, 0.3, 0.64]))
        w = ex.parapfd_encode(v, frac)
        assert np.array_equal(w, oracle.encode_block(v, frac))
        d, used = ex.parapfd_decode(w, n)
        assert used == len(w) and np.array_equal(d, v)
        assert np.array_equal(ex.encode_array_compat(v, frac), w)


def test_codec_golden_blocks():
    g = np.load(os.path.join(ROOT, "tests", "golden", "parapfd_blocks.npz"))
    vo, wo = 0, g["word_offsets"]
    for i, n in enumerate(g["n"]):
        v = g["values"][vo:vo + n]
        vo += n
        assert np.array_equal(ex.parapfd_encode(v, float(g["frac"][i])), g["words"][wo[i]:wo[i + 1]])


def test_codec_edge_cases():
    # all zeros -> lb = 0, descriptor only
    w = ex.parapfd_encode(np.zeros(128, np.uint32))
    assert list(w) == [0]
    # single value
    w = ex.parapfd_encode(np.array([5], np.uint32))
    assert ex.parapfd_decode(w, 1)[0][0] == 5
    # values needing 31 bits are fine; a block whose best width is 32 is rejected (b = 32 has no descriptor code)
    v = np.array([1 << 30, (1 << 31) - 1], np.uint32)
    assert np.array_equal(ex.parapfd_decode(ex.parapfd_encode(v), 2)[0], v)
    with pytest.raises(ex.ExclError):
        ex.parapfd_encode(np.full(8, 1 << 31, np.uint32))
    # truncated input is a format error
    w = ex.parapfd_encode(np.arange(256, dtype=np.uint32) * 1000)
    with pytest.raises(ex.ExclError):
        ex.parapfd_decode(w[:3], 256)


FORMATS = [("parapfd", 0), ("lrc", 1), ("lrcseg", 2), ("seglrc", 3), ("hs_seglrc", 4), ("hs_parapfd", 5),
           ("newpfd", 6)]


def _compare_index(w, cname, codec, block, frac, kb, ub, bucket=256):
    ix = ex.Index(w.docs, w.list_offsets, codec=cname, block=block, frac=frac, hs_bucket=bucket, hs_kbits=kb,
                  hs_ubits=ub)
    a = ix.export()
    for l in range(w.nlists):
        li = a.lists[l]
        d = w.list(l)
        enc = oracle.encode_list(d, codec, block=block, frac=frac, bucket=bucket, kbits=kb, ubits=ub)
        s0, ns, wb = int(li["seg_base"]), int(li["nseg"]), int(li["word_base"])
        assert ns == len(enc["starts"]), (cname, l)
        assert np.array_equal(a.words[wb:wb + len(enc["words"])], enc["words"]), (cname, l)
        assert np.array_equal(a.seg_head[s0:s0 + ns], enc["head"])
        assert np.array_equal(a.seg_rec[s0:s0 + ns, 0], enc["starts"])
        assert np.array_equal(a.seg_rec[s0:s0 + ns, 1], enc["off"])
        assert np.array_equal(a.seg_rec[s0:s0 + ns, 2], enc["aux"])
        assert np.array_equal(a.seg_rec[s0:s0 + ns, 3], enc["counts"])
        if codec in (3, 4):
            assert np.array_equal(a.seg_reg[s0:s0 + ns], enc["reg"])
        if codec == 1:
            assert np.array_equal(np.array(li["reg"], np.uint32)[:3], enc["listreg"][:3])
        if codec in (2, 3, 4):
            assert np.array_equal(np.array(li["reg"], np.uint32), enc["listreg"])
        if codec in (4, 5):
            assert int(li["dir_shift"]) == enc["shift"]
            d0 = int(li["dir_base"])
            assert np.array_equal(a.dir[d0:d0 + int(li["ndir"]) + 1], enc["first"])
        assert np.array_equal(oracle.decode_list(enc, codec, len(d)), d)
    ix.close()


@pytest.mark.parametrize("cname,codec", FORMATS)
@pytest.mark.parametrize("block", [128, 256])
@pytest.mark.parametrize("frac", [0.0, 0.1])
def test_index_build_matches_oracle(cname, codec, block, frac):
    lens = [1, 2, 3, 31, 127, 128, 129, 255, 256, 257, 1000, 5000, 40000]
    w = synth.clustered_lists(lens, ubits=22, seed=5)
    kb = 8 if codec == 5 else 0
    _compare_index(w, cname, codec, block, frac, kb, 22)


@pytest.mark.parametrize("cname,codec", FORMATS)
def test_index_build_uniform_wide_universe(cname, codec):
    w = synth.uniform_lists([1, 300, 4096, 70000], ubits=31, seed=9)
    _compare_index(w, cname, codec, 256, 0.0, 12 if codec == 5 else 0, 31)


def test_index_rejects_unrepresentable_gap():
    """A d-gap >= 2^31 needs b = 32, which the descriptor's 5-bit lb field cannot
    hold (ParaPFor.cpp:88 stores lb << 26 and :103 reads it back modulo 32)."""
    with pytest.raises(ex.ExclError) as e:
        ex.Index(np.array([0, 2 ** 32 - 8], np.uint32), np.array([0, 2], np.uint64), codec="parapfd")
    assert e.value.status == api.E_FORMAT


def test_index_rejects_bad_input():
    docs = np.array([5, 3, 9], np.uint32)
    with pytest.raises(ex.ExclError):
        ex.Index(docs, np.array([0, 3], np.uint64))
    with pytest.raises(ex.ExclError):
        ex.Index(np.array([1, 2], np.uint32), np.array([0, 0, 2], np.uint64))  # empty list
    with pytest.raises(ex.ExclError):
        ex.Index(np.array([1, 2], np.uint32), np.array([0, 2], np.uint64), block=100)


def test_abi_exports_every_declared_symbol():
    """The library loads and exports each function include/excl_gpu.h declares."""
    hdr = open(os.path.join(ROOT, "include", "excl_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    declared = set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", hdr)) - {"if", "sizeof"}
    declared = {d for d in declared if d.startswith("excl_") or d in ("encodeArray", "decodeArray")}
    import ctypes

    lib = ctypes.CDLL(api.library_path())
    missing = [d for d in sorted(declared) if not hasattr(lib, d)]
    assert not missing, missing
    assert set(api.EXPORTED) <= declared | {"encodeArray", "decodeArray"}


def test_checksum_matches_oracle():
    offs = np.array([0, 3, 3, 4, 9], np.uint32)
    docs = np.array([1, 5, 9, 2, 3, 4, 8, 16, 32], np.uint32)
    assert ex.checksum(offs, docs) == oracle.checksum(offs.astype(np.uint64), docs)


def test_newpfd_codec_matches_reference_golden_blocks():
    """Host NewPFD blocks equal the reference NewPFor.cpp's (golden vectors), and decode back."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "newpfd_blocks.npz"))
    vo, wo = 0, g["word_offsets"]
    for i, n in enumerate(g["n"]):
        v = g["values"][vo:vo + n]
        vo += n
        ref = g["words"][wo[i]:wo[i + 1]]
        assert np.array_equal(ex.newpfd_encode(v, float(g["frac"][i])), ref), f"block {i}"
        dec, used = ex.newpfd_decode(ref, int(n))
        assert used == len(ref) and np.array_equal(dec, v)


def test_newpfd_rejects_high_part_beyond_28_bits():
    # with b = 0 every nonzero value is an exception; a high part needs <= 28 bits
    with pytest.raises(ex.ExclError):
        ex.newpfd_encode(np.array([1 << 29] + [0] * 20, np.uint32), 0.1)
    with pytest.raises(ex.ExclError):
        ex.newpfd_decode(np.array([(0 << 26) | 3], np.uint32), 4)  # 3 exceptions, no Simple-16 words
