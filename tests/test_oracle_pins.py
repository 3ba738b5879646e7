"""Pins the CPU oracle to the reference: golden vectors made by the reference's
own ParaPFor.cpp / getRegressionInfo (tests/golden/make_golden.py), and, when
the reference tree is present, the compiled reference itself."""
import os

import numpy as np
import pytest

import oracle
from conftest import have_reference

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_oracle_codec_matches_reference_golden_blocks():
    g = np.load(os.path.join(GOLD, "parapfd_blocks.npz"))
    vo, wo = 0, g["word_offsets"]
    for i, n in enumerate(g["n"]):
        v = g["values"][vo:vo + n]
        vo += n
        ref_words = g["words"][wo[i]:wo[i + 1]]
        got = oracle.encode_block(v, float(g["frac"][i]))
        assert np.array_equal(got, ref_words), f"block {i}"
        dec, used = oracle.decode_block(ref_words, int(n))
        assert used == len(ref_words) and np.array_equal(dec, v)


def test_oracle_newpfd_matches_reference_golden_blocks():
    g = np.load(os.path.join(GOLD, "newpfd_blocks.npz"))
    vo, wo = 0, g["word_offsets"]
    for i, n in enumerate(g["n"]):
        v = g["values"][vo:vo + n]
        vo += n
        ref_words = g["words"][wo[i]:wo[i + 1]]
        assert np.array_equal(oracle.newpfd_encode_block(v, float(g["frac"][i])), ref_words), f"block {i}"
        dec, used = oracle.newpfd_decode_block(ref_words, int(n))
        assert used == len(ref_words) and np.array_equal(dec, v)


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_oracle_newpfd_vs_compiled_reference_random_blocks():
    rng = np.random.default_rng(11)
    for _ in range(300):
        n = int(rng.integers(1, 300))
        bits = int(rng.integers(0, 29))
        v = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32) if bits else np.zeros(n, np.uint32)
        frac = float(rng.choice([0.0, 0.1, 0.12, 0.5]))
        assert np.array_equal(oracle.newpfd_encode_block(v, frac), oracle.ref_newpfd_encode(v, frac))


def test_oracle_fits_match_reference_golden():
    g = np.load(os.path.join(GOLD, "regression_fits.npz"))
    o = 0
    for i, n in enumerate(g["n"]):
        y = g["y"][o:o + n]
        o += n
        assert np.array_equal(oracle.fit_seg_raw(y), g["seglrc"][i]), f"seglrc fit {i}"
        assert np.array_equal(oracle.fit_lrc_raw(y), g["lrc"][i]), f"lrc fit {i}"


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_oracle_vs_compiled_reference_random_blocks():
    rng = np.random.default_rng(7)
    for _ in range(300):
        n = int(rng.integers(1, 400))
        bits = int(rng.integers(0, 31))
        v = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32) if bits else np.zeros(n, np.uint32)
        frac = float(rng.choice([0.0, 0.1, 0.12, 0.5]))
        assert np.array_equal(oracle.encode_block(v, frac), oracle.ref_encode(v, frac))


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_inverted_list_fixture_digest():
    """The reference's shipped list encodes to the digests recorded from the reference codec."""
    import hashlib

    path = os.path.join(oracle.REFERENCE, "src/gpu/Preprocess/ExtractList/data/InvertedList")
    docs = np.fromfile(path, dtype=np.uint32)
    lines = [ln.split() for ln in open(os.path.join(GOLD, "inverted_list_digest.txt")) if ln.startswith("frac")]
    for _, frac, _, nw, _, h in lines:
        enc = oracle.encode_list(docs, 0, block=256, frac=float(frac))
        assert len(enc["words"]) == int(nw)
        assert hashlib.sha256(enc["words"].tobytes()).hexdigest() == h
        assert np.array_equal(oracle.decode_list(enc, 0, len(docs)), docs)


def test_oracle_intersection_and_checksum():
    a = np.array([1, 3, 5, 7, 9, 11], np.uint32)
    b = np.array([3, 4, 5, 9, 12], np.uint32)
    c = np.array([0, 5, 9, 100], np.uint32)
    assert list(oracle.intersect([a, b, c])) == [5, 9]
    assert list(oracle.intersect([a])) == list(a)
    assert len(oracle.intersect([a, np.array([2, 4], np.uint32)])) == 0
    offs = np.array([0, 2, 2, 5], np.uint64)
    res = np.array([5, 9, 1, 2, 3], np.uint32)
    e, tot, x = oracle.checksum(offs, res)
    assert (e, tot) == (1, 5)
    assert x == (5 ^ 9 ^ 9) ^ (1 ^ 3 ^ 2)


def test_oracle_regression_arithmetic_known_answers():
    """Hand-checked fits: two points give the exact line; one point the reference's special case."""
    a, b, L, R = oracle.fit_seg(np.array([10, 20], np.uint32))
    assert (a, b) == (10.0, 10.0) and (L, R) == (1, 1)
    a, b, L, R = oracle.fit_seg(np.array([123456], np.uint32))
    assert (a, b, L, R) == (1.0, 123456.0, 0, 0)
    raw = oracle.fit_lrc_raw(np.array([7], np.uint32))
    assert raw[1] == 7 and np.uint32(raw[0]).view(np.float32) == 1.0
