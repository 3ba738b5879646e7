"""The reference's on-disk file sets and query stream: this library writes the
bytes the reference's compressors write for the same lists (fixture made with
the reference's own ParaPFor/NewPFor encoders and fits,
tests/golden/make_golden.py), loads such file sets back into the same index
without re-encoding, and rejects inconsistent ones."""
import os

import numpy as np
import pytest

import exclucene_b200 as ex

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_files.npz")
SETS = {"parapfd": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".segMedian"),
        "newpfd": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".segMedian"),
        "seglrc": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".ind2_distance_base",
                   ".regression_info", ".regression_info_list"),
        "lrc": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".regression_info"),
        "lrcseg": (".ind1", ".ind2", ".segNum", ".segHead", ".segOffset", ".ind2_distance_base",
                   ".regression_info"),
        "hs_seglrc": (".ind1", ".ind2", ".HashSeg_offset", ".HashSeg_info", ".segNum", ".segOffset",
                      ".ind2_distance_base", ".regression_info")}
FRAC = {"parapfd": 0.12, "seglrc": 0.0, "newpfd": 0.12, "lrc": 0.0, "lrcseg": 0.0, "hs_seglrc": 0.0}
CODECS = list(SETS)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def _corpus(g, codec="parapfd"):
    pre = "hs_" if codec == "hs_seglrc" else ""
    lens = g[pre + "lens"].astype(np.uint64)
    return g[pre + "docs"], np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)


def _build(g, codec):
    docs, loff = _corpus(g, codec)
    return ex.Index(docs, loff, codec=codec, block=256, frac=FRAC[codec], hs_bucket=256)


def _write_golden(g, codec, d):
    for suffix in SETS[codec]:
        g[codec + suffix].tofile(os.path.join(d, "g" + suffix))


@pytest.mark.parametrize("codec", CODECS)
def test_writer_matches_reference_bytes(golden, tmp_path, codec):
    ix = _build(golden, codec)
    ix.save_reference(str(tmp_path), "x")
    for suffix in SETS[codec]:
        got = np.fromfile(os.path.join(tmp_path, "x" + suffix), np.uint8)
        assert np.array_equal(got, golden[codec + suffix]), suffix


@pytest.mark.parametrize("codec", CODECS)
def test_loader_rebuilds_the_same_index(golden, tmp_path, codec):
    _write_golden(golden, codec, str(tmp_path))
    got = ex.Index.load_reference(str(tmp_path), "g", codec).export()
    want = _build(golden, codec).export()
    for k in ("words", "seg_head", "seg_rec", "seg_reg", "dir"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    for f in ("word_base", "n", "seg_base", "nseg", "codec", "log2_block", "first_doc", "last_doc", "reg",
              "dir_shift", "dir_base", "ndir", "ntiles"):
        assert np.array_equal(got.lists[f], want.lists[f]), f


def test_query_stream_round_trip(golden):
    terms, toff = ex.query_parse(golden["queries"].tobytes())
    assert toff.tolist() == [0, 2, 5, 7, 10, 12, 13]
    assert terms.tolist() == [6, 7, 5, 6, 7, 0, 7, 7, 4, 3, 2, 2, 1]
    assert ex.query_encode(terms, toff) == golden["queries"].tobytes()
    assert ex.query_parse(b"")[1].tolist() == [0]
    with pytest.raises(ex.ExclError):
        ex.query_parse(np.array([3, 1, 2], np.uint32).tobytes())  # says 3 terms, has 2
    with pytest.raises(ex.ExclError):
        ex.query_parse(np.array([33] + list(range(33)), np.uint32).tobytes())  # more than 32 terms


def test_loader_rejects_inconsistent_sets(golden, tmp_path):
    d = str(tmp_path)
    _write_golden(golden, "parapfd", d)
    # a block offset past the list's words
    off = golden["parapfd.segOffset"].view(np.uint32).copy()
    off[3] = 1 << 20
    off.tofile(os.path.join(d, "g.segOffset"))
    with pytest.raises(ex.ExclError) as e:
        ex.Index.load_reference(d, "g", "parapfd")
    assert e.value.status == ex.api.E_FORMAT
    # .ind2 cut short
    _write_golden(golden, "parapfd", d)
    golden["parapfd.ind2"][:-64].tofile(os.path.join(d, "g.ind2"))
    with pytest.raises(ex.ExclError):
        ex.Index.load_reference(d, "g", "parapfd")
    # segment counts that do not add up
    _write_golden(golden, "parapfd", d)
    sn = golden["parapfd.segNum"].view(np.uint32).copy()
    sn[2] += 1
    sn.tofile(os.path.join(d, "g.segNum"))
    with pytest.raises(ex.ExclError):
        ex.Index.load_reference(d, "g", "parapfd")
    # a missing file, and a format this writer does not produce
    with pytest.raises(ex.ExclError):
        ex.Index.load_reference(d, "nothere", "parapfd")
    docs, loff = _corpus(golden)
    with pytest.raises(ex.ExclError):
        ex.Index(docs, loff, codec="parapfd", block=128).save_reference(d, "y")
    with pytest.raises(ex.ExclError):  # HS by top bits: not the reference's bucketing
        ex.Index(docs, loff, codec="hs_seglrc", hs_kbits=8, hs_ubits=22).save_reference(d, "y")
    with pytest.raises(ex.ExclError):  # HS ParaPFD has no reference file set
        ex.Index(docs, loff, codec="hs_parapfd", hs_bucket=256).save_reference(d, "y")


def test_hs_loader_rejects_inconsistent_buckets(golden, tmp_path):
    d = str(tmp_path)
    # a bucket's base moved so its docIDs leave the bucket
    _write_golden(golden, "hs_seglrc", d)
    base = golden["hs_seglrc.ind2_distance_base"].view(np.uint32).copy()
    base[1] = (int(base[1]) + (1 << 21)) & 0xFFFFFFFF
    base.tofile(os.path.join(d, "g.ind2_distance_base"))
    with pytest.raises(ex.ExclError) as e:
        ex.Index.load_reference(d, "g", "hs_seglrc")
    assert e.value.status == ex.api.E_FORMAT
    # bucket offsets that do not end at the list length
    _write_golden(golden, "hs_seglrc", d)
    info = golden["hs_seglrc.HashSeg_info"].view(np.uint32).copy()
    info[2 + info[1]] -= 1
    info.tofile(os.path.join(d, "g.HashSeg_info"))
    with pytest.raises(ex.ExclError):
        ex.Index.load_reference(d, "g", "hs_seglrc")
    # a bucket count past the end of the record file
    _write_golden(golden, "hs_seglrc", d)
    info = golden["hs_seglrc.HashSeg_info"].view(np.uint32).copy()
    info[1] = 1 << 20
    info.tofile(os.path.join(d, "g.HashSeg_info"))
    with pytest.raises(ex.ExclError):
        ex.Index.load_reference(d, "g", "hs_seglrc")


def test_hs_empty_buckets_are_written_as_the_generator_leaves_them(golden):
    """The clustered list's empty buckets: fit {1, 0, 0, 0}, base = the next docID."""
    info = golden["hs_seglrc.HashSeg_info"].view(np.uint32)
    hoff = golden["hs_seglrc.HashSeg_offset"].view(np.uint32)
    bnum = golden["hs_seglrc.segNum"].view(np.uint32)
    base = golden["hs_seglrc.ind2_distance_base"].view(np.uint32)
    reg = golden["hs_seglrc.regression_info"].view(np.uint32).reshape(-1, 4)
    docs, loff = _corpus(golden, "hs_seglrc")
    h, nb = int(hoff[2]), int(info[hoff[2] + 1])
    off = info[h + 2:h + 3 + nb]
    empty = [b for b in range(nb) if off[b + 1] == off[b]]
    assert empty
    for b in empty:
        assert reg[bnum[2] + b].tolist() == [np.float32(1).view(np.uint32), 0, 0, 0]
        assert base[bnum[2] + b] == docs[loff[2] + off[b]]
