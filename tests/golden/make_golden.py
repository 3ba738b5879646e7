"""Writes tests/golden/*.npz from the reference's own code compiled from its
sources (oracle/_ref: ParaPFor.cpp and the generators' getRegressionInfo).

Run in a tree that has the reference sources (at EXCL_REFERENCE, default
/root/reference):
    make -C oracle all ref && python tests/golden/make_golden.py
The fixtures hold seeded synthetic inputs and the reference's outputs, so the
checks that use them run anywhere (no reference tree needed).
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
FRACS = [0.0, 0.04, 0.08, np.float32(np.float32(0.04) + np.float32(0.04)) + np.float32(0.04), 0.1, 0.2, 0.64]
INVERTED_LIST = os.path.join(oracle.REFERENCE, "src/gpu/Preprocess/ExtractList/data/InvertedList")


def codec_vectors():
    rng = np.random.default_rng(0xC0DEC)
    ins, ns, fr, outs, offs = [], [], [], [], [0]
    for t in range(400):
        n = int(rng.integers(1, 300))
        bits = int(rng.integers(0, 31))
        v = (rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32) if bits
             else np.zeros(n, np.uint32))
        k = int(rng.integers(0, max(1, n // 4)))
        v[rng.integers(0, n, size=k)] = rng.integers(0, 1 << 30, size=k).astype(np.uint32)
        f = float(FRACS[t % len(FRACS)])
        w = oracle.ref_encode(v, f)
        ins.append(v)
        ns.append(n)
        fr.append(f)
        outs.append(w)
        offs.append(offs[-1] + len(w))
    np.savez_compressed(os.path.join(OUT, "parapfd_blocks.npz"), values=np.concatenate(ins),
                        n=np.array(ns, np.uint32), frac=np.array(fr, np.float32), words=np.concatenate(outs),
                        word_offsets=np.array(offs, np.uint64))


def newpfd_vectors():
    """NewPFD blocks from the reference's own NewPFor.cpp (Simple-16 exceptions)."""
    rng = np.random.default_rng(0x5E16)
    ins, ns, fr, outs, offs = [], [], [], [], [0]
    for t in range(300):
        n = int(rng.integers(1, 300))
        bits = int(rng.integers(0, 29))
        v = (rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32) if bits
             else np.zeros(n, np.uint32))
        k = int(rng.integers(0, max(1, n // 3)))
        v[rng.integers(0, n, size=k)] = rng.integers(0, 1 << 28, size=k).astype(np.uint32)
        f = float(FRACS[t % len(FRACS)])
        w = oracle.ref_newpfd_encode(v, f)
        ins.append(v)
        ns.append(n)
        fr.append(f)
        outs.append(w)
        offs.append(offs[-1] + len(w))
    np.savez_compressed(os.path.join(OUT, "newpfd_blocks.npz"), values=np.concatenate(ins),
                        n=np.array(ns, np.uint32), frac=np.array(fr, np.float32), words=np.concatenate(outs),
                        word_offsets=np.array(offs, np.uint64))


def fit_vectors():
    rng = np.random.default_rng(0xF17)
    ys, ns, seg, lrc = [], [], [], []
    for t in range(300):
        n = int(rng.integers(1, 700))
        ub = int(rng.choice([12, 20, 24, 28, 31]))
        n = min(n, (1 << ub) - 1)
        y = np.sort(rng.choice(1 << ub, size=n, replace=False)).astype(np.uint32)
        ys.append(y)
        ns.append(n)
        seg.append(oracle.ref_fit_seg_raw(y))
        lrc.append(oracle.ref_fit_lrc_raw(y))
    np.savez_compressed(os.path.join(OUT, "regression_fits.npz"), y=np.concatenate(ys), n=np.array(ns, np.uint32),
                        seglrc=np.stack(seg), lrc=np.stack(lrc))


def inverted_list_digest():
    """Digest of the reference encoding of the shipped InvertedList fixture
    (256-entry d-gap blocks, ParaPFD_Compression/main.cpp:163-189)."""
    docs = np.fromfile(INVERTED_LIST, dtype=np.uint32)
    gaps = np.empty_like(docs)
    gaps[0] = docs[0]
    gaps[1:] = np.diff(docs)
    rows = []
    for frac in (0.0, 0.12):
        words = [oracle.ref_encode(gaps[s:s + 256], frac) for s in range(0, len(gaps), 256)]
        allw = np.concatenate(words)
        rows.append((frac, len(allw), hashlib.sha256(allw.tobytes()).hexdigest()))
    with open(os.path.join(OUT, "inverted_list_digest.txt"), "w") as f:
        f.write(f"# reference ParaPFor encoding of InvertedList ({len(docs)} postings), 256-blocks\n")
        f.write(f"postings {len(docs)} first {docs[0]} last {docs[-1]} sha256_docs "
                f"{hashlib.sha256(docs.tobytes()).hexdigest()}\n")
        for frac, nw, h in rows:
            f.write(f"frac {frac} words {nw} sha256 {h}\n")


def hash_info(d):
    """HS_SegLRC_Generator.cu:545-581 restated: the bucket shift from the
    length (kExceptedBucketSize 256) and each bucket's first element."""
    n = len(d)
    maxb = int(d[-1]).bit_length()
    if n <= 256:
        return maxb, [0, n]
    shift = maxb - ((n + 255) // 256).bit_length()
    nb = (int(d[-1]) >> shift) + 1
    off = [int(np.searchsorted(d, b << shift)) for b in range(nb)] + [n]
    return shift, off


def hs_file_set(lists):
    """HS_SegLRC file set (HS_SegLRC_Generator.cu:180-594, HS_SegLRC_Compression/
    main.cpp:78-190): per-bucket fits from the reference's getRegressionInfo,
    blocks from the reference's ParaPFor.cpp (FRAC 0). Residuals are computed
    against each element's own bucket; the reference generator's lower-bound
    search gives the first element after empty buckets to the first of them
    (HS_SegLRC_Generator_kernel.cu:73-85), so for a list with empty buckets
    this set differs from its output in exactly those elements' residuals and
    their buckets' bases and blocks (the list here that has them: the third)."""
    import struct

    ind1, ind2, hoff, hinfo, bnum, boff, base, reg = b"", [], [], [], [], [], [], []
    words_total = 0
    for d in lists:
        n = len(d)
        shift, off = hash_info(d)
        hoff.append(len(hinfo))
        hinfo += [shift, len(off) - 1] + off
        bnum.append(len(boff))
        enc = oracle.encode_list(d, 4, 256, 0.0, bucket=256)
        assert enc["shift"] == shift and np.array_equal(enc["starts"], [o for o, e in zip(off, off[1:]) if e > o])
        ind1 += struct.pack("<IIQ", n, 0, 4 * words_total)
        nw, k = 0, 0
        for b in range(len(off) - 1):
            lo, hi = off[b], off[b + 1]
            boff.append(nw)
            if hi == lo:
                # an empty bucket as the generator leaves it: empty fit, next docID as base
                reg.append(oracle.ref_fit_seg_raw(np.zeros(0, np.uint32)))
                base.append(int(d[lo]))
                continue
            raw = oracle.ref_fit_seg_raw(d[lo:hi])
            assert np.array_equal(raw, enc["reg"][k]), "oracle bucket fit differs from the reference's"
            vals = oracle.decode_block(enc["words"][enc["off"][k]:], hi - lo)[0]
            reg.append(raw)
            base.append(int(enc["aux"][k]))
            w = oracle.ref_encode(np.ascontiguousarray(vals, np.uint32), 0.0)
            ind2.append(w)
            nw += len(w)
            k += 1
        words_total += nw
    return {".ind1": np.frombuffer(ind1, np.uint8), ".ind2": np.concatenate(ind2).view(np.uint8),
            ".HashSeg_offset": np.array(hoff, np.uint32).view(np.uint8),
            ".HashSeg_info": np.array(hinfo, np.uint32).view(np.uint8),
            ".segNum": np.array(bnum, np.uint32).view(np.uint8),
            ".segOffset": np.array(boff, np.uint32).view(np.uint8),
            ".ind2_distance_base": np.array(base, np.uint32).view(np.uint8),
            ".regression_info": np.stack(reg).reshape(-1).view(np.uint8)}


def reference_file_sets():
    """The reference's compressed file sets for a small seeded corpus, laid out
    as its compressors write them (ParaPFD_Compression/main.cpp:81-232,
    SegLRC_Compression/main.cpp:80-207, LRC_Compression/main.cpp:94-215,
    LRCSeg_Compression/main.cpp:78-200), every block encoded by the
    reference's own ParaPFor.cpp (NewPFor.cpp for NewPFD). ParaPFD: d-gaps
    over the whole list, FRAC 0.12. SegLRC / LRCSeg / LRC: fits from the
    reference's getRegressionInfo (the oracle's restated fits are pinned to it
    by regression_fits.npz) per segment / per list, residuals
    doc - (int)(i * a + b) (LRC: (int)((float)i * slope) + intercept) minus the
    segment's (LRC: the list's) minimum, FRAC 0. HS_SegLRC on its own corpus
    (hs_file_set)."""
    import struct

    rng = np.random.default_rng(0xF11E5)
    lens = [1, 100, 255, 256, 257, 700, 2000, 5000]
    lists = [np.sort(rng.choice(1 << 22, size=n, replace=False)).astype(np.uint32) for n in lens]
    out = {"docs": np.concatenate(lists), "lens": np.array(lens, np.uint32)}
    for codec, name, frac in ((0, "parapfd", 0.12), (3, "seglrc", 0.0), (6, "newpfd", 0.12), (1, "lrc", 0.0),
                              (2, "lrcseg", 0.0)):
        ind1, ind2, seg_num, heads, offs, aux, reg, listreg = b"", [], [], [], [], [], [], []
        words_total = 0
        for d in lists:
            n = len(d)
            seg_num.append(len(heads))
            if codec in (0, 6):
                gaps = np.empty_like(d)
                gaps[0] = d[0]
                gaps[1:] = np.diff(d)
                vals, med = gaps, [int(d[s + min(256, n - s) // 2]) for s in range(0, n, 256)]
                segvals = [vals[s:s + 256] for s in range(0, n, 256)]
            else:
                enc = oracle.encode_list(d, codec, 256, 0.0)
                segvals = [oracle.decode_block(enc["words"][o:], int(c))[0] for o, c in zip(enc["off"], enc["counts"])]
                med = [int(x) for x in enc["aux"]]
                reg.append(enc["reg"].astype(np.uint32))
                listreg.append(enc["listreg"].astype(np.uint32))
                if codec == 3:
                    for k, (s0, c) in enumerate(zip(enc["starts"], enc["counts"])):
                        raw = oracle.ref_fit_seg_raw(d[s0:s0 + c])
                        assert np.array_equal(raw, enc["reg"][k]), "oracle segment fit differs from the reference's"
                if codec in (2, 3):
                    assert np.array_equal(oracle.ref_fit_seg_raw(d), enc["listreg"]), "list fit differs"
                else:
                    # LRC: slope and range as the reference's fit; the intercept moved by the residual minimum
                    raw = oracle.ref_fit_lrc_raw(d)
                    assert raw[0] == enc["listreg"][0] and raw[2] == enc["listreg"][2], "LRC fit differs"
            ind1 += struct.pack("<IIQ", n, 0, 4 * words_total)
            nw = 0
            for k, v in enumerate(segvals):
                heads.append(int(d[256 * k]))
                offs.append(nw)
                enc_fn = oracle.ref_newpfd_encode if codec == 6 else oracle.ref_encode
                w = enc_fn(np.ascontiguousarray(v, np.uint32), frac)
                ind2.append(w)
                nw += len(w)
            aux.extend(med)
            words_total += nw
        files = {".ind1": np.frombuffer(ind1, np.uint8),
                 ".ind2": np.concatenate(ind2).view(np.uint8),
                 ".segNum": np.array(seg_num, np.uint32).view(np.uint8),
                 ".segHead": np.array(heads, np.uint32).view(np.uint8),
                 ".segOffset": np.array(offs, np.uint32).view(np.uint8)}
        if codec in (0, 6):
            files[".segMedian"] = np.array(aux, np.uint32).view(np.uint8)
        elif codec == 3:
            files[".ind2_distance_base"] = np.array(aux, np.uint32).view(np.uint8)
            files[".regression_info"] = np.concatenate(reg).reshape(-1).view(np.uint8)
            files[".regression_info_list"] = np.stack(listreg).reshape(-1).view(np.uint8)
        elif codec == 2:
            files[".ind2_distance_base"] = np.array(aux, np.uint32).view(np.uint8)
            files[".regression_info"] = np.stack(listreg).reshape(-1).view(np.uint8)
        else:
            files[".regression_info"] = np.stack(listreg)[:, :3].reshape(-1).view(np.uint8)
        for suffix, data in files.items():
            out[name + suffix] = data
    # HS_SegLRC: uniform lists, a clustered one with empty buckets, short ones
    hrng = np.random.default_rng(0x4A5B)
    hl = [np.sort(hrng.choice(1 << 22, size=n, replace=False)).astype(np.uint32) for n in (3000, 700)]
    gap = np.concatenate([hrng.choice(1 << 18, size=600, replace=False),
                          (3 << 20) + hrng.choice(1 << 18, size=600, replace=False)])
    hl.append(np.sort(gap).astype(np.uint32))
    hl += [np.sort(hrng.choice(1 << 22, size=n, replace=False)).astype(np.uint32) for n in (1, 256, 257)]
    out["hs_docs"] = np.concatenate(hl)
    out["hs_lens"] = np.array([len(x) for x in hl], np.uint32)
    for suffix, data in hs_file_set(hl).items():
        out["hs_seglrc" + suffix] = data
    # a .query stream over the corpus (ParaPFD_Intersection.cu:139-142)
    q = [[6, 7], [5, 6, 7], [0, 7], [7, 4, 3], [2, 2], [1]]
    out["queries"] = np.array([x for t in q for x in [len(t)] + t], np.uint32).view(np.uint8)
    np.savez_compressed(os.path.join(OUT, "reference_files.npz"), **out)


if __name__ == "__main__":
    assert oracle.have_ref_codec() and oracle.have_ref_fit() and oracle.have_ref_newpfd(), \
        "build the reference first: make -C oracle ref"
    codec_vectors()
    fit_vectors()
    newpfd_vectors()
    reference_file_sets()
    if os.path.exists(INVERTED_LIST):
        inverted_list_digest()
    print("golden fixtures written to", OUT)
