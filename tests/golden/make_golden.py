"""Writes tests/golden/*.npz from the reference's own code compiled from its
sources (oracle/_ref: ParaPFor.cpp and the generators' getRegressionInfo).

Run in a tree that has the reference sources at /root/reference:
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
INVERTED_LIST = "/root/reference/src/gpu/Preprocess/ExtractList/data/InvertedList"


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


if __name__ == "__main__":
    assert oracle.have_ref_codec() and oracle.have_ref_fit(), "build the reference first: make -C oracle ref"
    codec_vectors()
    fit_vectors()
    if os.path.exists(INVERTED_LIST):
        inverted_list_digest()
    print("golden fixtures written to", OUT)
