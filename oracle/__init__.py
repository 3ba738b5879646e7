"""CPU ORACLE — test infrastructure only.

ctypes wrapper of oracle/liboracle.so (oracle.c: a plain-C restatement of the
reference's ParaPFD codec, list formats, regression arithmetic, hash-segment
partition, exact intersection and checksum), and of the reference's own code
compiled from its sources into oracle/_ref/ (ParaPFor.cpp; the generators'
getRegressionInfo). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs use this package, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_CODEC = os.path.join(HERE, "_ref", "libparapfor_ref.so")
REF_NEWPFD = os.path.join(HERE, "_ref", "libnewpfor_ref.so")
REF_FIT = os.path.join(HERE, "_ref", "libfit_ref.so")
# Root of the reference source tree used by the pinning builds and tests; the
# EXCL_REFERENCE environment variable overrides the default location.
REFERENCE = os.environ.get("EXCL_REFERENCE", "/root/reference")


def have_reference_tree() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "src", "gpu"))


def build(ref: bool | None = None) -> None:
    """make -C oracle (and the reference builds when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref is None:
        ref = have_reference_tree()
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE}"], check=True)


if not os.path.exists(LIB):
    build(ref=False)
_lib = C.CDLL(LIB)

u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)
u64p = C.POINTER(C.c_uint64)


def _f(lib, name, res, *args):
    fn = getattr(lib, name)
    fn.restype = res
    fn.argtypes = list(args)
    return fn


_enc_block = _f(_lib, "or_parapfd_encode_block", C.c_uint32, u32p, C.c_uint32, C.c_float, u32p, C.POINTER(C.c_int))
_dec_block = _f(_lib, "or_parapfd_decode_block", C.c_uint32, u32p, C.c_uint32, u32p)
_nenc_block = _f(_lib, "or_newpfd_encode_block", C.c_uint32, u32p, C.c_uint32, C.c_float, u32p, C.POINTER(C.c_int))
_ndec_block = _f(_lib, "or_newpfd_decode_block", C.c_uint32, u32p, C.c_uint32, u32p)
_enc_npfd = _f(_lib, "or_encode_newpfd_list", C.c_int64, u32p, C.c_uint32, C.c_uint32, C.c_float, u32p, u32p, u32p,
               u32p)
_fit_seg = _f(_lib, "or_fit_seg", None, u32p, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), u32p, u32p)
_fit_lrc = _f(_lib, "or_fit_lrc", None, u32p, C.c_uint32, C.POINTER(C.c_float), i32p, C.POINTER(C.c_float))
_enc_pfd = _f(_lib, "or_encode_parapfd_list", C.c_int64, u32p, C.c_uint32, C.c_uint32, C.c_float, u32p, u32p, u32p,
              u32p)
_enc_pfd_segs = _f(_lib, "or_encode_parapfd_segs", C.c_int64, u32p, C.c_uint32, C.c_uint32, u32p, C.c_float, u32p,
                   u32p, u32p, u32p)
_enc_res = _f(_lib, "or_encode_residual_list", C.c_int64, C.c_int, u32p, C.c_uint32, C.c_uint32, u32p, C.c_float,
              u32p, u32p, u32p, u32p, i32p, u32p)
_hs = _f(_lib, "or_hs_partition", C.c_uint32, u32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p)
_dec_list = _f(_lib, "or_decode_list", C.c_int, C.c_int, u32p, C.c_uint32, C.c_uint32, u32p, u32p, u32p, u32p, i32p,
               u32p, u32p)
_isect = _f(_lib, "or_intersect", C.c_uint64, C.c_uint32, C.POINTER(u32p), u64p, u32p)
_cs = _f(_lib, "or_checksum", None, C.c_uint32, u64p, u32p, u64p)
_runq = _f(_lib, "or_run_queries", C.c_double, u32p, u64p, u32p, u64p, C.c_uint32, C.c_uint32, C.c_uint64, u64p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _p(a: np.ndarray, t=u32p):
    return a.ctypes.data_as(t)


def encode_block(values, frac: float = 0.0) -> np.ndarray:
    v = _u32(values)
    out = np.zeros(3 * len(v) + 8, dtype=np.uint32)
    err = C.c_int(0)
    w = _enc_block(_p(v), len(v), frac, _p(out), C.byref(err))
    if err.value:
        raise ValueError("block not representable in ParaPFD")
    return out[:w].copy()


def decode_block(words, n: int) -> tuple[np.ndarray, int]:
    w = np.zeros(len(words) + 4, dtype=np.uint32)
    w[: len(words)] = words
    out = np.zeros(max(n, 1), dtype=np.uint32)
    used = _dec_block(_p(w), n, _p(out))
    return out[:n], int(used)


def newpfd_encode_block(values, frac: float = 0.0) -> np.ndarray:
    v = _u32(values)
    out = np.zeros(3 * len(v) + 8, dtype=np.uint32)
    err = C.c_int(0)
    w = _nenc_block(_p(v), len(v), frac, _p(out), C.byref(err))
    if err.value:
        raise ValueError("block not representable in NewPFD")
    return out[:w].copy()


def newpfd_decode_block(words, n: int) -> tuple[np.ndarray, int]:
    w = np.zeros(len(words) + 4, dtype=np.uint32)
    w[: len(words)] = words
    out = np.zeros(max(n, 1), dtype=np.uint32)
    used = _ndec_block(_p(w), n, _p(out))
    return out[:n], int(used)


def fit_seg(y) -> tuple[float, float, int, int]:
    y = _u32(y)
    a, b = C.c_float(), C.c_float()
    L, R = C.c_uint32(), C.c_uint32()
    _fit_seg(_p(y), len(y), C.byref(a), C.byref(b), C.byref(L), C.byref(R))
    return a.value, b.value, L.value, R.value


def fit_seg_raw(y) -> np.ndarray:
    a, b, L, R = fit_seg(y)
    return np.array([np.float32(a).view(np.uint32), np.float32(b).view(np.uint32), L, R], dtype=np.uint32)


def fit_lrc_raw(y) -> np.ndarray:
    y = _u32(y)
    s, r = C.c_float(), C.c_float()
    i = C.c_int32()
    _fit_lrc(_p(y), len(y), C.byref(s), C.byref(i), C.byref(r))
    return np.array([np.float32(s.value).view(np.uint32), np.int32(i.value).view(np.uint32),
                     np.float32(r.value).view(np.uint32)], dtype=np.uint32)


def hs_partition(docs, bucket: int = 256, kbits: int = 0, ubits: int = 32) -> tuple[int, np.ndarray]:
    d = _u32(docs)
    nb_max = (int(d[-1]) >> max(0, ubits - kbits)) + 2 if kbits else len(d) * 2 + 4
    bnd = np.zeros(nb_max + 2, dtype=np.uint32)
    sh = C.c_uint32()
    nb = _hs(_p(d), len(d), bucket, kbits, ubits, C.byref(sh), _p(bnd))
    return int(sh.value), bnd[: nb + 1].copy()


CODECS = {"parapfd": 0, "lrc": 1, "lrcseg": 2, "seglrc": 3, "hs_seglrc": 4, "hs_parapfd": 5}


def segment_starts(docs, codec: int, block: int, bucket: int = 256, kbits: int = 0, ubits: int = 32):
    """Segment start elements of a list, as the formats cut it: fixed blocks, or
    the non-empty buckets (HS_SegLRC) / blocks inside buckets (HS_ParaPFD).
    Returns (starts, shift, bucket->first segment table or None)."""
    n = len(docs)
    if codec not in (4, 5):
        return np.arange(0, n, block, dtype=np.uint32), None, None
    shift, bnd = hs_partition(docs, bucket, kbits, ubits)
    starts, first = [], []
    for b in range(len(bnd) - 1):
        first.append(len(starts))
        lo, hi = int(bnd[b]), int(bnd[b + 1])
        step = block if codec == 5 else max(hi - lo, 1)
        for k in range(lo, hi, step):
            starts.append(k)
    first.append(len(starts))
    return np.array(starts, dtype=np.uint32), shift, np.array(first, dtype=np.uint32)


def encode_list(docs, codec: int, block: int = 256, frac: float = 0.0, bucket: int = 256, kbits: int = 0,
                ubits: int = 32) -> dict:
    """Oracle encoding of one list in the given codec: blocks and metadata."""
    d = _u32(docs)
    n = len(d)
    starts, shift, first = segment_starts(d, codec, block, bucket, kbits, ubits)
    ns = len(starts)
    words = np.zeros(3 * n + 8 * ns + 8, dtype=np.uint32)
    off = np.zeros(ns, dtype=np.uint32)
    head = np.zeros(ns, dtype=np.uint32)
    aux = np.zeros(ns, dtype=np.uint32)
    reg = np.zeros((ns, 4), dtype=np.uint32)
    base = np.zeros(ns, dtype=np.int32)
    listreg = np.zeros(4, dtype=np.uint32)
    if codec == 6:
        w = _enc_npfd(_p(d), n, block, frac, _p(words), _p(off), _p(head), _p(aux))
    elif codec in (0, 5):
        if codec == 0:
            w = _enc_pfd(_p(d), n, block, frac, _p(words), _p(off), _p(head), _p(aux))
        else:
            w = _enc_pfd_segs(_p(d), n, ns, _p(starts), frac, _p(words), _p(off), _p(head), _p(aux))
    else:
        ocodec = 4 if codec == 4 else codec
        w = _enc_res(ocodec, _p(d), n, ns, _p(starts), frac, _p(words), _p(off), _p(head), _p(reg),
                     _p(base, i32p), _p(listreg))
        aux = base.view(np.uint32)
    if w < 0:
        raise ValueError("list not representable in this format")
    counts = np.diff(np.append(starts, n)).astype(np.uint32)
    return dict(words=words[:w].copy(), off=off, head=head, aux=aux, reg=reg, listreg=listreg, starts=starts,
                counts=counts, shift=shift, first=first)


def decode_list(enc: dict, codec: int, n: int) -> np.ndarray:
    words = np.zeros(len(enc["words"]) + 8, dtype=np.uint32)
    words[: len(enc["words"])] = enc["words"]
    out = np.zeros(max(n, 1), dtype=np.uint32)
    ocodec = {0: 0, 5: 0, 1: 1, 2: 2, 3: 3, 4: 3, 6: 6}[codec]
    reg = np.ascontiguousarray(enc["reg"].reshape(-1), dtype=np.uint32)
    base = np.ascontiguousarray(enc["aux"]).view(np.int32)
    _dec_list(ocodec, _p(words), n, len(enc["starts"]), _p(_u32(enc["starts"])), _p(_u32(enc["off"])),
              _p(_u32(enc["head"])), _p(reg), _p(np.ascontiguousarray(base), i32p), _p(_u32(enc["listreg"])),
              _p(out))
    return out[:n]


def intersect(lists) -> np.ndarray:
    arrs = [_u32(a) for a in lists]
    if not arrs:
        return np.zeros(0, dtype=np.uint32)
    ptrs = (u32p * len(arrs))(*[_p(a) if len(a) else _p(np.zeros(1, np.uint32)) for a in arrs])
    lens = np.array([len(a) for a in arrs], dtype=np.uint64)
    out = np.zeros(max(1, min(len(a) for a in arrs)), dtype=np.uint32)
    r = _isect(len(arrs), ptrs, _p(lens, u64p), _p(out))
    return out[:r].copy()


def run_queries(docs, list_offsets, terms, term_offsets, threads: int = 1) -> tuple[float, np.ndarray]:
    """Exact AND of every query on `threads` host threads; (seconds, counts)."""
    d = _u32(docs)
    lo = np.ascontiguousarray(list_offsets, dtype=np.uint64)
    t = _u32(terms) if len(terms) else np.zeros(1, np.uint32)
    to = np.ascontiguousarray(term_offsets, dtype=np.uint64)
    nq = len(to) - 1
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    maxl = int(np.diff(lo).max()) if len(lo) > 1 else 1
    secs = _runq(_p(d), _p(lo, u64p), _p(t), _p(to, u64p), nq, threads, maxl, _p(counts, u64p))
    return float(secs), counts[:nq]


_runqc = _f(_lib, "or_run_queries_compressed", C.c_double, u32p, u32p, u32p, u32p, u32p, u64p, u32p, u32p, u32p,
            u32p, u32p, u64p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u64p)


class CompressedImage:
    """The arrays of a compressed index, laid out for the compressed CPU path:
    from an exported index (`arrays`), or from encode_corpus (oracle encoder)."""

    def __init__(self, arrays=None):
        if arrays is None:
            return
        L = arrays.lists
        self.words = np.ascontiguousarray(arrays.words, dtype=np.uint32)
        self.lcodec = np.ascontiguousarray(L["codec"], dtype=np.uint32)
        self.ln = np.ascontiguousarray(L["n"], dtype=np.uint32)
        self.lseg = np.ascontiguousarray(L["seg_base"], dtype=np.uint32)
        self.lnseg = np.ascontiguousarray(L["nseg"], dtype=np.uint32)
        self.lword = np.ascontiguousarray(L["word_base"], dtype=np.uint64)
        self.lreg = np.ascontiguousarray(np.stack([np.asarray(L["reg"][:, i]) for i in range(4)], axis=1)
                                         if len(L) else np.zeros((0, 4)), dtype=np.uint32).reshape(-1)
        self.head = np.ascontiguousarray(arrays.seg_head, dtype=np.uint32)
        self.rec = np.ascontiguousarray(arrays.seg_rec, dtype=np.uint32).reshape(-1)
        self.sreg = np.ascontiguousarray(arrays.seg_reg, dtype=np.uint32).reshape(-1)
        self.max_list = int(self.ln.max()) if len(self.ln) else 1
        self.max_seg = int(arrays.seg_rec[:, 3].max()) if len(arrays.seg_rec) else 1


def run_queries_compressed(img: CompressedImage, terms, term_offsets, threads: int = 1):
    """Decode + exact AND of every query on the compressed image; (seconds, counts)."""
    t = _u32(terms) if len(terms) else np.zeros(1, np.uint32)
    to = np.ascontiguousarray(term_offsets, dtype=np.uint64)
    nq = len(to) - 1
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    secs = _runqc(_p(img.words), _p(img.lcodec), _p(img.ln), _p(img.lseg), _p(img.lnseg), _p(img.lword, u64p),
                  _p(img.lreg), _p(img.head), _p(img.rec), _p(img.sreg), _p(t), _p(to, u64p), nq, threads,
                  img.max_list, img.max_seg, _p(counts, u64p))
    return float(secs), counts[:nq]


_mlp_grad = _f(_lib, "or_mlp_grad", None, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
               C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double))
_model_check = _f(_lib, "or_model_check", C.c_uint64, C.POINTER(C.c_float), C.c_float, C.c_float, C.c_uint32,
                  i32p, u32p, C.c_uint64, u32p)

MLP_PARAMS = 1153


def mlp_grad(params, x, y) -> tuple[np.ndarray, float]:
    """Double-precision gradient of the mean squared error of the root MLP."""
    P = np.ascontiguousarray(params, dtype=np.float32)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    ys = np.ascontiguousarray(y, dtype=np.float32)
    g = np.zeros(MLP_PARAMS, dtype=np.float64)
    loss = C.c_double(0)
    fp = C.POINTER(C.c_float)
    _mlp_grad(P.ctypes.data_as(fp), xs.ctypes.data_as(fp), ys.ctypes.data_as(fp), len(xs),
              g.ctypes.data_as(C.POINTER(C.c_double)), C.byref(loss))
    return g, loss.value


_model_leaves = _f(_lib, "or_model_leaves", None, C.POINTER(C.c_float), C.c_float, C.c_float, C.c_uint32, u32p,
                   C.c_uint64, u32p)


def model_leaves(root, hdr4, keys) -> np.ndarray:
    """Leaf of each key as the root network routes it (FP32 restatement)."""
    P = np.ascontiguousarray(root, dtype=np.float32)
    k = _u32(keys)
    out = np.zeros(max(len(k), 1), dtype=np.uint32)
    _model_leaves(P.ctypes.data_as(C.POINTER(C.c_float)), float(hdr4[0]), float(hdr4[1]), int(hdr4[2]), _p(k), len(k),
                  _p(out))
    return out[:len(k)]


def model_check(root, hdr4, leaves, keys) -> tuple[int, np.ndarray]:
    """Keys whose rank falls outside their leaf's window (0 = exact), and keys per leaf."""
    P = np.ascontiguousarray(root, dtype=np.float32)
    lv = np.ascontiguousarray(leaves, dtype=np.int32).reshape(-1)
    k = _u32(keys)
    L = int(hdr4[2])
    counts = np.zeros(L, dtype=np.uint32)
    bad = _model_check(P.ctypes.data_as(C.POINTER(C.c_float)), float(hdr4[0]), float(hdr4[1]), L,
                       lv.ctypes.data_as(i32p), _p(k), len(k), _p(counts))
    return int(bad), counts


def answer(docs, list_offsets, terms, term_offsets) -> tuple[np.ndarray, np.ndarray]:
    """Expected (offsets[nq+1], docids) of a batch."""
    lo = np.asarray(list_offsets, dtype=np.uint64)
    to = np.asarray(term_offsets, dtype=np.uint64)
    res, offs = [], [0]
    for q in range(len(to) - 1):
        ts = terms[int(to[q]):int(to[q + 1])]
        if len(ts) == 0:
            r = np.zeros(0, dtype=np.uint32)
        else:
            r = intersect([docs[int(lo[t]):int(lo[t + 1])] for t in ts])
        res.append(r)
        offs.append(offs[-1] + len(r))
    return np.array(offs, dtype=np.uint64), (np.concatenate(res) if res else np.zeros(0, np.uint32))


def checksum(offsets, docids) -> tuple[int, int, int]:
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    d = _u32(docids) if len(docids) else np.zeros(1, np.uint32)
    cs = np.zeros(3, dtype=np.uint64)
    _cs(len(o) - 1, _p(o, u64p), _p(d), _p(cs, u64p))
    return int(cs[0]), int(cs[1]), int(cs[2])


# ---------------------------------------------------------------------------
# The reference's own code (built from its sources; absent off this machine
# unless oracle/_ref travelled with the tree).

def have_ref_codec() -> bool:
    return os.path.exists(REF_CODEC)


def have_ref_fit() -> bool:
    return os.path.exists(REF_FIT)


_ref_codec = None
_ref_fit = None


def _rc():
    global _ref_codec
    if _ref_codec is None:
        lib = C.CDLL(REF_CODEC)
        _f(lib, "ref_set_frac", None, C.c_float)
        _f(lib, "ref_encode", C.c_uint32, u32p, u32p, C.c_uint32)
        _f(lib, "ref_decode", C.c_uint32, u32p, u32p, C.c_uint32)
        _ref_codec = lib
    return _ref_codec


def ref_encode(values, frac: float) -> np.ndarray:
    v = _u32(values)
    out = np.zeros(3 * len(v) + 16, dtype=np.uint32)
    lib = _rc()
    lib.ref_set_frac(frac)
    w = lib.ref_encode(_p(v), _p(out), len(v))
    return out[:w].copy()


def ref_decode(words, n: int) -> tuple[np.ndarray, int]:
    w = np.zeros(len(words) + 4, dtype=np.uint32)
    w[: len(words)] = words
    out = np.zeros(max(n, 1) + 2, dtype=np.uint32)
    used = _rc().ref_decode(_p(w), _p(out), n)
    return out[:n].copy(), int(used)


def have_ref_newpfd() -> bool:
    return os.path.exists(REF_NEWPFD)


_ref_newpfd = None


def _rn():
    global _ref_newpfd
    if _ref_newpfd is None:
        lib = C.CDLL(REF_NEWPFD)
        _f(lib, "ref_newpfd_set_frac", None, C.c_float)
        _f(lib, "ref_newpfd_encode", C.c_uint32, u32p, u32p, C.c_uint32)
        _f(lib, "ref_newpfd_decode", C.c_uint32, u32p, u32p, C.c_uint32)
        _ref_newpfd = lib
    return _ref_newpfd


def ref_newpfd_encode(values, frac: float) -> np.ndarray:
    v = _u32(values)
    out = np.zeros(3 * len(v) + 16, dtype=np.uint32)
    lib = _rn()
    lib.ref_newpfd_set_frac(frac)
    w = lib.ref_newpfd_encode(_p(v), _p(out), len(v))
    return out[:w].copy()


def ref_newpfd_decode(words, n: int) -> tuple[np.ndarray, int]:
    w = np.zeros(len(words) + 32, dtype=np.uint32)
    w[: len(words)] = words
    out = np.zeros(max(n, 1) + 2, dtype=np.uint32)
    used = _rn().ref_newpfd_decode(_p(w), _p(out), n)
    return out[:n].copy(), int(used)


def _rf():
    global _ref_fit
    if _ref_fit is None:
        lib = C.CDLL(REF_FIT)
        _f(lib, "ref_fit_seglrc", None, u32p, C.c_uint32, u32p)
        _f(lib, "ref_fit_lrc", None, u32p, C.c_uint32, u32p)
        _ref_fit = lib
    return _ref_fit


def ref_fit_seg_raw(y) -> np.ndarray:
    y = _u32(y)
    out = np.zeros(4, dtype=np.uint32)
    _rf().ref_fit_seglrc(_p(y), len(y), _p(out))
    return out


def ref_fit_lrc_raw(y) -> np.ndarray:
    y = _u32(y)
    out = np.zeros(3, dtype=np.uint32)
    _rf().ref_fit_lrc(_p(y), len(y), _p(out))
    return out


# ---------------------------------------------------------------------------
# The benchmark's seeded workloads, restated here (workloads.c) so the CPU
# reference arm needs no product code; whole-corpus encoding with this
# oracle's encoders; exact answers of whole batches on host threads.

_wl_new = {
    "pairs": _f(_lib, "or_wl_pairs", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                C.c_uint32),
    "zipf": _f(_lib, "or_wl_zipf_corpus", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
               C.c_uint32, C.c_uint32, C.c_uint32),
    "skewed": _f(_lib, "or_wl_skewed", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                 C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32),
    "learned": _f(_lib, "or_wl_learned", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                  C.c_uint32, C.c_double, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32),
    "serving": _f(_lib, "or_wl_serving", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                  C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32),
}
_wl_free = _f(_lib, "or_wl_free", None, C.c_void_p)
_wl_get = {n: _f(_lib, "or_wl_" + n, r, C.c_void_p) for n, r in (
    ("ndocs", C.c_uint64), ("nlists", C.c_uint32), ("nqueries", C.c_uint32), ("nterms", C.c_uint64),
    ("ninfo", C.c_uint32), ("docs", C.c_void_p), ("loff", C.c_void_p), ("terms", C.c_void_p), ("toff", C.c_void_p),
    ("codecs", C.c_void_p), ("info", C.c_void_p))}


class Workload:
    """Concatenated sorted docID lists (list_offsets), queries (term_offsets)."""

    def __init__(self, docs, list_offsets, terms, term_offsets, codecs, info):
        self.docs, self.list_offsets, self.terms, self.term_offsets = docs, list_offsets, terms, term_offsets
        self.codecs, self.info = codecs, info

    @property
    def nlists(self) -> int:
        return len(self.list_offsets) - 1

    @property
    def nq(self) -> int:
        return len(self.term_offsets) - 1

    def list(self, i: int) -> np.ndarray:
        return self.docs[self.list_offsets[i]:self.list_offsets[i + 1]]


def _wl_arr(ptr, n, ct, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy()


def _wl_take(h) -> Workload:
    g = _wl_get
    try:
        nd, nl, nq, nt, ni = g["ndocs"](h), g["nlists"](h), g["nqueries"](h), g["nterms"](h), g["ninfo"](h)
        cod = g["codecs"](h)
        return Workload(_wl_arr(g["docs"](h), nd, C.c_uint32, np.uint32),
                        _wl_arr(g["loff"](h), nl + 1, C.c_uint64, np.uint64),
                        _wl_arr(g["terms"](h), nt, C.c_uint32, np.uint32),
                        _wl_arr(g["toff"](h), nq + 1, C.c_uint32, np.uint32),
                        _wl_arr(cod, nl, C.c_uint8, np.uint8) if cod else None,
                        _wl_arr(g["info"](h), ni, C.c_double, np.float64))
    finally:
        _wl_free(h)


def _threads(t: int) -> int:
    return t if t > 0 else (os.cpu_count() or 1)


def wl_pairs(seed=0xEC1E0001, npairs=1000, short_len=4096, long_len=1 << 20, ubits=23, threads=0) -> Workload:
    return _wl_take(_wl_new["pairs"](seed, npairs, short_len, long_len, ubits, _threads(threads)))


def wl_zipf_corpus(seed=0xEC1E0002, ndocs=10_000_000, nterms=100_000, cap=5_000_000, nq=10_000, qmin=2, qmax=5,
                   threads=0) -> Workload:
    return _wl_take(_wl_new["zipf"](seed, ndocs, nterms, cap, nq, qmin, qmax, _threads(threads)))


def wl_skewed(seed=0xEC1E0003, ubits=26, npool=32, long_min=1_000_000, long_max=20_000_000, nq=5000,
              short_min=1000, short_max=10_000, run_mean=64.0, gap_mean=4096.0, threads=0) -> Workload:
    return _wl_take(_wl_new["skewed"](seed, ubits, npool, long_min, long_max, nq, short_min, short_max, run_mean,
                                      gap_mean, _threads(threads)))


def wl_learned(seed=0xEC1E0004, ubits=31, nclust=64, nzipf=64, lmin=10_000_000, lmax=100_000_000, zipf_s=1.2,
               zipf_cap=1 << 20, nq=20_000, kmin=1000, kmax=100_000, threads=0) -> Workload:
    return _wl_take(_wl_new["learned"](seed, ubits, nclust, nzipf, lmin, lmax, zipf_s, zipf_cap, nq, kmin, kmax,
                                       _threads(threads)))


def wl_serving(seed=0xEC1E0005, ubits=28, nterms=2_000_000, total=1_000_000_000, nq=100_000, qmin=2, qmax=8,
               pfd_below=10_000, threads=0) -> Workload:
    return _wl_take(_wl_new["serving"](seed, ubits, nterms, total, nq, qmin, qmax, pfd_below, _threads(threads)))


_corpus_plan = _f(_lib, "or_corpus_plan", None, u32p, u64p, C.c_uint32, C.POINTER(C.c_uint8), C.c_uint32,
                  C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p)
_corpus_enc = _f(_lib, "or_corpus_encode", C.c_int, u32p, u64p, C.c_uint32, C.POINTER(C.c_uint8), C.c_uint32,
                 C.c_float, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u32p, u64p, u64p, u32p, u32p, u32p, u32p,
                 u32p, u32p)


def encode_corpus(docs, list_offsets, codecs, block: int = 256, frac: float = 0.0, bucket: int = 256,
                  kbits: int = 0, ubits: int = 32, threads: int = 0) -> CompressedImage:
    """Every list encoded by this oracle's block encoders (per-list codec ids
    as in CODECS, or one id for all), as the compressed CPU path's image."""
    d = _u32(docs)
    lo = np.ascontiguousarray(list_offsets, dtype=np.uint64)
    nl = len(lo) - 1
    cod = (np.full(nl, int(codecs), dtype=np.uint8) if np.isscalar(codecs)
           else np.ascontiguousarray(codecs, dtype=np.uint8))
    cp = cod.ctypes.data_as(C.POINTER(C.c_uint8))
    th = _threads(threads)
    nseg = np.zeros(max(nl, 1), dtype=np.uint32)
    _corpus_plan(_p(d), _p(lo, u64p), nl, cp, block, bucket, kbits, ubits, th, _p(nseg))
    nseg = nseg[:nl]
    seg_base = np.zeros(nl + 1, dtype=np.uint64)
    np.cumsum(nseg, out=seg_base[1:])
    lens = np.diff(lo)
    slot = 3 * lens + 8 * nseg.astype(np.uint64) + 8
    word_cap = np.zeros(nl + 1, dtype=np.uint64)
    np.cumsum(slot, out=word_cap[1:])
    ns = int(seg_base[-1])
    words = np.zeros(int(word_cap[-1]) + 8, dtype=np.uint32)
    nwords = np.zeros(max(nl, 1), dtype=np.uint32)
    head = np.zeros(max(ns, 1), dtype=np.uint32)
    rec = np.zeros(4 * max(ns, 1), dtype=np.uint32)
    sreg = np.zeros(4 * max(ns, 1), dtype=np.uint32)
    lreg = np.zeros(4 * max(nl, 1), dtype=np.uint32)
    r = _corpus_enc(_p(d), _p(lo, u64p), nl, cp, block, frac, bucket, kbits, ubits, th, _p(nseg),
                    _p(seg_base, u64p), _p(word_cap, u64p), _p(words), _p(nwords), _p(head), _p(rec), _p(sreg),
                    _p(lreg))
    if r != 0:
        raise ValueError("a list is not representable in its format")
    # pack the per-list word slots back to back
    nw = nwords[:nl].astype(np.int64)
    base = np.zeros(nl + 1, dtype=np.uint64)
    np.cumsum(nw, out=base[1:])
    packed = np.zeros(int(base[-1]) + 8, dtype=np.uint32)
    idx = (np.repeat(word_cap[:-1].astype(np.int64), nw) + np.arange(int(base[-1]), dtype=np.int64) -
           np.repeat(base[:-1].astype(np.int64), nw))
    packed[: int(base[-1])] = words[idx]
    img = CompressedImage()
    img.words = packed
    img.lcodec = cod.astype(np.uint32)
    img.ln = lens.astype(np.uint32)
    img.lseg = seg_base[:-1].astype(np.uint32)
    img.lnseg = nseg.astype(np.uint32)
    img.lword = np.ascontiguousarray(base[:-1])
    img.lreg = lreg
    img.head = head
    img.rec = rec
    img.sreg = sreg
    img.max_list = int(lens.max()) if nl else 1
    img.max_seg = int(rec[3::4].max()) if ns else 1
    img.nsegs = ns
    return img


_ans_pass = _f(_lib, "or_answer_pass", None, u32p, u64p, u32p, u64p, C.c_uint32, C.c_uint32, C.c_uint64, u64p, u64p,
               u32p)


def answer_batch(docs, list_offsets, terms, term_offsets, threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """answer() on host threads: exact (offsets[nq+1], docids) of a batch."""
    d = _u32(docs)
    lo = np.ascontiguousarray(list_offsets, dtype=np.uint64)
    t = _u32(terms) if len(terms) else np.zeros(1, np.uint32)
    to = np.ascontiguousarray(term_offsets, dtype=np.uint64)
    nq = len(to) - 1
    th = _threads(threads)
    counts = np.zeros(max(nq, 1), dtype=np.uint64)
    maxl = int(np.diff(lo).max()) if len(lo) > 1 else 1
    _ans_pass(_p(d), _p(lo, u64p), _p(t), _p(to, u64p), nq, th, maxl, _p(counts, u64p), None, None)
    offs = np.zeros(nq + 1, dtype=np.uint64)
    np.cumsum(counts[:nq], out=offs[1:])
    out = np.zeros(max(int(offs[-1]), 1), dtype=np.uint32)
    _ans_pass(_p(d), _p(lo, u64p), _p(t), _p(to, u64p), nq, th, maxl, None, _p(offs, u64p), _p(out))
    return offs, out[: int(offs[-1])]
