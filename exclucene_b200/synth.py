"""ctypes binding of libexcl_synth.so: seeded synthetic workloads.

The reference's Baidu/GOV2 indexes and query logs are not available; these
generators stand in for them with the shapes of the five workloads (uniform,
Zipf-frequency corpora, clustered-run mixtures and Zipf-gap lists).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libexcl_synth.so")
if not os.path.exists(_LIB_PATH):
    raise ImportError(f"{_LIB_PATH} is not built; run `python -m exclucene_b200.build`")
_lib = C.CDLL(_LIB_PATH)

u32p = C.POINTER(C.c_uint32)


def _f(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_pairs = _f("synth_pairs", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32)
_zipf = _f("synth_zipf_corpus", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
           C.c_uint32, C.c_uint32)
_skew = _f("synth_skewed", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
           C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_uint32)
_learn = _f("synth_learned", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
            C.c_double, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32)
_serve = _f("synth_serving", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32,
            C.c_uint32, C.c_uint32, C.c_uint32)
_unif = _f("synth_uniform_lists", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, u32p, C.c_uint32)
_clus = _f("synth_clustered_lists", C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, u32p, C.c_double, C.c_double,
           C.c_uint32)
_free = _f("synth_free", None, C.c_void_p)
_ndocs = _f("synth_ndocs", C.c_uint64, C.c_void_p)
_nlists = _f("synth_nlists", C.c_uint32, C.c_void_p)
_nq = _f("synth_nqueries", C.c_uint32, C.c_void_p)
_nterms = _f("synth_nterms", C.c_uint64, C.c_void_p)
_ninfo = _f("synth_ninfo", C.c_uint32, C.c_void_p)
_docs = _f("synth_docs", C.c_void_p, C.c_void_p)
_loff = _f("synth_loff", C.c_void_p, C.c_void_p)
_terms = _f("synth_terms", C.c_void_p, C.c_void_p)
_toff = _f("synth_toff", C.c_void_p, C.c_void_p)
_codecs = _f("synth_codecs", C.c_void_p, C.c_void_p)
_info = _f("synth_info", C.c_void_p, C.c_void_p)


@dataclass
class Workload:
    docs: np.ndarray          # concatenated sorted docID lists (uint32)
    list_offsets: np.ndarray  # nlists + 1 (uint64)
    terms: np.ndarray         # concatenated query terms (uint32)
    term_offsets: np.ndarray  # nq + 1 (uint32)
    codecs: np.ndarray | None
    info: np.ndarray

    @property
    def nlists(self) -> int:
        return len(self.list_offsets) - 1

    @property
    def nq(self) -> int:
        return len(self.term_offsets) - 1

    def list(self, i: int) -> np.ndarray:
        return self.docs[self.list_offsets[i]:self.list_offsets[i + 1]]


def _arr(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    ct = {np.uint32: C.c_uint32, np.uint64: C.c_uint64, np.uint8: C.c_uint8, np.float64: C.c_double}[dtype]
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy()


def _take(h) -> Workload:
    try:
        nd, nl, nq, nt, ni = _ndocs(h), _nlists(h), _nq(h), _nterms(h), _ninfo(h)
        cod = _codecs(h)
        return Workload(_arr(_docs(h), nd, np.uint32), _arr(_loff(h), nl + 1, np.uint64),
                        _arr(_terms(h), nt, np.uint32), _arr(_toff(h), nq + 1, np.uint32),
                        _arr(cod, nl, np.uint8) if cod else None, _arr(_info(h), ni, np.float64))
    finally:
        _free(h)


def pairs(seed=0xEC1E0001, npairs=1000, short_len=4096, long_len=1 << 20, ubits=23, threads=0) -> Workload:
    """2-term queries of a short and a long uniform list (ParaPFD workload)."""
    return _take(_pairs(seed, npairs, short_len, long_len, ubits, threads))


def zipf_corpus(seed=0xEC1E0002, ndocs=10_000_000, nterms=100_000, cap=5_000_000, nq=10_000, qmin=2, qmax=5,
                threads=0) -> Workload:
    """Zipf(1) document frequencies; queries of qmin..qmax terms drawn ~ df^0.5."""
    return _take(_zipf(seed, ndocs, nterms, cap, nq, qmin, qmax, threads))


def skewed(seed=0xEC1E0003, ubits=26, npool=32, long_min=1_000_000, long_max=20_000_000, nq=5000, short_min=1000,
           short_max=10_000, run_mean=64.0, gap_mean=4096.0, threads=0) -> Workload:
    """One short clustered list per query AND 1..3 long clustered pool lists."""
    return _take(_skew(seed, ubits, npool, long_min, long_max, nq, short_min, short_max, run_mean, gap_mean, threads))


def learned(seed=0xEC1E0004, ubits=31, nclust=64, nzipf=64, lmin=10_000_000, lmax=100_000_000, zipf_s=1.2,
            zipf_cap=1 << 20, nq=20_000, kmin=1000, kmax=100_000, threads=0) -> Workload:
    """Long clustered and Zipf-gap target lists plus per-query probe-key lists."""
    return _take(_learn(seed, ubits, nclust, nzipf, lmin, lmax, zipf_s, zipf_cap, nq, kmin, kmax, threads))


def serving(seed=0xEC1E0005, ubits=28, nterms=2_000_000, total=1_000_000_000, nq=100_000, qmin=2, qmax=8,
            pfd_below=10_000, threads=0) -> Workload:
    """Zipf(1) corpus scaled to `total` postings with per-list codecs (ParaPFD / SegLRC)."""
    return _take(_serve(seed, ubits, nterms, total, nq, qmin, qmax, pfd_below, threads))


def uniform_lists(lengths, ubits=23, seed=1, threads=0) -> Workload:
    L = np.ascontiguousarray(lengths, dtype=np.uint32)
    return _take(_unif(seed, ubits, len(L), L.ctypes.data_as(u32p), threads))


def clustered_lists(lengths, ubits=26, seed=1, run_mean=64.0, gap_mean=4096.0, threads=0) -> Workload:
    L = np.ascontiguousarray(lengths, dtype=np.uint32)
    return _take(_clus(seed, ubits, len(L), L.ctypes.data_as(u32p), run_mean, gap_mean, threads))
