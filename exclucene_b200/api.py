"""ctypes binding of libexcl_gpu.so (C ABI in include/excl_gpu.h).

Mirrors the reference's entry points for this path: the ParaPFD codec calls
(encodeArray/decodeArray, Compressed/include/ParaPFor.h:15-16), the index
build of the X_Compression/X_Generator tools, and the batched conjunctive
query pipeline (CPUPreprocess -> kernels -> results, ParaPFD_Intersection.cu).
There is no CPU fallback: every call goes to the compiled library, and a
missing library raises at import time.
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libexcl_gpu.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(f"{_LIB_PATH} is not built; run `python -m exclucene_b200.build`")
_lib = C.CDLL(_LIB_PATH)

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)

OK, E_INVALID, E_CUDA, E_CAPACITY, E_FORMAT, E_TIMEOUT, E_DEVICE_FLAG, E_NOMEM = range(8)
STATUS_NAMES = ["OK", "INVALID", "CUDA", "CAPACITY", "FORMAT", "TIMEOUT", "DEVICE_FLAG", "NOMEM"]

CODEC_PARAPFD, CODEC_LRC, CODEC_LRCSEG, CODEC_SEGLRC, CODEC_HS_SEGLRC, CODEC_HS_PARAPFD, CODEC_NEWPFD = range(7)
CODEC_NAMES = {"parapfd": 0, "lrc": 1, "lrcseg": 2, "seglrc": 3, "hs_seglrc": 4, "hs_parapfd": 5, "newpfd": 6}
ALGO_AUTO, ALGO_BSEARCH, ALGO_HASHSEG, ALGO_LEARNED, ALGO_SEGREG = range(5)
ALGO_NAMES = {"auto": 0, "bsearch": 1, "hashseg": 2, "learned": 3, "segreg": 4}


class ExclError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"EXCL_E_{name}: {msg}")


class BuildParams(C.Structure):
    _fields_ = [("codec", C.c_uint32), ("codecs", C.POINTER(C.c_uint8)), ("block", C.c_uint32),
                ("frac", C.c_float), ("hs_bucket", C.c_uint32), ("hs_kbits", C.c_uint32),
                ("hs_ubits", C.c_uint32), ("threads", C.c_uint32)]


class ListInfo(C.Structure):
    _fields_ = [("word_base", C.c_uint64), ("n", C.c_uint32), ("seg_base", C.c_uint32), ("nseg", C.c_uint32),
                ("codec", C.c_uint32), ("log2_block", C.c_uint32), ("first_doc", C.c_uint32),
                ("last_doc", C.c_uint32), ("reg", C.c_uint32 * 4), ("dir_shift", C.c_uint32),
                ("dir_base", C.c_uint32), ("ndir", C.c_uint32), ("tile_base", C.c_uint32),
                ("ntiles", C.c_uint32), ("model", C.c_uint32)]


class IndexSizes(C.Structure):
    _fields_ = [("nlists", C.c_uint32), ("nsegs", C.c_uint64), ("nwords", C.c_uint64), ("ndir", C.c_uint64),
                ("ntilemap", C.c_uint64), ("postings", C.c_uint64), ("device_bytes", C.c_uint64)]


class CtxConfig(C.Structure):
    _fields_ = [("max_queries", C.c_uint32), ("max_terms", C.c_uint32), ("max_keys", C.c_uint64),
                ("warps_per_cta", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("use_graphs", C.c_uint32),
                ("merge_segs", C.c_uint32)]

MERGE_OFF = 0xFFFFFFFF


class TuneReport(C.Structure):
    _fields_ = [("algo", C.c_uint32), ("warps_per_cta", C.c_uint32), ("ctas_per_sm", C.c_uint32),
                ("merge_segs", C.c_uint32), ("best_ms", C.c_float), ("default_ms", C.c_float), ("tried", C.c_uint32),
                ("tile_split", C.c_uint32)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["algo"] = {v: k for k, v in ALGO_NAMES.items()}.get(d["algo"], d["algo"])
        return d


class BatchStats(C.Structure):
    _fields_ = [("pack_ms", C.c_float), ("probe_ms", C.c_float), ("compact_ms", C.c_float),
                ("total_ms", C.c_float), ("tiles", C.c_uint64), ("keys", C.c_uint64), ("probes", C.c_uint64),
                ("fallbacks", C.c_uint64), ("merges", C.c_uint64)]


class LearnParams(C.Structure):
    _fields_ = [("min_postings", C.c_uint32), ("nleaves", C.c_uint32), ("steps", C.c_uint32), ("batch", C.c_uint32),
                ("lr", C.c_float), ("max_window", C.c_uint32), ("seed", C.c_uint32)]


class LearnReport(C.Structure):
    _fields_ = [("models", C.c_uint32), ("train_ms", C.c_double), ("fit_ms", C.c_double), ("final_loss", C.c_float),
                ("mean_window", C.c_double), ("wide_leaf_frac", C.c_double), ("params_bytes", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_encode = _sig("excl_parapfd_encode", C.c_int, u32p, C.c_uint32, C.c_float, u32p, C.c_size_t, C.POINTER(C.c_size_t))
_decode = _sig("excl_parapfd_decode", C.c_int, u32p, C.c_size_t, C.c_uint32, u32p, C.POINTER(C.c_size_t))
_set_frac = _sig("excl_set_frac", None, C.c_float)
_nencode = _sig("excl_newpfd_encode", C.c_int, u32p, C.c_uint32, C.c_float, u32p, C.c_size_t, C.POINTER(C.c_size_t))
_ndecode = _sig("excl_newpfd_decode", C.c_int, u32p, C.c_size_t, C.c_uint32, u32p, C.POINTER(C.c_size_t))
_encodeArray = _sig("encodeArray", C.c_uint32, u32p, u32p, C.c_uint32)
_decodeArray = _sig("decodeArray", C.c_uint32, u32p, u32p, C.c_uint32)
_build = _sig("excl_index_build", C.c_int, u32p, u64p, C.c_uint32, C.POINTER(BuildParams), C.POINTER(C.c_void_p))
_ifree = _sig("excl_index_free", C.c_int, C.c_void_p)
_isizes = _sig("excl_index_sizes_get", C.c_int, C.c_void_p, C.POINTER(IndexSizes))
_iexport = _sig("excl_index_export", C.c_int, C.c_void_p, C.POINTER(ListInfo), u32p, u32p, u32p, u32p, u32p)
_ctx_create = _sig("excl_ctx_create", C.c_int, C.c_int, C.POINTER(CtxConfig), C.POINTER(C.c_void_p))
_ctx_destroy = _sig("excl_ctx_destroy", C.c_int, C.c_void_p)
_last_error = _sig("excl_last_error", C.c_char_p, C.c_void_p)
_ctx_stream = _sig("excl_ctx_stream", C.c_void_p, C.c_void_p)
_upload = _sig("excl_index_upload", C.c_int, C.c_void_p, C.c_void_p)
_dec_dev = _sig("excl_decode_lists_device", C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p)
_dec_host = _sig("excl_decode_lists", C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, u32p, C.c_size_t)
_submit = _sig("excl_submit", C.c_int, C.c_void_p, C.c_void_p, u32p, u32p, C.c_uint32, C.c_uint32,
               C.POINTER(C.c_void_p))
_wait = _sig("excl_wait", C.c_int, C.c_void_p, u32p, u32p, C.c_size_t, C.c_int, u64p)
_bfree = _sig("excl_batch_free", C.c_int, C.c_void_p)
_submit_into = _sig("excl_submit_into", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                    C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p))
_halloc = _sig("excl_host_alloc", C.c_int, C.c_size_t, C.POINTER(C.c_void_p))
_hfree = _sig("excl_host_free", C.c_int, C.c_void_p)
_isect_dev = _sig("excl_intersect_device", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                  C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64)
_check = _sig("excl_ctx_check", C.c_int, C.c_void_p)
_stats = _sig("excl_last_stats", C.c_int, C.c_void_p, C.POINTER(BatchStats))
_checksum = _sig("excl_checksum", C.c_int, C.c_uint32, u32p, u32p, C.POINTER(C.c_uint64 * 3))

_build_dev = _sig("excl_index_build_device", C.c_int, C.c_void_p, C.c_void_p, u64p, C.c_uint32, C.POINTER(BuildParams),
                  C.POINTER(C.c_void_p))
_save_ref = _sig("excl_index_save_reference", C.c_int, C.c_void_p, C.c_char_p, C.c_char_p)
_load_ref = _sig("excl_index_load_reference", C.c_int, C.c_char_p, C.c_char_p, C.c_uint32, C.POINTER(C.c_void_p))
_qparse = _sig("excl_query_parse", C.c_int, C.c_void_p, C.c_size_t, u32p, C.c_size_t, u32p, C.c_size_t,
               C.POINTER(C.c_uint32), C.POINTER(C.c_size_t))
_qencode = _sig("excl_query_encode", C.c_int, u32p, u32p, C.c_uint32, C.c_void_p, C.c_size_t,
                C.POINTER(C.c_size_t))
_autotune = _sig("excl_autotune", C.c_int, C.c_void_p, C.c_void_p, u32p, u32p, C.c_uint32, C.POINTER(TuneReport))
_set_tuning = _sig("excl_ctx_set_tuning", C.c_int, C.c_void_p, C.POINTER(TuneReport))
_set_wait_check = _sig("excl_ctx_set_wait_check", C.c_int, C.c_void_p, C.c_uint32)


class LayoutCandidate(C.Structure):
    _fields_ = [("build", BuildParams), ("best_ms", C.c_float), ("tuning", TuneReport),
                ("device_bytes", C.c_uint64), ("status", C.c_int)]


_tune_layout = _sig("excl_autotune_layout", C.c_int, C.c_void_p, C.c_void_p, u64p, C.c_uint32,
                    C.POINTER(LayoutCandidate), C.c_uint32, u32p, u32p, C.c_uint32, C.POINTER(C.c_uint32),
                    C.POINTER(C.c_void_p))
_learn = _sig("excl_learn_models", C.c_int, C.c_void_p, C.c_void_p, C.POINTER(LearnParams), C.POINTER(LearnReport))
_mexport = _sig("excl_model_export", C.c_int, C.c_void_p, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                C.POINTER(C.c_int32), C.POINTER(C.c_uint32))
_mgrad = _sig("excl_model_grad", C.c_int, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
              C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float))

_mtables = _sig("excl_model_tables", C.c_int, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint16), u32p, u32p)

EXPORTED = ["excl_learn_models", "excl_model_export", "excl_model_grad", "excl_model_tables", "excl_parapfd_encode", "excl_parapfd_decode", "excl_set_frac", "encodeArray", "decodeArray",
            "excl_index_build", "excl_index_free", "excl_index_sizes_get", "excl_index_export", "excl_ctx_create",
            "excl_ctx_destroy", "excl_last_error", "excl_ctx_stream", "excl_index_upload",
            "excl_decode_lists_device", "excl_decode_lists", "excl_submit", "excl_wait", "excl_batch_free",
            "excl_intersect_device", "excl_ctx_check", "excl_last_stats", "excl_checksum", "excl_submit_into",
            "excl_host_alloc", "excl_host_free", "excl_ctx_set_tuning", "excl_ctx_set_wait_check",
            "excl_autotune_layout"]


def _p32(a: np.ndarray):
    return a.ctypes.data_as(u32p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def pinned_empty(n: int, dtype=np.uint32) -> np.ndarray:
    """A numpy array in page-locked, device-mapped host memory (excl_host_alloc),
    freed with the array; the buffers excl_submit_into reads and writes."""
    nbytes = max(int(n), 1) * np.dtype(dtype).itemsize
    p = C.c_void_p()
    _check_status(_halloc(nbytes, C.byref(p)), what="excl_host_alloc")
    buf = (C.c_uint8 * nbytes).from_address(p.value)
    weakref.finalize(buf, _hfree, p.value)
    return np.frombuffer(buf, dtype=dtype)[: int(n)]


def _check_status(st: int, ctx=None, what: str = "") -> None:
    if st != OK:
        msg = what
        if ctx is not None and ctx._h:
            msg += ": " + _last_error(ctx._h).decode(errors="replace")
        raise ExclError(st, msg)


# ---------------------------------------------------------------------------
# Codec calls

def parapfd_encode(values, frac: float = 0.0) -> np.ndarray:
    v = _u32(values)
    cap = 3 * len(v) + 8
    out = np.zeros(cap, dtype=np.uint32)
    w = C.c_size_t(0)
    _check_status(_encode(_p32(v), len(v), frac, _p32(out), cap, C.byref(w)), what="parapfd_encode")
    return out[: w.value].copy()


def parapfd_decode(words, n: int) -> tuple[np.ndarray, int]:
    w = _u32(words)
    out = np.zeros(max(n, 1), dtype=np.uint32)
    used = C.c_size_t(0)
    _check_status(_decode(_p32(w), len(w), n, _p32(out), C.byref(used)), what="parapfd_decode")
    return out[:n], used.value


def newpfd_encode(values, frac: float = 0.0) -> np.ndarray:
    """One NewPFD block (NewPFor.cpp:52-108)."""
    v = _u32(values)
    cap = 3 * len(v) + 8
    out = np.zeros(cap, dtype=np.uint32)
    w = C.c_size_t(0)
    _check_status(_nencode(_p32(v), len(v), frac, _p32(out), cap, C.byref(w)), what="newpfd_encode")
    return out[: w.value].copy()


def newpfd_decode(words, n: int) -> tuple[np.ndarray, int]:
    w = _u32(words)
    out = np.zeros(max(n, 1), dtype=np.uint32)
    used = C.c_size_t(0)
    _check_status(_ndecode(_p32(w), len(w), n, _p32(out), C.byref(used)), what="newpfd_decode")
    return out[:n], used.value


def encode_array_compat(values, frac: float = 0.0) -> np.ndarray:
    """Reference-signature shim: encodeArray(in, out, n) with a process-wide FRAC."""
    v = _u32(values)
    out = np.zeros(3 * len(v) + 8, dtype=np.uint32)
    _set_frac(frac)
    w = _encodeArray(_p32(v), _p32(out), len(v))
    return out[:w].copy()


# ---------------------------------------------------------------------------
# Index

@dataclass
class IndexArrays:
    lists: np.ndarray      # structured view of excl_list_info
    words: np.ndarray
    seg_head: np.ndarray
    seg_rec: np.ndarray    # (nseg, 4) start, off, aux, count
    seg_reg: np.ndarray    # (nseg, 4) raw a, b, L, R
    dir: np.ndarray


class Index:
    """A built index (host image); upload it with Context.upload."""

    def __init__(self, docs, list_offsets, codec="parapfd", block: int = 256, frac: float = 0.0,
                 hs_bucket: int = 256, hs_kbits: int = 0, hs_ubits: int = 32, codecs=None, threads: int = 0):
        self._h = None
        docs = _u32(docs)
        loff = np.ascontiguousarray(list_offsets, dtype=np.uint64)
        self.nlists = len(loff) - 1
        p = BuildParams()
        p.codec = CODEC_NAMES[codec] if isinstance(codec, str) else int(codec)
        self._codecs = None
        if codecs is not None:
            self._codecs = np.ascontiguousarray(codecs, dtype=np.uint8)
            p.codecs = self._codecs.ctypes.data_as(C.POINTER(C.c_uint8))
        p.block = block
        p.frac = frac
        p.hs_bucket = hs_bucket
        p.hs_kbits = hs_kbits
        p.hs_ubits = hs_ubits
        p.threads = threads
        h = C.c_void_p()
        _check_status(_build(_p32(docs), loff.ctypes.data_as(u64p), self.nlists, C.byref(p), C.byref(h)),
                      what="excl_index_build")
        self._h = h
        self.list_lengths = np.diff(loff).astype(np.uint64)

    @classmethod
    def from_handle(cls, h: C.c_void_p, nlists: int, lengths) -> "Index":
        self = cls.__new__(cls)
        self._h = h
        self.nlists = nlists
        self._codecs = None
        self.list_lengths = np.asarray(lengths, dtype=np.uint64)
        return self

    def save_reference(self, directory: str, name: str) -> None:
        """Write the reference's file set (ParaPFD or SegLRC, 256-entry segments)."""
        _check_status(_save_ref(self._h, directory.encode(), name.encode()), what="excl_index_save_reference")

    @classmethod
    def load_reference(cls, directory: str, name: str, codec="parapfd") -> "Index":
        """Load a reference file set (ParaPFD or SegLRC) without re-encoding."""
        c = CODEC_NAMES[codec] if isinstance(codec, str) else int(codec)
        h = C.c_void_p()
        _check_status(_load_ref(directory.encode(), name.encode(), c, C.byref(h)), what="excl_index_load_reference")
        s = IndexSizes()
        _check_status(_isizes(h, C.byref(s)))
        lists = (ListInfo * s.nlists)()
        _check_status(_iexport(h, lists, None, None, None, None, None))
        return cls.from_handle(h, s.nlists, [lists[i].n for i in range(s.nlists)])

    def sizes(self) -> IndexSizes:
        s = IndexSizes()
        _check_status(_isizes(self._h, C.byref(s)))
        return s

    def export(self) -> IndexArrays:
        s = self.sizes()
        lists = (ListInfo * s.nlists)()
        words = np.zeros(s.nwords, dtype=np.uint32)
        head = np.zeros(s.nsegs, dtype=np.uint32)
        rec = np.zeros((s.nsegs, 4), dtype=np.uint32)
        reg = np.zeros((s.nsegs, 4), dtype=np.uint32)
        d = np.zeros(max(s.ndir, 1), dtype=np.uint32)
        _check_status(_iexport(self._h, lists, _p32(words), _p32(head), _p32(rec), _p32(reg), _p32(d)))
        arr = np.ctypeslib.as_array(lists).copy() if s.nlists else np.zeros(0)
        return IndexArrays(arr, words, head, rec, reg, d[: s.ndir])

    def model(self, list_id: int):
        """(root params[1153], header {kmin, kscale, nleaves, max_window}, leaves[L, 4] as int32 words) or None."""
        L = C.c_uint32(0)
        hdr = np.zeros(4, dtype=np.float32)
        if _mexport(self._h, list_id, None, hdr.ctypes.data_as(C.POINTER(C.c_float)), None, C.byref(L)) != OK:
            return None
        root = np.zeros(1153, dtype=np.float32)
        leaves = np.zeros((L.value, 4), dtype=np.int32)
        _check_status(_mexport(self._h, list_id, root.ctypes.data_as(C.POINTER(C.c_float)),
                               hdr.ctypes.data_as(C.POINTER(C.c_float)), leaves.ctypes.data_as(C.POINTER(C.c_int32)),
                               C.byref(L)))
        return root, hdr, leaves

    def model_tables(self, list_id: int):
        """(grid[grid_n+1] uint16, bnd[nleaves] uint32, first, grid_shift) of a list's stored routing, or None."""
        meta = np.zeros(4, dtype=np.uint32)
        if _mtables(self._h, list_id, None, None, _p32(meta)) != OK:
            return None
        grid = np.zeros(int(meta[2]) + 1, dtype=np.uint16)
        bnd = np.zeros(int(meta[3]), dtype=np.uint32)
        _check_status(_mtables(self._h, list_id, grid.ctypes.data_as(C.POINTER(C.c_uint16)), _p32(bnd), _p32(meta)))
        return grid, bnd, int(meta[0]), int(meta[1])

    def close(self) -> None:
        if self._h:
            _ifree(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Context

class Context:
    def __init__(self, device: int = 0, max_queries: int = 65536, max_keys: int = 1 << 26, warps_per_cta: int = 0,
                 ctas_per_sm: int = 0, use_graphs: bool = False, merge_segs: int = 0):
        self._h = None
        cfg = CtxConfig(max_queries, 32, max_keys, warps_per_cta, ctas_per_sm, 1 if use_graphs else 0, merge_segs)
        h = C.c_void_p()
        st = _ctx_create(device, C.byref(cfg), C.byref(h))
        _check_status(st, what="excl_ctx_create")
        self._h = h
        self.device = device

    @property
    def stream(self) -> int:
        return _ctx_stream(self._h) or 0

    def last_error(self) -> str:
        return _last_error(self._h).decode(errors="replace")

    def upload(self, ix: Index) -> None:
        _check_status(_upload(self._h, ix._h), self, "excl_index_upload")

    def decode_lists(self, ix: Index, l0: int = 0, l1: int | None = None) -> np.ndarray:
        l1 = ix.nlists if l1 is None else l1
        n = int(ix.list_lengths[l0:l1].sum())
        out = np.zeros(max(n, 1), dtype=np.uint32)
        _check_status(_dec_host(self._h, ix._h, l0, l1, _p32(out), n), self, "excl_decode_lists")
        return out[:n]

    def decode_lists_device(self, ix: Index, l0: int, l1: int, d_out_ptr: int) -> None:
        _check_status(_dec_dev(self._h, ix._h, l0, l1, C.c_void_p(d_out_ptr)), self, "excl_decode_lists_device")

    def submit(self, ix: Index, terms, term_offsets, algo="auto"):
        t = _u32(terms)
        o = _u32(term_offsets)
        nq = len(o) - 1
        a = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
        b = C.c_void_p()
        if len(t) == 0:
            t = np.zeros(1, dtype=np.uint32)
        _check_status(_submit(self._h, ix._h, _p32(t), _p32(o), nq, a, C.byref(b)), self, "excl_submit")
        return Batch(self, b, nq)

    def submit_into(self, ix: Index, terms: np.ndarray, term_offsets: np.ndarray, offsets: np.ndarray,
                    docids: np.ndarray, algo="auto") -> "Batch":
        """Zero-copy batch (excl_submit_into): offsets[nq+1] and docids are pinned_empty
        arrays the batch kernel writes into; terms and term_offsets are read from host
        memory (pinned_empty ones asynchronously). Keep all four alive and unchanged
        until wait() returns the number of docIDs written."""
        for a in (terms, term_offsets, offsets, docids):
            if a.dtype != np.uint32 or not a.flags.c_contiguous:
                raise ExclError(E_INVALID, "excl_submit_into: arrays must be contiguous uint32")
        nq = len(term_offsets) - 1
        if len(offsets) < nq + 1:
            raise ExclError(E_INVALID, "excl_submit_into: offsets holds fewer than nq+1 entries")
        a = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
        b = C.c_void_p()
        st = _submit_into(self._h, ix._h, terms.ctypes.data, term_offsets.ctypes.data, nq, a, offsets.ctypes.data,
                          docids.ctypes.data, len(docids), C.byref(b))
        if st != OK:
            _check_status(st, self, "excl_submit_into")
        return Batch(self, b, nq, into=(terms, term_offsets, offsets, docids))

    def intersect(self, ix: Index, terms, term_offsets, algo="auto") -> tuple[np.ndarray, np.ndarray]:
        """Runs one batch and returns (offsets[nq+1], docids) — each query's docIDs sorted."""
        b = self.submit(ix, terms, term_offsets, algo)
        try:
            return b.wait()
        finally:
            b.free()

    def intersect_device(self, ix: Index, d_terms: int, d_toff: int, nq: int, algo, d_offsets: int, d_docids: int,
                         cap: int) -> None:
        a = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
        _check_status(_isect_dev(self._h, ix._h, C.c_void_p(d_terms), C.c_void_p(d_toff), nq, a,
                                 C.c_void_p(d_offsets), C.c_void_p(d_docids), cap), self, "excl_intersect_device")

    def check(self) -> None:
        _check_status(_check(self._h), self, "excl_ctx_check")

    def learn(self, ix: Index, min_postings: int = 1 << 20, nleaves: int = 4096, steps: int = 300,
              batch: int = 16384, lr: float = 3e-3, max_window: int = 4096, seed: int = 1) -> dict:
        """Trains the learned position models of the index's long lists on this device."""
        p = LearnParams(min_postings, nleaves, steps, batch, lr, max_window, seed)
        r = LearnReport()
        _check_status(_learn(self._h, ix._h, C.byref(p), C.byref(r)), self, "excl_learn_models")
        return r.as_dict()

    def model_grad(self, params, x, y) -> tuple[np.ndarray, float]:
        """Gradient of the training kernels for given samples (for checks)."""
        fp = C.POINTER(C.c_float)
        P = np.ascontiguousarray(params, dtype=np.float32)
        xs = np.ascontiguousarray(x, dtype=np.float32)
        ys = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(1153, dtype=np.float32)
        loss = C.c_float(0)
        _check_status(_mgrad(self._h, P.ctypes.data_as(fp), xs.ctypes.data_as(fp), ys.ctypes.data_as(fp), len(xs),
                             g.ctypes.data_as(fp), C.byref(loss)), self, "excl_model_grad")
        return g, loss.value

    def build_index(self, d_docs: int, list_offsets, codec="seglrc", block: int = 256, frac: float = 0.0,
                    hs_bucket: int = 256, hs_kbits: int = 0, hs_ubits: int = 32) -> Index:
        """Build an index (ParaPFD, NewPFD, LRC, LRCSeg, SegLRC, HS_SegLRC or HS_ParaPFD)
        on this context's GPU from a device docID array (pointer; list l =
        d_docs[list_offsets[l] .. list_offsets[l+1])). Byte-identical to
        Index(docs, list_offsets, ...) with the same parameters; upload it before use."""
        loff = np.ascontiguousarray(list_offsets, dtype=np.uint64)
        p = BuildParams()
        p.codec = CODEC_NAMES[codec] if isinstance(codec, str) else int(codec)
        p.block = block
        p.frac = frac
        p.hs_bucket = hs_bucket
        p.hs_kbits = hs_kbits
        p.hs_ubits = hs_ubits
        h = C.c_void_p()
        _check_status(_build_dev(self._h, C.c_void_p(d_docs), loff.ctypes.data_as(u64p), len(loff) - 1, C.byref(p),
                                 C.byref(h)), self, "excl_index_build_device")
        return Index.from_handle(h, len(loff) - 1, np.diff(loff))

    def autotune_layout(self, d_docs: int, list_offsets, candidates, terms, term_offsets):
        """excl_autotune_layout: builds the corpus (device docID array d_docs,
        CSR list_offsets) on the GPU under each candidate layout (dicts with
        build_index's keywords: codec, block, frac, hs_bucket, hs_kbits,
        hs_ubits), tunes and times the sample batch on each, and keeps the
        fastest. Returns (index of the chosen layout, uploaded; its position in
        `candidates`; one dict per candidate with its time, size, tuning and
        status)."""
        loff = np.ascontiguousarray(list_offsets, dtype=np.uint64)
        arr = (LayoutCandidate * len(candidates))()
        for c, kw in zip(arr, candidates):
            c.build.codec = CODEC_NAMES[kw.get("codec", "seglrc")]
            c.build.block = kw.get("block", 256)
            c.build.frac = kw.get("frac", 0.0)
            c.build.hs_bucket = kw.get("hs_bucket", 256)
            c.build.hs_kbits = kw.get("hs_kbits", 0)
            c.build.hs_ubits = kw.get("hs_ubits", 32)
        t = _u32(terms) if len(terms) else np.zeros(1, dtype=np.uint32)
        o = _u32(term_offsets)
        best = C.c_uint32(0)
        h = C.c_void_p()
        _check_status(_tune_layout(self._h, C.c_void_p(d_docs), loff.ctypes.data_as(u64p), len(loff) - 1, arr,
                                   len(candidates), _p32(t), _p32(o), len(o) - 1, C.byref(best), C.byref(h)),
                      self, "excl_autotune_layout")
        report = [dict(kw, best_ms=c.best_ms, device_bytes=int(c.device_bytes), status=int(c.status),
                       tuning=c.tuning.as_dict() if c.status == OK else None) for c, kw in zip(arr, candidates)]
        return Index.from_handle(h, len(loff) - 1, np.diff(loff)), int(best.value), report

    def set_wait_check(self, polls: int) -> None:
        """excl_ctx_set_wait_check: polls > 0 makes every later batch run one
        bounded device wait that gives up (the device failure path); 0 stops it."""
        _check_status(_set_wait_check(self._h, int(polls)), self, "excl_ctx_set_wait_check")

    def set_tuning(self, algo="auto", warps_per_cta: int = 8, ctas_per_sm: int = 5, merge_segs: int = 2,
                   tile_split: int = 0, **_ignored) -> None:
        """Apply a launch setting (e.g. the dict autotune returned) without timing."""
        r = TuneReport()
        r.algo = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
        r.warps_per_cta, r.ctas_per_sm, r.tile_split = warps_per_cta, ctas_per_sm, tile_split
        r.merge_segs = MERGE_OFF if merge_segs in (0, MERGE_OFF) else merge_segs
        _check_status(_set_tuning(self._h, C.byref(r)), self, "excl_ctx_set_tuning")

    def autotune(self, ix: Index, terms, term_offsets) -> dict:
        """Times the sample batch under every candidate setting and keeps the
        fastest for later batches run with algo="auto"."""
        t = _u32(terms) if len(terms) else np.zeros(1, dtype=np.uint32)
        o = _u32(term_offsets)
        r = TuneReport()
        _check_status(_autotune(self._h, ix._h, _p32(t), _p32(o), len(o) - 1, C.byref(r)), self, "excl_autotune")
        return r.as_dict()

    def stats(self) -> BatchStats:
        s = BatchStats()
        _check_status(_stats(self._h, C.byref(s)), self, "excl_last_stats")
        return s

    def close(self) -> None:
        if self._h:
            _ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    def __init__(self, ctx: Context, h: C.c_void_p, nq: int, into=None):
        self.ctx, self._h, self.nq = ctx, h, nq
        self._into = into  # the arrays of an excl_submit_into batch, kept alive until it is freed

    def wait(self, timeout_ms: int = -1):
        """(offsets, docids) of an excl_submit batch; the number of docIDs written
        for an excl_submit_into one."""
        if self._into is not None:
            tot = C.c_uint64(0)
            _check_status(_wait(self._h, None, None, 0, timeout_ms, C.byref(tot)), self.ctx, "excl_wait")
            return int(tot.value)
        offs = np.zeros(self.nq + 1, dtype=np.uint32)
        tot = C.c_uint64(0)
        _check_status(_wait(self._h, _p32(offs), None, 0, timeout_ms, C.byref(tot)), self.ctx, "excl_wait")
        docs = np.zeros(max(int(tot.value), 1), dtype=np.uint32)
        _check_status(_wait(self._h, _p32(offs), _p32(docs), len(docs), timeout_ms, C.byref(tot)), self.ctx,
                      "excl_wait")
        return offs, docs[: int(tot.value)]

    def wait_into(self, offsets: np.ndarray, docids: np.ndarray, timeout_ms: int = -1) -> int:
        tot = C.c_uint64(0)
        _check_status(_wait(self._h, _p32(offsets), _p32(docids), len(docids), timeout_ms, C.byref(tot)),
                      self.ctx, "excl_wait")
        return int(tot.value)

    def free(self) -> None:
        if self._h:
            _bfree(self._h)
            self._h = None


def checksum(offsets, docids) -> tuple[int, int, int]:
    o = _u32(offsets)
    d = _u32(docids) if len(docids) else np.zeros(1, dtype=np.uint32)
    cs = (C.c_uint64 * 3)()
    _check_status(_checksum(len(o) - 1, _p32(o), _p32(d), C.byref(cs)))
    return int(cs[0]), int(cs[1]), int(cs[2])


def query_parse(data: bytes) -> tuple[np.ndarray, np.ndarray]:
    """A reference .query stream -> (terms, term_offsets)."""
    buf = C.create_string_buffer(bytes(data), len(data))
    nq, nt = C.c_uint32(), C.c_size_t()
    _check_status(_qparse(buf, len(data), None, 0, None, 0, C.byref(nq), C.byref(nt)), what="excl_query_parse")
    terms = np.zeros(max(nt.value, 1), np.uint32)
    toff = np.zeros(nq.value + 1, np.uint32)
    _check_status(_qparse(buf, len(data), _p32(terms), nt.value, _p32(toff), nq.value + 1, C.byref(nq),
                          C.byref(nt)), what="excl_query_parse")
    return terms[:nt.value], toff


def query_encode(terms, term_offsets) -> bytes:
    """(terms, term_offsets) -> a reference .query stream."""
    t = _u32(terms) if len(terms) else np.zeros(1, np.uint32)
    o = _u32(term_offsets)
    nb = C.c_size_t()
    _check_status(_qencode(_p32(t), _p32(o), len(o) - 1, None, 0, C.byref(nb)))
    buf = C.create_string_buffer(max(nb.value, 1))
    _check_status(_qencode(_p32(t), _p32(o), len(o) - 1, buf, nb.value, C.byref(nb)))
    return buf.raw[:nb.value]


def library_path() -> str:
    return _LIB_PATH


# ---------------------------------------------------------------------------
# Allocation-free form of Context.intersect_device, for callers that cannot
# allocate device memory when they query (their budget is fixed at start-up,
# or they run without a Context, whose creation allocates the batch buffers).
# Its scratch is a fixed 5.6 MiB device array inside the library, shared by
# all calls: calls that overlap on the GPU race. The first call on a device
# looks the array up; make it before any stream capture.

NOALLOC_MAX_QUERIES = 4096
NOALLOC_MAX_KEYS = 1 << 20
_isect_noalloc = _sig("excl_intersect_device_noalloc", C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                      C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p)


def intersect_device_noalloc(ix: Index, d_terms: int, d_toff: int, nq: int, algo, d_offsets: int, d_docids: int,
                             cap: int, stream: int) -> None:
    """Runs one batch on `stream` (device pointers in and out) and returns when it is done."""
    a = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
    _check_status(_isect_noalloc(ix._h, C.c_void_p(d_terms), C.c_void_p(d_toff), nq, a, C.c_void_p(d_offsets),
                                 C.c_void_p(d_docids), cap, C.c_void_p(stream)), what="excl_intersect_device_noalloc")


# ---------------------------------------------------------------------------
# Serving loop: continuous batching of single queries on a resident index.

class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("max_batch_queries", C.c_uint32), ("max_batch_keys", C.c_uint64),
                ("hbm_budget_bytes", C.c_uint64), ("algo", C.c_uint32), ("warps_per_cta", C.c_uint32),
                ("ctas_per_sm", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("rejected", C.c_uint64), ("mean_batch", C.c_double), ("pool_bytes", C.c_uint64),
                ("pool_peak_bytes", C.c_uint64), ("max_inflight", C.c_uint32), ("p50_us", C.c_double),
                ("p99_us", C.c_double), ("max_us", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_srv_create = _sig("excl_server_create", C.c_int, C.c_int, C.c_void_p, C.POINTER(ServerConfig),
                   C.POINTER(C.c_void_p))
_srv_destroy = _sig("excl_server_destroy", C.c_int, C.c_void_p)
_srv_submit = _sig("excl_server_submit", C.c_int, C.c_void_p, u32p, C.c_uint32, C.POINTER(C.c_uint64))
_srv_wait = _sig("excl_server_wait", C.c_int, C.c_void_p, C.c_uint64, u32p, C.c_size_t, C.POINTER(C.c_uint32),
                 C.c_int)
_srv_stats = _sig("excl_server_stats_get", C.c_int, C.c_void_p, C.POINTER(ServerStats))
_srv_reset = _sig("excl_server_stats_reset", C.c_int, C.c_void_p)
_srv_replay = _sig("excl_server_replay", C.c_int, C.c_void_p, u32p, u32p, C.c_uint32, C.POINTER(C.c_double),
                   C.POINTER(C.c_double), C.POINTER(C.c_uint64 * 3), C.POINTER(C.c_double))
EXPORTED += ["excl_newpfd_encode", "excl_newpfd_decode", "excl_index_build_device", "excl_index_save_reference", "excl_index_load_reference", "excl_query_parse", "excl_query_encode",
             "excl_autotune", "excl_server_create", "excl_server_destroy", "excl_server_submit", "excl_server_wait",
             "excl_server_stats_get", "excl_server_stats_reset", "excl_server_replay",
             "excl_intersect_device_noalloc"]


class Server:
    """Continuous-batching server over an index uploaded to `device`."""

    def __init__(self, ix: Index, device: int = 0, slots: int = 4, max_batch_queries: int = 4096,
                 max_batch_keys: int = 1 << 22, hbm_budget_bytes: int = 0, algo="auto", warps_per_cta: int = 0,
                 ctas_per_sm: int = 0):
        self._h = None
        self._ix = ix  # the server reads the index; keep it alive
        a = ALGO_NAMES[algo] if isinstance(algo, str) else int(algo)
        cfg = ServerConfig(slots, max_batch_queries, max_batch_keys, hbm_budget_bytes, a, warps_per_cta, ctas_per_sm)
        h = C.c_void_p()
        _check_status(_srv_create(device, ix._h, C.byref(cfg), C.byref(h)), what="excl_server_create")
        self._h = h

    def submit(self, terms) -> int:
        t = _u32(terms) if len(terms) else np.zeros(1, dtype=np.uint32)
        tk = C.c_uint64()
        _check_status(_srv_submit(self._h, _p32(t), len(terms), C.byref(tk)), what="excl_server_submit")
        return int(tk.value)

    def wait(self, ticket: int, cap: int = 1 << 20, timeout_ms: int = -1) -> np.ndarray:
        out = np.zeros(max(cap, 1), dtype=np.uint32)
        n = C.c_uint32()
        _check_status(_srv_wait(self._h, ticket, _p32(out), cap, C.byref(n), timeout_ms), what="excl_server_wait")
        return out[: n.value].copy()

    def stats(self) -> dict:
        st = ServerStats()
        _check_status(_srv_stats(self._h, C.byref(st)))
        return st.as_dict()

    def reset_stats(self) -> None:
        _check_status(_srv_reset(self._h))

    def replay(self, terms, term_offsets, arrival_s) -> tuple[np.ndarray, tuple[int, int, int], float]:
        """Open-loop load: query q is submitted arrival_s[q] s after the start.
        Returns per-query latencies (s), the checksum triple and the wall time."""
        t = _u32(terms) if len(terms) else np.zeros(1, dtype=np.uint32)
        o = _u32(term_offsets)
        nq = len(o) - 1
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        lat = np.zeros(max(nq, 1), dtype=np.float64)
        cs = (C.c_uint64 * 3)()
        wall = C.c_double()
        dp = C.POINTER(C.c_double)
        _check_status(_srv_replay(self._h, _p32(t), _p32(o), nq, arr.ctypes.data_as(dp), lat.ctypes.data_as(dp),
                                  C.byref(cs), C.byref(wall)), what="excl_server_replay")
        return lat[:nq], (int(cs[0]), int(cs[1]), int(cs[2])), float(wall.value)

    def close(self) -> None:
        if self._h:
            _srv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
