"""exclucene_b200 — B200 (sm_100a) batched decode + AND intersection of
compressed posting lists in ExCLucene's ParaPFD, LRC, LRCSeg, SegLRC and
hash-segmentation formats.

The work happens in libexcl_gpu.so (C ABI: include/excl_gpu.h); this package
is its ctypes binding. Before the library is built only the build module
(`python -m exclucene_b200.build`) is usable: any other name of the package
raises ImportError, so no call can silently fall back to the CPU.
"""
import os as _os

_LIB = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "libexcl_gpu.so")

__all__ = ["Context", "Index", "Batch", "Server", "query_parse", "query_encode", "ExclError", "checksum", "parapfd_encode", "parapfd_decode",
           "encode_array_compat", "library_path", "CODEC_PARAPFD", "CODEC_LRC", "CODEC_LRCSEG", "CODEC_SEGLRC",
           "CODEC_HS_SEGLRC", "CODEC_HS_PARAPFD", "CODEC_NEWPFD", "newpfd_encode", "newpfd_decode", "ALGO_AUTO", "ALGO_BSEARCH", "ALGO_HASHSEG", "ALGO_LEARNED",
           "ALGO_SEGREG", "pinned_empty"]

_API_NAMES = set(__all__)


def __getattr__(name):
    # the binding is loaded on first use, so the build module imports (and can
    # rebuild) even when the library is missing or older than the binding
    if name in _API_NAMES or name == "api":
        if not _os.path.exists(_LIB):
            raise ImportError(f"{_LIB} is not built; run `python -m exclucene_b200.build`")
        import importlib

        api = importlib.import_module(__name__ + ".api")
        return api if name == "api" else getattr(api, name)
    raise AttributeError(name)
