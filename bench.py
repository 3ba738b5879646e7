"""Benchmark of the batched decode + AND-intersection path on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--workload zipf|pairs|skewed|learned|serving] [--scale S]

One step = one batch of the workload's queries through the device pipeline
(one persistent kernel: pack -> probe -> scatter), with the compressed index
resident in HBM. Prints ONE JSON line on rank 0.

Workloads (seeded synthetic stand-ins for the reference's Baidu/GOV2 data):
  zipf     10M docs, 100k terms, df_r = min(5M, 5M/r) (~60.4M postings), SegLRC
           (256-entry segments, FRAC 0), 10,000 queries of 2-5 terms ~ df^0.5
  pairs    1,000 pairs of 4,096 / 1,048,576 uniform docIDs over 2^23, ParaPFD
           blocks of 128, FRAC 0.10
  skewed   2^26 universe, clustered-run lists, HS-bucketed ParaPFD, 5,000 queries
  learned  64 clustered + 64 Zipf-gap long lists, 20,000 probe-key lists
  serving  1e9 postings over 2M terms, ParaPFD / SegLRC by length, 100,000 queries

Parity: the CPU oracle (oracle/, test infrastructure) is the checker. Before
any timing it computes the exact AND of the batch; after each timed region the
last result of that configuration is compared with it query by query, and the
line's "parity" object reports the mismatches (the run exits 1 on any). The
oracle also supplies the CPU baseline legs; it is never inside a timed GPU
region. --impl reference runs only the oracle's CPU path, on inputs made by
the oracle's own restatement of the workload generators and encoders, so that
arm loads no library of the package.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# dram__bytes_read.sum + dram__bytes_write.sum of one k_batch launch on the full-size workload,
# from one ncu capture (profiles/k_batch_zipf_seglrc.md: 45.47 MB read + 0.30 MB written)
NCU_BATCH_TRAFFIC: dict = {"zipf": 45_472_768 + 302_080}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="zipf", choices=["zipf", "pairs", "skewed", "learned", "serving"])
    p.add_argument("--codec", default=None)
    p.add_argument("--algo", default=None, help="search method for `value` (default: best measured)")
    p.add_argument("--cpu-sample-s", type=float, default=15.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--scale", type=float, default=1.0, help="workload size factor (1.0 = the named config)")
    p.add_argument("--learn-min", type=int, default=None,
                   help="lists with at least this many postings get a learned model (default per workload)")
    p.add_argument("--no-learn", action="store_true")
    p.add_argument("--no-serve", action="store_true", help="skip the serving-loop latency measurement")
    p.add_argument("--no-layout-tune", action="store_true", help="skip the index-layout autotuner")
    p.add_argument("--ctas-per-sm", type=int, default=0,
                   help="with --algo: batch kernel CTAs per SM (4, 5 or 6) instead of the default launch shape")
    return p.parse_args()


# ---------------------------------------------------------------------------
# workloads

def make_workload(name: str, scale: float, gen=None, nq_factor: int = 1):
    """The named workload at `scale`. `gen` supplies the generators: the
    package's (GPU arm) or the oracle's restatement of the same seeded
    generators (CPU reference arm, which loads no product code); both give the
    same lists and queries bit for bit. `nq_factor` > 1 draws that many times
    the queries from the same stream for the query-stream workloads (zipf,
    serving: one batch per rank under --gpus N, the first being the
    single-GPU batch); the list-per-query workloads ignore it (every rank runs
    the same batch, so no rank holds other ranks' lists)."""
    if gen is None:
        from exclucene_b200 import synth as gen
    synth = gen
    if name == "zipf":
        nt = max(1000, int(100_000 * scale))
        w = synth.zipf_corpus(ndocs=int(10_000_000 * max(scale, 0.01)), nterms=nt, cap=int(5_000_000 * scale),
                              nq=max(100, int(10_000 * scale)) * nq_factor, qmin=2, qmax=5)
        return w, dict(codec="seglrc", block=256, frac=0.0), (
            f"zipf corpus: {int(10_000_000 * max(scale, 0.01))} docs, {nt} terms, df_r=min(cap,cap/r), "
            f"{w.nq // nq_factor} queries of 2-5 terms ~ df^0.5; SegLRC 256-entry segments, FRAC 0")
    if name == "pairs":
        npairs = max(10, int(1000 * scale))
        w = synth.pairs(npairs=npairs)
        return w, dict(codec="parapfd", block=128, frac=0.10), (
            f"{npairs} pairs of 4096/1048576 uniform docIDs over 2^23; ParaPFD blocks of 128, FRAC 0.10")
    if name == "skewed":
        nq = max(100, int(5000 * scale))
        w = synth.skewed(nq=nq, npool=32)
        return w, dict(codec="hs_parapfd", block=128, frac=0.10, hs_kbits=16, hs_ubits=26), (
            f"2^26 universe, 32 clustered long lists 1e6-2e7, {nq} short lists 1e3-1e4, 1-3 long per query; "
            "HS top-16-bit buckets, ParaPFD blocks of 128, FRAC 0.10")
    if name == "learned":
        nq = max(100, int(20_000 * scale))
        lmin, lmax = int(10_000_000 * scale), int(100_000_000 * scale)
        w = synth.learned(lmin=lmin, lmax=lmax, nq=nq)
        return w, dict(codec="seglrc", block=256, frac=0.0), (
            f"learned vs plain: 64 clustered-run lists of log-U[{lmin:.0e}, {lmax:.0e}] and 64 Zipf(1.2)-gap "
            f"lists over 2^31; {nq} queries, each a probe-key list of log-U[1e3, 1e5] keys (half from the "
            "target list) AND its target; SegLRC 256-entry segments, FRAC 0")
    if name == "serving":
        total, nterms = int(1_000_000_000 * scale), max(1000, int(2_000_000 * scale))
        nq = max(1000, int(100_000 * min(scale * 10, 1.0)))
        w = synth.serving(total=total, nterms=nterms, nq=nq * nq_factor)
        return w, dict(codec="seglrc", block=256, frac=0.0, codecs=w.codecs), (
            f"serving corpus: {total:.2e} postings over {nterms} terms (Zipf(1) dfs, 2^28 universe), ParaPFD "
            f"below 1e4 postings else SegLRC; {nq} queries of 2-8 terms ~ df^0.5")
    raise ValueError(name)


# Candidate index layouts for the layout autotuner, per workload: the skewed
# workload's HS top-k bits (8..16), the Zipf corpus's codec and block size.
LAYOUT_CANDIDATES = {
    "skewed": lambda p: [dict(p, hs_kbits=k) for k in (8, 10, 12, 14, 16)],
    "zipf": lambda p: [dict(codec=c, block=b, frac=p["frac"]) for c in ("seglrc", "parapfd") for b in (256, 128)],
}


def query_postings(w) -> int:
    lens = np.diff(w.list_offsets).astype(np.int64)
    return int(lens[w.terms.astype(np.int64)].sum())


def batch_bytes(w, tiles: int, results: int) -> int:
    """Bookkeeping bytes of one batch beside the probe's (algorithmic_bytes):
    the pack phase reads the query offsets and terms and three fields of each
    term's list descriptor and writes the sorted terms, per-query counts and
    prefixes and a 16-byte work record per tile; the probe phase reads each
    tile's record, query row and prefixes and writes its count and slot and
    the survivors; the scatter phase reads tile counts and slots, writes and
    reads tile positions, moves the survivors and writes the offsets."""
    nq, nterms = w.nq, len(w.terms)
    pack = 4 * (nq + 1) + 4 * nterms + 12 * nterms + 4 * nterms + 4 * nq + 8 * (nq + 2) + 16 * tiles
    probe = tiles * (16 + 4 + 4 + 8) + 4 * nterms + 4 * results
    scatter = tiles * (8 + 4 + 4) + 4 * results + 4 * (nq + 1)
    return pack + probe + scatter


def algorithmic_bytes(w, arrays) -> int:
    """Bytes one step must move at minimum (per query: the shortest list's
    compressed bytes + for each longer list min(whole list, blocks hit by the
    surviving probes + their metadata) + 4 bytes per result)."""
    lists = arrays.lists
    nseg_all = len(arrays.seg_head)
    seg_rec = arrays.seg_rec
    # words per segment: blocks are stored list after list, segment after segment
    nseg = lists["nseg"].astype(np.int64)
    seg_of_list = np.repeat(np.arange(len(lists)), nseg)
    gstart = lists["word_base"].astype(np.int64)[seg_of_list] + seg_rec[:nseg_all, 1].astype(np.int64)
    seg_words = np.diff(np.append(gstart, len(arrays.words) - 8))
    codec_meta = {0: 12, 1: 8, 2: 12, 3: 28, 4: 28, 5: 12, 6: 12}
    total = 0
    lens = np.diff(w.list_offsets).astype(np.int64)
    for q in range(w.nq):
        ts = w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]
        if len(ts) == 0:
            continue
        order = sorted(ts.tolist(), key=lambda t: lens[t])
        meta = codec_meta[int(lists[order[0]]["codec"])]
        s0, ns = int(lists[order[0]]["seg_base"]), int(lists[order[0]]["nseg"])
        total += 4 * int(seg_words[s0:s0 + ns].sum()) + meta * ns
        keys = w.list(order[0])
        for t in order[1:]:
            if len(keys) == 0:
                break
            li = lists[t]
            s0, ns = int(li["seg_base"]), int(li["nseg"])
            meta = codec_meta[int(li["codec"])]
            heads = arrays.seg_head[s0:s0 + ns]
            segs = np.unique(np.clip(np.searchsorted(heads, keys, side="right") - 1, 0, ns - 1))
            hit = 4 * int(seg_words[s0 + segs].sum()) + meta * len(segs)
            whole = 4 * int(seg_words[s0:s0 + ns].sum()) + meta * ns
            total += min(hit, whole)
            lst = w.list(t)
            pos = np.minimum(np.searchsorted(lst, keys), len(lst) - 1)
            keys = keys[lst[pos] == keys]
        total += 4 * len(keys)
    return total


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and
                          s[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def flush_l2(buf):
    """Evict L2 (126 MB) by reading a 512 MB buffer: the cache ends up holding
    clean lines, so the next timed kernel pays no write-back for the flush."""
    buf.sum(dtype=__import__("torch").int64)


def peak_hbm():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# CPU legs (oracle restatement of the reference path, all host threads)

def cpu_run(w, img, seconds: float, threads: int):
    """The reference's CPU work on the same compressed index (decode with the
    ParaPFD/regression arithmetic + exact AND), over a bounded sample: whole
    batches repeated, or a prefix of the queries, for about `seconds`."""
    import oracle

    lens = np.diff(w.list_offsets).astype(np.int64)
    nq = w.nq
    n = max(1, min(nq, 256))
    while True:
        t, _ = oracle.run_queries_compressed(img, w.terms[:int(w.term_offsets[n])], w.term_offsets[:n + 1],
                                             threads)
        if t >= seconds or n >= nq:
            break
        n = min(nq, max(n * 2, int(n * seconds / max(t, 1e-3) * 0.9)))
    postings = int(lens[w.terms[:int(w.term_offsets[n])].astype(np.int64)].sum())
    reps = 1
    if n >= nq and t < seconds:
        reps = int(min(1000, np.ceil(seconds / max(t, 1e-6))))
        t = 0.0
        for _ in range(reps):
            dt, _ = oracle.run_queries_compressed(img, w.terms, w.term_offsets, threads)
            t += dt
    return t, n, postings * reps, reps


def bench_config(w, params, desc) -> dict:
    """The `config` object of both arms' JSON lines (identical for the same
    workload): what one step processes, nothing about how."""
    lens = np.diff(w.list_offsets).astype(np.int64)
    return {"workload": desc, "codec": params["codec"] if "codecs" not in params else "parapfd+seglrc",
            "block": params["block"], "frac": params["frac"], "queries_per_step": int(w.nq),
            "postings_per_step": int(lens[w.terms.astype(np.int64)].sum()),
            "l2": "GPU arm: flushed (512 MB read on the batch's stream) before each timed step; CPU arm: n/a"}


def reference_arm(args, w, desc, params):
    """The reference's CPU path (oracle port: ParaPFD/regression block decode +
    exact AND) on the box's host cores. Its inputs come from the oracle's
    restatement of the workload generators and its compressed index from the
    oracle's block encoders (byte-pinned to the reference codec), so this arm
    loads no library of the package under test."""
    import oracle

    threads = os.cpu_count() or 1
    codecs = params.get("codecs")
    img = oracle.encode_corpus(w.docs, w.list_offsets,
                               codecs if codecs is not None else oracle.CODECS[params["codec"]],
                               block=params["block"], frac=params["frac"], bucket=params.get("hs_bucket", 256),
                               kbits=params.get("hs_kbits", 0), ubits=params.get("hs_ubits", 32))
    vals, secs = [], []
    n = p = reps = 0
    for i in range(args.warmup + args.steps):
        t, n, p, reps = cpu_run(w, img, max(1.0, args.cpu_sample_s / max(args.steps, 1)), threads)
        if i >= args.warmup:
            vals.append(p / t)
            secs.append(t)
    v = float(np.median(vals))
    sample = (f"per step {reps} x the first {n} of {w.nq} queries; ParaPFD/regression decode + exact AND on "
              f"the compressed index built by the oracle's encoders (oracle port of the reference CPU path), "
              f"{threads} threads")
    line = {"metric": "postings/s", "value": v, "unit": "postings/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            # one step = one bounded CPU sample of the workload (see cpu_baseline.sample)
            "ms_per_step": float(np.mean(secs)) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": bench_config(w, params, desc),
            "cpu_baseline": {"value": v, "unit": "postings/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "postings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def decode_measure(ctx, ix, w, sizes, arrays, stream, flush, args):
    """Decode every list of the index on the device; device time per pass with
    CUDA events on the context stream, L2 flushed before each pass."""
    import torch

    n = int(sizes.postings)
    meta_per_seg = {0: 12, 1: 8, 2: 12, 3: 28, 4: 28, 5: 12, 6: 12}
    codecs = arrays.lists["codec"].astype(np.int64)
    nseg = arrays.lists["nseg"].astype(np.int64)
    meta = int(sum(meta_per_seg[int(c)] * int(s) for c, s in zip(codecs, nseg)))
    alg = 4 * (int(sizes.nwords) - 8) + meta + 4 * n
    out = torch.empty(n, dtype=torch.int32, device=flush.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        ctx.decode_lists_device(ix, 0, ix.nlists, out.data_ptr())
    times = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush_l2(flush)  # on the decode's stream, no host sync: the events time the kernel alone
            e0.record(stream)
            ctx.decode_lists_device(ix, 0, ix.nlists, out.data_ptr())
            e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    # every decoded posting against the source docIDs, 256M at a time on the device
    ok, step = True, 1 << 28
    for i in range(0, n, step):
        src = torch.from_numpy(w.docs[i:i + step].view(np.int32)).to(out.device)
        ok &= bool(torch.equal(out[i:i + step], src))
        del src
    ms = float(np.mean(times))
    peak, kind = peak_hbm()
    gbs = alg / (ms / 1e3) / 1e9
    del out
    return {"kernel": "k_decode_lists", "postings": n, "ms": ms, "postings_per_s": n / (ms / 1e3),
            "algorithmic_bytes": alg, "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
            "peak_kind": kind, "matches_source": ok}


def serving_measure(ix, w, algos, device, want_cs, seed=0xEC1E0005):
    """Continuous-batching server on the resident index: open-loop Poisson
    arrivals of the workload's queries at several rates (and all at once for
    the saturated throughput); p50/p99 submit->result latency per rate, for
    each search method. The replay's result checksum must equal the batch's."""
    import exclucene_b200 as ex

    lens = np.diff(w.list_offsets).astype(np.int64)
    max_keys = max(int(min(lens[w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]], default=0)) for q in range(w.nq))
    out = {}
    rng = np.random.default_rng(seed)
    rates = [5_000, 50_000, 200_000]
    arrivals = {r: np.cumsum(rng.exponential(1.0 / r, w.nq)) for r in rates}
    for a in algos:
        srv = ex.Server(ix, device=device, slots=4, max_batch_queries=4096, max_batch_keys=max(1 << 22, max_keys),
                        algo=a)
        try:
            srv.replay(w.terms, w.term_offsets, np.zeros(w.nq))  # warm-up
            res = {}
            for r in rates:
                srv.reset_stats()
                lat, cs, wall = srv.replay(w.terms, w.term_offsets, arrivals[r])
                st = srv.stats()
                res[f"{r}"] = {"offered_qps": r, "qps": w.nq / wall, "p50_us": float(np.percentile(lat, 50) * 1e6),
                               "p99_us": float(np.percentile(lat, 99) * 1e6), "mean_batch": st["mean_batch"],
                               "max_inflight": st["max_inflight"], "checksum_ok": cs == want_cs}
            srv.reset_stats()
            lat, cs, wall = srv.replay(w.terms, w.term_offsets, np.zeros(w.nq))
            st = srv.stats()
            res["saturated"] = {"qps": w.nq / wall, "p50_us": float(np.percentile(lat, 50) * 1e6),
                                "p99_us": float(np.percentile(lat, 99) * 1e6), "mean_batch": st["mean_batch"],
                                "max_inflight": st["max_inflight"], "checksum_ok": cs == want_cs,
                                "pool_peak_bytes": st["pool_peak_bytes"]}
            out[a] = res
        finally:
            srv.close()
    return {"slots": 4, "max_batch_queries": 4096, "queries": w.nq,
            "arrivals": "open-loop Poisson, seeded; latency = submit to result in host memory", "by_algo": out}


# ---------------------------------------------------------------------------

def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # rank 0 alone, on the single-GPU batch; no product code is loaded
        if rank == 0:
            import oracle

            gen = type("OracleGen", (), {k[3:]: staticmethod(getattr(oracle, k)) for k in dir(oracle)
                                         if k.startswith("wl_")})
            w, params, desc = make_workload(args.workload, args.scale, gen)
            if args.codec:
                params["codec"] = args.codec
            reference_arm(args, w, desc, params)
        return

    # under --gpus N the query-stream workloads draw N batches from one stream
    # and rank r takes batch r (replicas.shard_queries); the others run the
    # same batch on every rank. Either way each rank's batch is a full step.
    import copy

    import torch
    import torch.distributed as dist

    import exclucene_b200 as ex
    from exclucene_b200 import replicas

    stream_wl = args.workload in ("zipf", "serving")
    wall, params, desc = make_workload(args.workload, args.scale, nq_factor=world if stream_wl else 1)
    if args.codec:
        params["codec"] = args.codec
    w = wall
    if world > 1 and stream_wl:
        w = copy.copy(wall)
        w.terms, w.term_offsets, _, _ = replicas.shard_queries(wall.terms, wall.term_offsets, rank, world)

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    lens = np.diff(w.list_offsets).astype(np.int64)
    shortest = sum(int(min(lens[w.terms[w.term_offsets[q]:w.term_offsets[q + 1]]], default=0)) for q in range(w.nq))
    ctx = ex.Context(local, max_queries=max(w.nq, 1024), max_keys=max(1 << 20, 2 * shortest))
    layout = None
    if not args.no_layout_tune and args.workload in LAYOUT_CANDIDATES and "codecs" not in params:
        # index-layout autotuner on this batch: candidate layouts built on the
        # GPU, each tuned and timed; for the skewed workload (HS top-k bits
        # 8..16 autotuned) the chosen layout is the one measured below, for the
        # others the named layout is kept and the tuner's result is reported
        d_all = torch.from_numpy(w.docs.view(np.int32)).to(dev)
        torch.cuda.synchronize()
        cands = LAYOUT_CANDIDATES[args.workload](params)
        t0 = time.perf_counter()
        lix, lbest, lrep = ctx.autotune_layout(d_all.data_ptr(), w.list_offsets, cands, w.terms, w.term_offsets)
        lix.close()
        del d_all
        layout = {"candidates": [{k: v for k, v in r.items() if k != "tuning"} | {"algo": (r["tuning"] or {}).get("algo")}
                                 for r in lrep], "chosen": lbest, "wall_s": time.perf_counter() - t0,
                  "applied": args.workload == "skewed"}
        if args.workload == "skewed":
            params.update({k: v for k, v in cands[lbest].items()})
        ctx.set_tuning(algo="auto", warps_per_cta=8, ctas_per_sm=5, merge_segs=2, tile_split=0)  # back to defaults
    t_build = time.perf_counter()
    ix = ex.Index(w.docs, w.list_offsets, **params)
    host_build_s = time.perf_counter() - t_build
    ctx.upload(ix)
    learn = None
    if not args.no_learn:
        lmin = args.learn_min or {"zipf": 1 << 16, "pairs": 1 << 20, "skewed": 1 << 20, "learned": 1 << 20,
                                  "serving": 1 << 20}[args.workload]
        t0 = time.perf_counter()
        learn = ctx.learn(ix, min_postings=lmin)
        learn["wall_s"] = time.perf_counter() - t0
        learn["min_postings"] = lmin
    sizes = ix.sizes()
    arrays = ix.export()
    index_build = None
    if params["codec"] in ("parapfd", "seglrc", "lrc", "lrcseg", "hs_seglrc", "hs_parapfd") and "codecs" not in params:
        # the same index built by the device kernels, from the docIDs in HBM
        d_all = torch.from_numpy(w.docs.view(np.int32)).to(dev)
        torch.cuda.synchronize()
        hs = {k: params[k] for k in ("hs_bucket", "hs_kbits", "hs_ubits") if k in params}
        ctx.build_index(d_all.data_ptr(), w.list_offsets, codec=params["codec"], block=params["block"],
                        frac=params["frac"], **hs).close()  # warm-up
        t_build = time.perf_counter()
        dix = ctx.build_index(d_all.data_ptr(), w.list_offsets, codec=params["codec"], block=params["block"],
                              frac=params["frac"], **hs)
        dev_build_s = time.perf_counter() - t_build
        da = dix.export()
        same = all(np.array_equal(getattr(da, k), getattr(arrays, k)) for k in ("words", "seg_head", "seg_rec",
                                                                                 "seg_reg", "dir"))
        dix.close()
        del d_all
        index_build = {"host_s": host_build_s, "host_threads": os.cpu_count(), "device_s": dev_build_s,
                       "device_image_identical": bool(same),
                       "device_note": "fits, residuals, blocks on the GPU; includes copying the image to the host"}
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    d_terms = torch.from_numpy(w.terms.astype(np.int32)).to(dev)
    d_toff = torch.from_numpy(w.term_offsets.astype(np.int32)).to(dev)
    cap = max(1, shortest)
    d_offs = torch.zeros(w.nq + 1, dtype=torch.int32, device=dev)
    d_docs = torch.zeros(cap, dtype=torch.int32, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.int32, device=dev)  # > L2 (126 MB)
    torch.cuda.synchronize()

    # a second context on the same resident index replays each batch as a CUDA graph
    gctx = ex.Context(local, max_queries=max(w.nq, 1024), max_keys=max(1 << 20, 2 * shortest), use_graphs=True)
    if args.algo and args.ctas_per_sm:
        for c in (ctx, gctx):
            c.set_tuning(algo=args.algo, warps_per_cta=8, ctas_per_sm=args.ctas_per_sm, merge_segs=2, tile_split=0)

    def step(c, algo):
        c.intersect_device(ix, d_terms.data_ptr(), d_toff.data_ptr(), w.nq, algo, d_offs.data_ptr(),
                           d_docs.data_ptr(), cap)

    def measure(c, algo, k, warm):
        for _ in range(warm):
            step(c, algo)
        c.check()
        tot, probe = [], []
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        # the L2 flush runs on the batch's own stream just before it, with no
        # host sync in between: the host has enqueued the batch while the
        # flush runs, so the events around the batch time the kernel on the
        # device, not the host's launch call (e2e below times that)
        cstream = torch.cuda.ExternalStream(c.stream, device=dev)
        for _ in range(k):
            with torch.cuda.stream(cstream):
                flush_l2(flush)
            step(c, algo)
            st = c.stats()
            tot.append(st.total_ms)
            probe.append(st.probe_ms)
        torch.cuda.synchronize()
        c.check()
        if world > 1:
            dist.barrier()
        # outside the timed region: the last timed step's result against the oracle
        offs_h = d_offs.cpu().numpy().astype(np.uint32)
        parity[algo if c is ctx else algo + "/graph"] = mismatched_queries(
            offs_h, d_docs[: int(offs_h[-1])].cpu().numpy().astype(np.uint32))
        return float(np.mean(tot)), float(np.mean(probe)), st

    # The checker: the exact AND of this rank's batch by the CPU oracle,
    # computed once before any timing; every timed configuration's last
    # result is compared with it query by query after its timed region.
    import oracle

    ora_offs, ora_docs = oracle.answer_batch(w.docs, w.list_offsets, w.terms, w.term_offsets)
    ora_cs = oracle.checksum(ora_offs, ora_docs)
    parity = {}

    def mismatched_queries(offs_h, docs_h) -> int:
        o = offs_h.astype(np.uint64)
        if len(o) != len(ora_offs):
            return w.nq
        if np.array_equal(o, ora_offs):
            if len(ora_docs) == 0:
                return 0
            diff = (docs_h != ora_docs).astype(np.int64)
            starts = ora_offs[:-1].astype(np.int64)
            nonempty = np.diff(ora_offs) > 0
            per_q = np.zeros(w.nq, dtype=np.int64)
            per_q[nonempty] = np.add.reduceat(diff, starts[nonempty])
            return int((per_q > 0).sum())
        bad = 0
        for q in range(w.nq):
            a = docs_h[int(o[q]):int(o[q + 1])] if o[q + 1] >= o[q] else None
            if a is None or not np.array_equal(a, ora_docs[int(ora_offs[q]):int(ora_offs[q + 1])]):
                bad += 1
        return bad

    postings = query_postings(w)
    algos = [args.algo] if args.algo else ["bsearch", "hashseg", "segreg"] + ([] if args.no_learn else ["learned"])
    per_algo, per_algo_graph = {}, {}
    tune = None
    with ClockSampler(local) as clk:
        for a in algos:
            per_algo[a] = measure(ctx, a, args.steps, args.warmup)
            per_algo_graph[a] = measure(gctx, a, args.steps, args.warmup)
        if not args.algo:
            # the autotuner on the workload's own batch; "tuned" runs algo=auto with its choice
            tune = gctx.autotune(ix, w.terms, w.term_offsets)
            per_algo_graph["tuned"] = measure(gctx, "auto", args.steps, args.warmup)
            ctx.autotune(ix, w.terms, w.term_offsets)  # stream-launch twin, for the per-kernel times
            per_algo["tuned"] = measure(ctx, "auto", args.steps, args.warmup)
    clocks = clk.summary()
    best = min(per_algo, key=lambda a: min(per_algo[a][0], per_algo_graph[a][0])) if not args.algo else args.algo
    ms, pms, st = per_algo[best]
    launch_mode = "stream"
    if per_algo_graph[best][0] < ms:
        ms, launch_mode = per_algo_graph[best][0], "cuda graph"
    main_ctx = gctx if launch_mode == "cuda graph" else ctx
    best_algo = "auto" if best == "tuned" else best  # the tuned setting runs as algo=auto
    # every rank ran a full batch; the job time is the slowest rank's and the
    # job's work is the sum of the ranks' batches
    ms = replicas.max_over_ranks(ms, device=dev)
    pms = replicas.max_over_ranks(pms, device=dev)
    job_postings = replicas.sum_over_ranks(postings, device=dev)
    job_queries = replicas.sum_over_ranks(w.nq, device=dev)
    value = job_postings / (ms / 1e3)
    cs = ora_cs

    # end to end through the public host API, inputs and results in host memory:
    # excl_submit_into (H2D of the queries from pinned memory; the last kernel
    # writes offsets and docIDs through the mapping of pinned host arrays), and
    # excl_submit + excl_wait (pinned staging, D2H copies after the batch)
    p_terms, p_toff = ex.pinned_empty(len(w.terms)), ex.pinned_empty(len(w.term_offsets))
    p_terms[:], p_toff[:] = w.terms, w.term_offsets
    p_off, p_docs = ex.pinned_empty(w.nq + 1), ex.pinned_empty(cap)
    h_off = np.zeros(w.nq + 1, dtype=np.uint32)
    h_docs = np.zeros(cap, dtype=np.uint32)

    def e2e_into():
        b = main_ctx.submit_into(ix, p_terms, p_toff, p_off, p_docs, best_algo)
        tot = b.wait()
        b.free()
        return tot

    def e2e_copy():
        b = main_ctx.submit(ix, w.terms, w.term_offsets, best_algo)
        tot = b.wait_into(h_off, h_docs)
        b.free()
        return tot

    e2e_ms = {}
    for name, fn in (("submit_into", e2e_into), ("submit_wait", e2e_copy)):
        for _ in range(args.warmup):
            fn()
        e2e_t = []
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tot = fn()
            e2e_t.append(time.perf_counter() - t0)
        e2e_ms[name] = replicas.max_over_ranks(float(np.mean(e2e_t)), device=dev) * 1e3
    parity["e2e submit_into"] = mismatched_queries(np.asarray(p_off, dtype=np.uint32),
                                                   np.asarray(p_docs[:tot], dtype=np.uint32))
    parity["e2e submit_wait"] = mismatched_queries(h_off, h_docs[:tot])
    e2e_s = e2e_ms["submit_into"] / 1e3
    h2d = w.terms.nbytes + w.term_offsets.nbytes
    d2h = h_off.nbytes + 4 * tot

    peak, peak_kind = peak_hbm()
    probe_bytes = algorithmic_bytes(w, arrays)
    algo_bytes = probe_bytes + batch_bytes(w, int(st.tiles), int(ora_offs[-1]))
    # the dominant kernel is the batch kernel itself (one launch per step):
    # its duration is the stream-launched step's CUDA-event time
    kms = replicas.max_over_ranks(per_algo[best][0], device=dev)
    achieved = algo_bytes / (kms / 1e3) / 1e9

    # whole-index decode (K1/K2): compressed words + per-segment metadata read, 4 B per posting written
    dec = decode_measure(ctx, ix, w, sizes, arrays, stream, flush, args)
    serving = None
    if not args.no_serve:
        serving = serving_measure(ix, w, ["segreg"] + ([] if args.no_learn else ["learned"]), local, cs)
    if serving:
        for a, res in serving["by_algo"].items():
            parity[f"serving {a}"] = sum(0 if r["checksum_ok"] else 1 for r in res.values())
    mism = int(replicas.sum_over_ranks(sum(parity.values()), device=dev))
    parity_line = {"checked_queries": int(job_queries), "mismatches": mism,
                   "per_run": parity, "oracle_checksum": list(ora_cs),
                   "checker": "CPU oracle exact AND (oracle.answer_batch) of the same batch, per query; "
                              "serving runs by result checksum"}
    line = {
        "metric": "postings/s", "value": value, "unit": "postings/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": bench_config(w, params, desc),
        "algo": best, "index_device_bytes": int(sizes.device_bytes), "index_postings": int(sizes.postings),
        "queries_per_s": job_queries / (ms / 1e3),
        "launch": launch_mode,
        "per_algo_ms": {a: round(per_algo[a][0], 4) for a in per_algo},
        "per_algo_graph_ms": {a: round(per_algo_graph[a][0], 4) for a in per_algo_graph},
        "per_algo_probe_ms": {a: round(per_algo[a][1], 4) for a in per_algo},
        "learned_over_plain": (min(min(per_algo[a][0], per_algo_graph[a][0]) for a in per_algo
                                   if a in ("bsearch", "hashseg")) /
                               min(per_algo["learned"][0], per_algo_graph["learned"][0]))
        if "learned" in per_algo else None,
        "learned_over_bsearch": (min(per_algo["bsearch"][0], per_algo_graph["bsearch"][0]) /
                                 min(per_algo["learned"][0], per_algo_graph["learned"][0]))
        if "learned" in per_algo and "bsearch" in per_algo else None,
        # against the codec's own linear model (SegLRC segment regression windows)
        "learned_over_segreg": (min(per_algo["segreg"][0], per_algo_graph["segreg"][0]) /
                                min(per_algo["learned"][0], per_algo_graph["learned"][0]))
        if "learned" in per_algo and "segreg" in per_algo else None,
        "learned_models": learn,
        "index_build": index_build,
        "layout_tune": layout,
        "autotune": tune,
        "per_algo_postings_per_s": {a: job_postings / (min(per_algo[a][0], per_algo_graph[a][0]) / 1e3)
                                    for a in per_algo},
        "stats": {"tiles": int(st.tiles), "keys": int(st.keys), "probes": int(st.probes),
                  "fallbacks": int(st.fallbacks), "probe_ms": pms, "pack_ms": st.pack_ms,
                  "compact_ms": st.compact_ms},
        "checksum": list(cs),
        "parity": parity_line,
        "roofline": {"bound": "hbm", "kernel": "k_batch", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "kernel_ms": kms,
                     "traffic": NCU_BATCH_TRAFFIC.get(args.workload) if args.scale == 1.0 else None,
                     "traffic_note": "ncu dram read+write per k_batch launch",
                     "algorithmic_bytes": algo_bytes, "probe_bytes": probe_bytes,
                     "probe_phase_gbs": probe_bytes / (pms / 1e3) / 1e9 if pms > 0 else None,
                     "peak_kind": peak_kind},
        "e2e": {"value": job_postings / e2e_s, "unit": "postings/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_s * 1e3, "api": "excl_submit_into + excl_wait",
                "ms_per_step_submit_wait": e2e_ms["submit_wait"],
                "l2": "flushed before each step (outside the wall-clock region)"},
        # one batch kernel per step: the per-algo runs (stream and graph), the tuned runs, the two e2e arms
        "gpu_launches": (2 * len(algos) + (2 if tune else 0) + 2) * args.steps,
        "clocks": clocks,
        "decode": dec,
        "serving": serving,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        img = oracle.encode_corpus(w.docs, w.list_offsets,
                                   params["codecs"] if params.get("codecs") is not None
                                   else oracle.CODECS[params["codec"]], block=params["block"], frac=params["frac"],
                                   bucket=params.get("hs_bucket", 256), kbits=params.get("hs_kbits", 0),
                                   ubits=params.get("hs_ubits", 32))
        t, n, p, reps = cpu_run(w, img, args.cpu_sample_s, threads)
        line["cpu_baseline"] = {"value": p / t, "unit": "postings/s", "cores": threads, "kind": "port",
                                "sample": f"{reps} x the first {n} of {w.nq} queries ({t:.1f} s); ParaPFD/regression "
                                          "decode + exact AND on the index built by the oracle's encoders "
                                          "(oracle port)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    gctx.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    if mism:
        sys.stderr.write(f"parity: {mism} queries differ from the oracle\n")
        sys.exit(1)


if __name__ == "__main__":
    main()
