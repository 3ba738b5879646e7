"""Learned position models: the training kernels' gradient against the CPU
oracle, exactness of every leaf window (checked on the CPU with the oracle's
restatement of the FP32 inference), bit-exact learned intersections, and
what training gains over the untrained network."""
import numpy as np
import pytest

import exclucene_b200 as ex
import oracle
from exclucene_b200 import synth


def _random_params(rng):
    P = np.zeros(1153, np.float32)
    P[0:32] = rng.uniform(0.5, 2.0, 32)            # w1 >= 0
    P[32:64] = -rng.uniform(0.0, 1.0, 32)          # b1
    P[64:64 + 1024] = rng.uniform(0.0, 0.1, 1024)  # w2 >= 0
    P[1088:1120] = rng.uniform(-0.05, 0.05, 32)    # b2
    P[1120:1152] = rng.uniform(0.0, 0.1, 32)       # w3 >= 0
    P[1152] = 0.01
    return P


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    P = _random_params(rng)
    x = rng.uniform(0, 1, 64).astype(np.float32)
    y = np.sort(rng.uniform(0, 1, 64)).astype(np.float32)
    g, _ = oracle.mlp_grad(P, x, y)
    for j in [0, 5, 40, 64, 64 + 33 * 7, 1088 + 3, 1120 + 9, 1152]:
        e = 1e-2 * max(abs(float(P[j])), 1e-2)
        Pp, Pm = P.copy(), P.copy()
        Pp[j] += e
        Pm[j] -= e
        num = (oracle.mlp_grad(Pp, x, y)[1] - oracle.mlp_grad(Pm, x, y)[1]) / (float(Pp[j]) - float(Pm[j]))
        assert abs(num - g[j]) <= 1e-3 * max(1e-3, np.abs(g).max()), (j, num, g[j])


@pytest.mark.gpu
def test_training_gradient_matches_oracle(gpu_ctx):
    rng = np.random.default_rng(5)
    for n in (1, 127, 4096):
        P = _random_params(rng)
        x = rng.uniform(0, 1, n).astype(np.float32)
        y = np.clip(x + rng.normal(0, 0.05, n), 0, 1).astype(np.float32)
        g_gpu, l_gpu = gpu_ctx.model_grad(P, x, y)
        g_cpu, l_cpu = oracle.mlp_grad(P, x, y)
        scale = max(np.abs(g_cpu).max(), 1e-6)
        # FP32 kernel vs double oracle: agreement to 1e-4 of the largest component
        assert np.abs(g_gpu - g_cpu).max() <= 1e-4 * scale + 1e-7, n
        assert abs(l_gpu - l_cpu) <= 1e-4 * max(l_cpu, 1e-6)


@pytest.fixture(scope="module")
def long_lists():
    lens = [300_000, 450_000, 120_000, 2000, 70_000]
    a = synth.uniform_lists(lens[:3], ubits=24, seed=11)
    b = synth.clustered_lists(lens[3:] + [500_000], ubits=24, seed=12)
    docs = np.concatenate([a.docs, b.docs])
    loff = np.concatenate([a.list_offsets, a.list_offsets[-1] + b.list_offsets[1:]]).astype(np.uint64)
    return docs, loff


@pytest.mark.gpu
@pytest.mark.parametrize("codec", ["seglrc", "parapfd"])
def test_learned_windows_are_exact_and_probes_bit_exact(gpu_ctx, long_lists, codec):
    docs, loff = long_lists
    ix = ex.Index(docs, loff, codec=codec, block=256 if codec == "seglrc" else 128)
    gpu_ctx.upload(ix)
    rep = gpu_ctx.learn(ix, min_postings=100_000, nleaves=1024, steps=200, batch=8192)
    assert rep["models"] == 4
    for l in range(ix.nlists):
        m = ix.model(l)
        n = int(loff[l + 1] - loff[l])
        if n < 100_000:
            assert m is None
            continue
        root, hdr, leaves = m
        assert (root[0:32] >= 0).all() and (root[64:1088] >= 0).all() and (root[1120:1152] >= 0).all()
        keys = docs[loff[l]:loff[l + 1]]
        bad, counts = oracle.model_check(root, hdr, leaves, keys)
        assert bad == 0, f"list {l}: {bad} keys outside their leaf window"
        assert counts.sum() == n
        # the stored routing tables reproduce the network's routing exactly,
        # on the list's keys and on every other key tried in its range
        grid, bnd, first, shift = ix.model_tables(l)
        probe = np.unique(np.concatenate([keys, np.random.default_rng(l).integers(
            int(keys[0]), int(keys[-1]) + 1, 200_000, dtype=np.uint64).astype(np.uint32)]))
        j = (probe.astype(np.int64) - first) >> shift
        lo, hi = grid[j].astype(np.int64), grid[j + 1].astype(np.int64)
        glob = np.searchsorted(bnd, probe, side="right") - 1
        assert ((glob >= lo) & (glob <= hi)).all(), "grid does not bracket the leaf"
        assert np.array_equal(glob.astype(np.uint32), oracle.model_leaves(root, hdr, probe))
    # probes: keys from the lists and random keys, AND with each long list
    rng = np.random.default_rng(9)
    probes = [np.unique(np.concatenate([rng.choice(docs[loff[l]:loff[l + 1]], 3000),
                                        rng.integers(0, 1 << 24, 3000)]).astype(np.uint32)) for l in range(ix.nlists)]
    all_docs = np.concatenate([docs] + probes)
    all_off = np.concatenate([loff, loff[-1] + np.cumsum([len(p) for p in probes])]).astype(np.uint64)
    ix2 = ex.Index(all_docs, all_off, codec=codec, block=256 if codec == "seglrc" else 128)
    gpu_ctx.upload(ix2)
    gpu_ctx.learn(ix2, min_postings=100_000, nleaves=1024, steps=200, batch=8192)
    nl = ix.nlists
    terms = np.array([t for l in range(nl) for t in (nl + l, l)], np.uint32)
    toff = np.arange(0, 2 * nl + 1, 2, dtype=np.uint32)
    eo, ed = oracle.answer(all_docs, all_off, terms, toff)
    for algo in ("learned", "auto", "hashseg", "segreg", "bsearch"):
        offs, got = gpu_ctx.intersect(ix2, terms, toff, algo=algo)
        assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(got, ed), algo
    ix.close()
    ix2.close()


@pytest.mark.gpu
def test_training_narrows_the_windows(gpu_ctx, long_lists):
    """What the trained network gains: the same two-stage model with the root
    left at its initial weights (1 step) routes keys far less evenly, so its
    leaf windows are wider than after training."""
    docs, loff = long_lists
    ix = ex.Index(docs, loff, codec="seglrc")
    gpu_ctx.upload(ix)
    untrained = gpu_ctx.learn(ix, min_postings=100_000, nleaves=1024, steps=1, batch=8192)
    trained = gpu_ctx.learn(ix, min_postings=100_000, nleaves=1024, steps=300, batch=16384)
    assert trained["final_loss"] < untrained["final_loss"]
    assert trained["mean_window"] < untrained["mean_window"]
    ix.close()


@pytest.mark.gpu
def test_learned_beats_the_plain_methods(gpu_ctx):
    """What the trained model gains over the method without it: on a fixed
    batch of probe-key lists ANDed with long SegLRC lists, the learned probe
    (model window, then a search inside it) takes less device time than both
    plain comparators (binary search over the heads or the bucket directory,
    then a binary search over the block), with bit-exact output for all three.
    Times are the fastest of 7 batches after a warm-up (CUDA events), which is
    the least sensitive to other work on a shared GPU."""
    lens = [3_000_000, 2_000_000, 4_000_000, 1_500_000]
    t = synth.uniform_lists(lens, ubits=28, seed=21)
    rng = np.random.default_rng(22)
    keys = []
    for q in range(400):
        l = q % len(lens)
        lst = t.docs[t.list_offsets[l]:t.list_offsets[l + 1]]
        k = np.unique(np.concatenate([rng.choice(lst, 6000, replace=False),
                                      rng.integers(0, 1 << 28, 6000, dtype=np.uint64).astype(np.uint32)]))
        keys.append(k.astype(np.uint32))
    docs = np.concatenate([t.docs] + keys)
    loff = np.concatenate([t.list_offsets, t.list_offsets[-1] + np.cumsum([len(k) for k in keys])]).astype(np.uint64)
    nl = len(lens)
    terms = np.array([x for q in range(400) for x in (nl + q, q % nl)], np.uint32)
    toff = np.arange(0, 801, 2, dtype=np.uint32)
    ix = ex.Index(docs, loff, codec="seglrc")
    gpu_ctx.upload(ix)
    gpu_ctx.learn(ix, min_postings=1_000_000, steps=300, batch=16384)
    eo, ed = oracle.answer(docs, loff, terms, toff)
    ms = {}
    for algo in ("learned", "bsearch", "hashseg"):
        offs, got = gpu_ctx.intersect(ix, terms, toff, algo=algo)
        assert np.array_equal(offs.astype(np.uint64), eo) and np.array_equal(got, ed), algo
        runs = []
        for _ in range(7):
            gpu_ctx.intersect(ix, terms, toff, algo=algo)
            runs.append(gpu_ctx.stats().total_ms)
        ms[algo] = float(min(runs))
    assert ms["learned"] < min(ms["bsearch"], ms["hashseg"]), ms
    ix.close()
