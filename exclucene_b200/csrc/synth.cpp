// Seeded synthetic posting lists and query streams for the five benchmark
// workloads (libexcl_synth.so). The reference's real indexes (Baidu, GOV2) and
// query logs are not available; these generators stand in for them with the
// shapes, sizes and value distributions of the workloads:
//   uniform   sorted docIDs drawn uniformly without replacement
//   clustered 70% of the docIDs in dense runs (run length ~ Geometric(mean 64),
//             inter-run gap ~ Geometric(mean g)) and 30% uniform
//   zipfgap   gaps ~ Zipf(s) clipped to 2^20, up to the universe end
// PRNG: splitmix64 seeding xoshiro256**; every list has its own sub-seed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t &x) {
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        for (auto &v : s) v = splitmix(seed);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint64_t below(uint64_t n) { return (uint64_t)(((unsigned __int128)next() * n) >> 64); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    // Geometric on {1, 2, ...} with the given mean
    uint64_t geom(double mean) {
        if (mean <= 1.0) return 1;
        const double p = 1.0 / mean;
        const double u = unit();
        return 1 + (uint64_t)std::floor(std::log1p(-u) / std::log1p(-p));
    }
};

uint64_t sub_seed(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t x = seed ^ (a * 0x9e3779b97f4a7c15ull) ^ (b * 0xc2b2ae3d27d4eb4full);
    return Rng::splitmix(x);
}

// k distinct values of [0, N), sorted: draw, sort, unique, top up.
void uniform_sorted(Rng &r, uint64_t N, uint64_t k, std::vector<uint32_t> &out) {
    out.clear();
    if (k == 0) return;
    if (k > N) k = N;
    if (k > N / 2) {
        std::vector<uint32_t> comp;
        uniform_sorted(r, N, N - k, comp);
        out.reserve(k);
        uint64_t j = 0;
        for (uint64_t v = 0; v < N; ++v) {
            if (j < comp.size() && comp[j] == v) {
                ++j;
                continue;
            }
            out.push_back((uint32_t)v);
        }
        return;
    }
    out.reserve(k + k / 8 + 16);
    while (out.size() < k) {
        const uint64_t need = k - out.size();
        const size_t old = out.size();
        for (uint64_t i = 0; i < need; ++i) out.push_back((uint32_t)r.below(N));
        std::sort(out.begin() + old, out.end());
        std::inplace_merge(out.begin(), out.begin() + old, out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    }
}

// Clustered mixture of exactly n docIDs in [0, U).
void clustered_sorted(Rng &r, uint64_t U, uint64_t n, double run_mean, double gap_mean, std::vector<uint32_t> &out) {
    out.clear();
    if (n > U) n = U;
    const uint64_t nrun = (uint64_t)(0.7 * (double)n);
    // shrink the inter-run gap when the runs would not fit the universe
    const double runs = std::max(1.0, (double)nrun / run_mean);
    const double fit = (double)U / runs - run_mean;
    const double g = std::max(1.0, std::min(gap_mean, fit * 0.9));
    std::vector<uint32_t> a;
    a.reserve(n + n / 4);
    uint64_t pos = r.below(std::max<uint64_t>(1, (uint64_t)g));
    while (a.size() < nrun) {
        const uint64_t len = r.geom(run_mean);
        for (uint64_t i = 0; i < len && a.size() < nrun; ++i) {
            a.push_back((uint32_t)(pos % U));
            ++pos;
        }
        pos += r.geom(g);
    }
    std::vector<uint32_t> u;
    uniform_sorted(r, U, n - a.size(), u);
    std::sort(a.begin(), a.end());
    out.resize(a.size() + u.size());
    std::merge(a.begin(), a.end(), u.begin(), u.end(), out.begin());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    while (out.size() < n) {
        std::vector<uint32_t> extra;
        uniform_sorted(r, U, n - out.size(), extra);
        std::vector<uint32_t> m(out.size() + extra.size());
        std::merge(out.begin(), out.end(), extra.begin(), extra.end(), m.begin());
        m.erase(std::unique(m.begin(), m.end()), m.end());
        out.swap(m);
    }
    if (out.size() > n) {
        // drop random surplus elements (rare) keeping the order
        std::vector<uint8_t> drop(out.size(), 0);
        uint64_t extra = out.size() - n;
        while (extra) {
            const uint64_t i = r.below(out.size());
            if (!drop[i]) {
                drop[i] = 1;
                --extra;
            }
        }
        size_t w = 0;
        for (size_t i = 0; i < out.size(); ++i)
            if (!drop[i]) out[w++] = out[i];
        out.resize(w);
    }
}

// Gaps ~ Zipf(s) on {1..cap} from the start until the universe end.
void zipfgap_sorted(Rng &r, uint64_t U, double s, uint32_t cap, const std::vector<double> &cdf,
                    std::vector<uint32_t> &out) {
    out.clear();
    uint64_t pos = r.below(1024);
    while (pos < U) {
        out.push_back((uint32_t)pos);
        const double u = r.unit() * cdf.back();
        const uint64_t g = (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin()) + 1;
        pos += std::min<uint64_t>(g, cap);
    }
    (void)s;
}

struct Set {
    std::vector<uint32_t> docs;
    std::vector<uint64_t> loff{0};
    std::vector<uint32_t> terms;
    std::vector<uint32_t> toff{0};
    std::vector<uint8_t> codecs;
    std::vector<double> info;  // workload-specific facts (e.g. realized gap means)
};

template <typename F>
void parallel_lists(uint32_t nl, unsigned threads, std::vector<std::vector<uint32_t>> &lists, F gen) {
    lists.assign(nl, {});
    std::atomic_uint next{0};
    std::vector<std::thread> th;
    if (!threads) threads = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned t = 0; t < threads; ++t)
        th.emplace_back([&]() {
            for (;;) {
                const uint32_t l = next.fetch_add(1);
                if (l >= nl) break;
                gen(l, lists[l]);
            }
        });
    for (auto &t : th) t.join();
}

void append_lists(Set &s, std::vector<std::vector<uint32_t>> &lists) {
    size_t tot = s.docs.size();
    for (auto &l : lists) tot += l.size();
    s.docs.reserve(tot);
    for (auto &l : lists) {
        s.docs.insert(s.docs.end(), l.begin(), l.end());
        s.loff.push_back(s.docs.size());
        std::vector<uint32_t>().swap(l);
    }
}

void add_query(Set &s, std::initializer_list<uint32_t> t) {
    for (uint32_t v : t) s.terms.push_back(v);
    s.toff.push_back((uint32_t)s.terms.size());
}

}  // namespace

extern "C" {

typedef struct synth_set synth_set;

// Config 1: npairs of (short, long) uniform lists over 2^ubits; query i = lists (2i, 2i+1).
synth_set *synth_pairs(uint64_t seed, uint32_t npairs, uint32_t short_len, uint32_t long_len, uint32_t ubits,
                       uint32_t threads) {
    Set *s = new Set();
    const uint64_t U = 1ull << ubits;
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(2 * npairs, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 1, l));
        uniform_sorted(r, U, (l & 1) ? long_len : short_len, out);
    });
    append_lists(*s, lists);
    for (uint32_t i = 0; i < npairs; ++i) add_query(*s, {2 * i, 2 * i + 1});
    return (synth_set *)s;
}

// Config 2: Zipf(1) document frequencies df_r = min(cap, round(cap / r)) over
// ndocs documents; nq queries of qmin..qmax distinct terms drawn with
// probability proportional to df^0.5.
synth_set *synth_zipf_corpus(uint64_t seed, uint32_t ndocs, uint32_t nterms, uint32_t cap, uint32_t nq, uint32_t qmin,
                             uint32_t qmax, uint32_t threads) {
    Set *s = new Set();
    std::vector<uint32_t> df(nterms);
    for (uint32_t r = 0; r < nterms; ++r) {
        const double v = std::round((double)cap / (double)(r + 1));
        df[r] = (uint32_t)std::max(1.0, std::min((double)cap, v));
    }
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(nterms, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 2, l));
        uniform_sorted(r, ndocs, df[l], out);
    });
    append_lists(*s, lists);
    std::vector<double> cdf(nterms);
    double acc = 0;
    for (uint32_t r = 0; r < nterms; ++r) cdf[r] = (acc += std::sqrt((double)df[r]));
    Rng r(sub_seed(seed, 3, 0));
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = qmin + (uint32_t)r.below(qmax - qmin + 1);
        std::vector<uint32_t> t;
        while (t.size() < k) {
            const double u = r.unit() * acc;
            const uint32_t id = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
            const uint32_t c = std::min(id, nterms - 1);
            if (std::find(t.begin(), t.end(), c) == t.end()) t.push_back(c);
        }
        for (uint32_t v : t) s->terms.push_back(v);
        s->toff.push_back((uint32_t)s->terms.size());
    }
    return (synth_set *)s;
}

// Config 3: a pool of `npool` long clustered lists (lengths log-uniform in
// [long_min, long_max]) and, per query, one short clustered list (log-uniform
// in [short_min, short_max]) plus 1..3 pool lists. Lists 0..npool-1 are the
// pool, list npool+q is query q's short list.
synth_set *synth_skewed(uint64_t seed, uint32_t ubits, uint32_t npool, uint32_t long_min, uint32_t long_max,
                        uint32_t nq, uint32_t short_min, uint32_t short_max, double run_mean, double gap_mean,
                        uint32_t threads) {
    Set *s = new Set();
    const uint64_t U = 1ull << ubits;
    std::vector<uint32_t> len(npool + nq);
    Rng lr(sub_seed(seed, 4, 0));
    auto logu = [&](Rng &r, double a, double b) { return (uint32_t)std::exp(std::log(a) + r.unit() * (std::log(b) - std::log(a))); };
    for (uint32_t i = 0; i < npool; ++i) len[i] = logu(lr, long_min, long_max);
    for (uint32_t q = 0; q < nq; ++q) len[npool + q] = logu(lr, short_min, short_max);
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(npool + nq, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 5, l));
        clustered_sorted(r, U, len[l], run_mean, gap_mean, out);
    });
    append_lists(*s, lists);
    Rng r(sub_seed(seed, 6, 0));
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = 1 + (uint32_t)r.below(3);
        std::vector<uint32_t> t{npool + q};
        while (t.size() < k + 1) {
            const uint32_t c = (uint32_t)r.below(npool);
            if (std::find(t.begin(), t.end(), c) == t.end()) t.push_back(c);
        }
        for (uint32_t v : t) s->terms.push_back(v);
        s->toff.push_back((uint32_t)s->terms.size());
    }
    return (synth_set *)s;
}

// Config 4: nclust clustered lists (log-uniform lengths in [lmin, lmax]) and
// nzipf Zipf-gap lists over 2^ubits, then nq probe-key lists of log-uniform
// length in [kmin, kmax] (half drawn from the target list, half uniform).
// Lists 0..nclust+nzipf-1 are targets; query q = (target list, key list).
synth_set *synth_learned(uint64_t seed, uint32_t ubits, uint32_t nclust, uint32_t nzipf, uint32_t lmin, uint32_t lmax,
                         double zipf_s, uint32_t zipf_cap, uint32_t nq, uint32_t kmin, uint32_t kmax,
                         uint32_t threads) {
    Set *s = new Set();
    const uint64_t U = 1ull << ubits;
    const uint32_t nt = nclust + nzipf;
    std::vector<uint32_t> len(nt);
    Rng lr(sub_seed(seed, 7, 0));
    auto logu = [&](Rng &r, double a, double b) { return (uint32_t)std::exp(std::log(a) + r.unit() * (std::log(b) - std::log(a))); };
    for (uint32_t i = 0; i < nclust; ++i) len[i] = logu(lr, lmin, lmax);
    std::vector<double> cdf(zipf_cap);
    double acc = 0;
    for (uint32_t g = 1; g <= zipf_cap; ++g) cdf[g - 1] = (acc += std::pow((double)g, -zipf_s));
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(nt, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 8, l));
        if (l < nclust) clustered_sorted(r, U, len[l], 64.0, 4096.0, out);
        else zipfgap_sorted(r, U, zipf_s, zipf_cap, cdf, out);
    });
    // probe-key lists
    std::vector<uint32_t> tgt(nq), klen(nq);
    Rng qr(sub_seed(seed, 9, 0));
    for (uint32_t q = 0; q < nq; ++q) {
        tgt[q] = (uint32_t)qr.below(nt);
        klen[q] = logu(qr, kmin, kmax);
    }
    std::vector<std::vector<uint32_t>> keys;
    parallel_lists(nq, threads, keys, [&](uint32_t q, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 10, q));
        const std::vector<uint32_t> &L = lists[tgt[q]];
        const uint64_t want = std::min<uint64_t>(klen[q], L.size() + U / 2);
        std::vector<uint32_t> a;
        const uint64_t half = std::min<uint64_t>(want / 2, L.size());
        std::vector<uint32_t> pick;
        uniform_sorted(r, L.size(), half, pick);
        for (uint32_t i : pick) a.push_back(L[i]);
        std::vector<uint32_t> u;
        uniform_sorted(r, U, want - half, u);
        out.resize(a.size() + u.size());
        std::merge(a.begin(), a.end(), u.begin(), u.end(), out.begin());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    });
    for (uint32_t l = 0; l < nt; ++l) s->info.push_back((double)lists[l].size());
    append_lists(*s, lists);
    append_lists(*s, keys);
    for (uint32_t q = 0; q < nq; ++q) add_query(*s, {tgt[q], nt + q});
    return (synth_set *)s;
}

// Config 5: nterms lists with Zipf(1) document frequencies scaled to `total`
// postings over 2^ubits; queries of qmin..qmax terms drawn proportional to
// df^0.5. codecs[l] = ParaPFD below `pfd_below` postings, else SegLRC.
synth_set *synth_serving(uint64_t seed, uint32_t ubits, uint32_t nterms, uint64_t total, uint32_t nq, uint32_t qmin,
                         uint32_t qmax, uint32_t pfd_below, uint32_t threads) {
    Set *s = new Set();
    const uint64_t U = 1ull << ubits;
    double H = 0;
    for (uint32_t r = 1; r <= nterms; ++r) H += 1.0 / r;
    std::vector<uint32_t> df(nterms);
    for (uint32_t r = 0; r < nterms; ++r)
        df[r] = (uint32_t)std::max(1.0, std::min((double)U, std::round((double)total / (H * (r + 1)))));
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(nterms, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 11, l));
        uniform_sorted(r, U, df[l], out);
    });
    append_lists(*s, lists);
    s->codecs.resize(nterms);
    for (uint32_t r = 0; r < nterms; ++r) s->codecs[r] = df[r] < pfd_below ? 0 : 3;
    std::vector<double> cdf(nterms);
    double acc = 0;
    for (uint32_t r = 0; r < nterms; ++r) cdf[r] = (acc += std::sqrt((double)df[r]));
    Rng r(sub_seed(seed, 12, 0));
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = qmin + (uint32_t)r.below(qmax - qmin + 1);
        std::vector<uint32_t> t;
        while (t.size() < k) {
            const uint32_t id = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r.unit() * acc) - cdf.begin());
            const uint32_t c = std::min(id, nterms - 1);
            if (std::find(t.begin(), t.end(), c) == t.end()) t.push_back(c);
        }
        for (uint32_t v : t) s->terms.push_back(v);
        s->toff.push_back((uint32_t)s->terms.size());
    }
    return (synth_set *)s;
}

// Generic: nlists uniform lists with the given lengths over 2^ubits, no queries.
synth_set *synth_uniform_lists(uint64_t seed, uint32_t ubits, uint32_t nlists, const uint32_t *lens, uint32_t threads) {
    Set *s = new Set();
    std::vector<uint32_t> L(lens, lens + nlists);
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(nlists, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 13, l));
        uniform_sorted(r, 1ull << ubits, L[l], out);
    });
    append_lists(*s, lists);
    return (synth_set *)s;
}

// Generic: clustered lists with the given lengths over 2^ubits, no queries.
synth_set *synth_clustered_lists(uint64_t seed, uint32_t ubits, uint32_t nlists, const uint32_t *lens, double run_mean,
                                 double gap_mean, uint32_t threads) {
    Set *s = new Set();
    std::vector<uint32_t> L(lens, lens + nlists);
    std::vector<std::vector<uint32_t>> lists;
    parallel_lists(nlists, threads, lists, [&](uint32_t l, std::vector<uint32_t> &out) {
        Rng r(sub_seed(seed, 14, l));
        clustered_sorted(r, 1ull << ubits, L[l], run_mean, gap_mean, out);
    });
    append_lists(*s, lists);
    return (synth_set *)s;
}

void synth_free(synth_set *s) { delete (Set *)s; }
uint64_t synth_ndocs(const synth_set *s) { return ((const Set *)s)->docs.size(); }
uint32_t synth_nlists(const synth_set *s) { return (uint32_t)((const Set *)s)->loff.size() - 1; }
uint32_t synth_nqueries(const synth_set *s) { return (uint32_t)((const Set *)s)->toff.size() - 1; }
uint64_t synth_nterms(const synth_set *s) { return ((const Set *)s)->terms.size(); }
uint32_t synth_ninfo(const synth_set *s) { return (uint32_t)((const Set *)s)->info.size(); }
const uint32_t *synth_docs(const synth_set *s) { return ((const Set *)s)->docs.data(); }
const uint64_t *synth_loff(const synth_set *s) { return ((const Set *)s)->loff.data(); }
const uint32_t *synth_terms(const synth_set *s) { return ((const Set *)s)->terms.data(); }
const uint32_t *synth_toff(const synth_set *s) { return ((const Set *)s)->toff.data(); }
const uint8_t *synth_codecs(const synth_set *s) {
    const Set *x = (const Set *)s;
    return x->codecs.empty() ? nullptr : x->codecs.data();
}
const double *synth_info(const synth_set *s) { return ((const Set *)s)->info.data(); }
}
