// Test driver for include/excl_scorer.hpp: reads posting lists, queries and a
// batch's AND results (offsets / docids) from a file, then walks every query
// twice -- with CLucene's leapfrog conjunction over term scorers (restated
// from ConjunctionScorer.cpp:52-104, doc/skipTo contract of Scorer.h) and with
// GpuConjunction over the batch results -- and checks that both visit the
// same documents with the same scores, and that skipTo agrees. Prints "OK".
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

#include "excl_scorer.hpp"

namespace {

// A term scorer over a sorted list: next/doc/skipTo with Scorer's contract,
// score = a fixed function of the docID and the list (tf-idf shaped).
struct ListScorer {
    const std::vector<uint32_t> *d;
    float w;
    long pos = -1;
    bool next() { return ++pos < (long)d->size(); }
    int32_t doc() const { return (int32_t)(*d)[pos]; }
    bool skipTo(int32_t target) {
        do {
            if (!next()) return false;
        } while ((uint32_t)target > (*d)[pos]);
        return true;
    }
    float score() const { return w * (1.0f + (float)((*d)[pos] % 7u)) / (1.0f + (float)((*d)[pos] % 3u)); }
};

// CLucene's ConjunctionScorer, restated: init (every scorer next(), then the
// doNext leapfrog) and next().
struct Leapfrog {
    std::vector<ListScorer *> s;
    bool first = true, more = false;
    int32_t last = -1;
    bool doNext() {
        size_t f = 0;
        ListScorer *lastS = s.back();
        while (more && s[f]->doc() < (last = lastS->doc())) {
            more = s[f]->skipTo(last);
            lastS = s[f];
            f = f == s.size() - 1 ? 0 : f + 1;
        }
        return more;
    }
    bool next() {
        if (first) {
            // init(0): every scorer on its first doc, then sorted by doc (the
            // leapfrog's invariant), then all but the last reversed
            first = false;
            more = true;
            for (ListScorer *x : s)
                if (!(more = x->next())) return false;
            std::stable_sort(s.begin(), s.end(), [](const ListScorer *a, const ListScorer *b) {
                return a->doc() < b->doc();
            });
            doNext();
            const long end = (long)s.size() - 2;
            for (long i = 0; i < (end >> 1); ++i) std::swap(s[i], s[end - i]);
            return more;
        }
        if (more) more = s.back()->next();
        return doNext();
    }
};

uint32_t rd(FILE *f) {
    uint32_t v;
    if (std::fread(&v, 4, 1, f) != 1) std::exit(3);
    return v;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 2) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    const uint32_t nl = rd(f);
    std::vector<std::vector<uint32_t>> lists(nl);
    for (auto &l : lists) {
        l.resize(rd(f));
        for (auto &x : l) x = rd(f);
    }
    const uint32_t nq = rd(f);
    std::vector<std::vector<uint32_t>> qs(nq);
    for (auto &q : qs) {
        q.resize(rd(f));
        for (auto &x : q) x = rd(f);
    }
    std::vector<uint32_t> off(nq + 1);
    for (auto &x : off) x = rd(f);
    std::vector<uint32_t> docs(off[nq]);
    for (auto &x : docs) x = rd(f);
    std::fclose(f);
    excl::BatchResults res(off.data(), docs.data(), nq);
    size_t visited = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        if (qs[q].size() < 2) continue;  // ConjunctionScorer needs two scorers
        const float coord = 1.0f;
        // reference walk
        std::vector<ListScorer> a, b;
        for (uint32_t t : qs[q]) a.push_back({&lists[t], 1.0f + (float)(t % 5u)});
        b = a;
        Leapfrog lf;
        for (auto &x : a) lf.s.push_back(&x);
        std::vector<ListScorer *> bs;
        for (auto &x : b) bs.push_back(&x);
        excl::GpuConjunction<ListScorer> gc(res.query(q), bs, coord);
        for (;;) {
            const bool m1 = lf.next(), m2 = gc.next();
            if (m1 != m2) {
                std::printf("query %u: walks end apart\n", q);
                return 1;
            }
            if (!m1) break;
            // GpuConjunction sums in the given order (exact); the leapfrog in
            // its own order (equal up to float reassociation)
            float s1 = 0.0f;
            for (ListScorer *x : lf.s) s1 += x->score();
            float s2 = 0.0f;
            for (ListScorer *x : bs) s2 += x->score();
            const float g = gc.score();
            if (lf.last != gc.doc() || s2 * coord != g || std::fabs(s1 * coord - g) > 1e-5f * std::fabs(g)) {
                std::printf("query %u: doc %d vs %d\n", q, lf.last, gc.doc());
                return 1;
            }
            ++visited;
        }
        // skipTo: every match reached from its predecessor, and past the end
        excl::QueryCursor c = res.query(q);
        for (size_t i = 0; i < c.cost(); ++i) {
            excl::QueryCursor d = res.query(q);
            const bool ok = d.skipTo((int32_t)docs[off[q] + i]);
            if (!ok || d.udoc() != docs[off[q] + i]) {
                std::printf("query %u: skipTo %zu\n", q, i);
                return 1;
            }
            if (i + 1 < c.cost() && (!d.skipTo((int32_t)docs[off[q] + i]) || d.udoc() != docs[off[q] + i + 1])) {
                std::printf("query %u: skipTo does not move past the current match\n", q);
                return 1;
            }
        }
        excl::QueryCursor e = res.query(q);
        if (c.cost() && e.skipTo((int32_t)(docs[off[q + 1] - 1] + 1)) &&
            docs[off[q + 1] - 1] + 1 > docs[off[q + 1] - 1]) {
            std::printf("query %u: skipTo past the end\n", q);
            return 1;
        }
    }
    std::printf("OK %zu\n", visited);
    return 0;
}
