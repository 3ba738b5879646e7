/* C++ scorer adapters over a finished batch of GPU AND queries.
 *
 * The reference ranks a conjunctive query with CLucene's ConjunctionScorer
 * (src/core/CLucene/search/ConjunctionScorer.cpp:52-104): it leapfrogs the
 * term scorers with skipTo until they agree on a document, then sums their
 * scores times the coordination factor. With this library the intersection is
 * already done on the GPU: a batch's offsets[nq + 1] / docids (from excl_wait
 * or excl_submit_into) hold every query's matching docIDs in ascending order.
 * These classes walk those results with the Scorer protocol (next / doc /
 * skipTo / score), so a host keeps its term scorers for ranking and drops the
 * leapfrogging:
 *
 *   BatchResults       one batch's output; query(q) gives a cursor
 *   QueryCursor        next / doc / skipTo / cost over one query's docIDs
 *   GpuConjunction<S>  a cursor plus the query's term scorers (any type with
 *                      bool skipTo(int32_t) and float score()): each
 *                      candidate is a document of every term's list, so every
 *                      term scorer lands on it exactly, and score() is
 *                      ConjunctionScorer::score() (sum times coord)
 *
 * Header only, no CUDA types; a CLucene Scorer subclass binds it by
 * forwarding next/skipTo/doc/score to a GpuConjunction. docIDs above INT32_MAX are not
 * representable in CLucene's int32_t doc(); doc() returns them cast, and
 * skipTo compares as unsigned.
 */
#ifndef EXCL_SCORER_HPP
#define EXCL_SCORER_HPP

#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <utility>
#include <vector>

namespace excl {

// Cursor over one query's matching docIDs (ascending). Before the first
// next() / skipTo() it is unpositioned; after the last it is exhausted.
class QueryCursor {
  public:
    QueryCursor() = default;
    QueryCursor(const uint32_t *docids, size_t n) : d_(docids), n_(n) {}

    // Advance to the next match (Scorer::next, ConjunctionScorer.cpp:52-59).
    bool next() {
        pos_ = pos_ == kUnset ? 0 : std::min(pos_ + 1, n_);
        return pos_ < n_;
    }
    // The current match; undefined unless the last next()/skipTo() returned true.
    int32_t doc() const { return (int32_t)d_[pos_]; }
    uint32_t udoc() const { return d_[pos_]; }
    // Scorer::skipTo (ConjunctionScorer.cpp:73-79), with CLucene's contract:
    // as if `do { if (!next()) return false; } while (target > doc());`, so it
    // always moves past the current match. Galloping, then binary search.
    bool skipTo(int32_t target) { return skip_to_unsigned((uint32_t)target); }
    bool skip_to_unsigned(uint32_t target) {
        size_t lo = pos_ == kUnset ? 0 : std::min(pos_ + 1, n_);
        if (lo >= n_ || d_[lo] >= target) {
            pos_ = lo;
            return pos_ < n_;
        }
        size_t step = 1, hi = lo + 1;
        while (hi < n_ && d_[hi] < target) {
            lo = hi;
            step <<= 1;
            hi = lo + step;
        }
        hi = std::min(hi, n_);
        pos_ = (size_t)(std::lower_bound(d_ + lo, d_ + hi, target) - d_);
        return pos_ < n_;
    }
    // Number of matches (what a WAND / max-score driver orders cursors by).
    size_t cost() const { return n_; }
    bool exhausted() const { return pos_ != kUnset && pos_ >= n_; }

  private:
    static constexpr size_t kUnset = (size_t)-1;
    const uint32_t *d_ = nullptr;
    size_t n_ = 0;
    size_t pos_ = kUnset;
};

// One batch's output: offsets[nq + 1] (exclusive prefix) and the concatenated
// docIDs. The arrays are borrowed and must outlive the cursors.
class BatchResults {
  public:
    BatchResults(const uint32_t *offsets, const uint32_t *docids, uint32_t nq)
        : off_(offsets), docs_(docids), nq_(nq) {}
    uint32_t queries() const { return nq_; }
    size_t count(uint32_t q) const { return off_[q + 1] - off_[q]; }
    QueryCursor query(uint32_t q) const { return QueryCursor(docs_ + off_[q], count(q)); }

  private:
    const uint32_t *off_;
    const uint32_t *docs_;
    uint32_t nq_;
};

// A query's GPU matches plus its term scorers. Scorer: any type with
// bool skipTo(int32_t) and float score() (CLucene's TermScorer, or a wrapper).
// coord is Similarity::coord(terms, terms) as ConjunctionScorer computes it
// (ConjunctionScorer.cpp:27).
template <class Scorer>
class GpuConjunction {
  public:
    GpuConjunction(QueryCursor matches, std::vector<Scorer *> scorers, float coord)
        : m_(matches), s_(std::move(scorers)), coord_(coord) {}

    bool next() { return m_.next() && align(); }
    int32_t doc() const { return m_.doc(); }
    bool skipTo(int32_t target) { return m_.skipTo(target) && align(); }
    // ConjunctionScorer::score (:122-128): the term scorers' sum times coord,
    // summed in the order of `scorers` (ConjunctionScorer sums in its own
    // order, fixed by a qsort of equal docs at init, so the last bit of a
    // score can differ from CLucene's).
    float score() {
        float sum = 0.0f;
        for (Scorer *s : s_) sum += s->score();
        return sum * coord_;
    }
    size_t cost() const { return m_.cost(); }

  private:
    // every term's list holds the match, so each scorer lands on it exactly
    // (each is behind it: matches ascend, and a scorer only moves to matches)
    bool align() {
        for (Scorer *s : s_)
            if (!s->skipTo(m_.doc())) return false;
        return true;
    }
    QueryCursor m_;
    std::vector<Scorer *> s_;
    float coord_;
};

}  // namespace excl

#endif  // EXCL_SCORER_HPP
