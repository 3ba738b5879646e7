/* CPU ORACLE — test infrastructure only (part of liboracle.so).
 *
 * 1. The seeded synthetic workloads of the benchmark, restated independently
 *    of the library under test so that the CPU reference arm of bench.py
 *    builds its inputs without loading any product code. The rules are the
 *    benchmark's workload definitions: PRNG splitmix64 seeding xoshiro256**,
 *    one sub-seed per list, k distinct uniform values by draw / sort / unique /
 *    top-up rounds, clustered runs (Geometric run lengths and gaps) mixed with
 *    30% uniform docIDs, Zipf-gap lists, Zipf(1) document frequencies and
 *    queries drawn with probability proportional to df^0.5. The test suite
 *    checks these outputs against the product's generator bit for bit.
 * 2. A whole-corpus encoder into the compressed-image layout the CPU path
 *    (or_run_queries_compressed) reads, built from this oracle's own block
 *    encoders (ParaPFor.cpp:56-94 restated in oracle.c).
 * 3. The exact answer of a whole batch (offsets and docIDs) on host threads.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* oracle.c */
int64_t or_encode_parapfd_list(const uint32_t *docs, uint32_t n, uint32_t bs, float frac, uint32_t *words,
                               uint32_t *off, uint32_t *head, uint32_t *median);
int64_t or_encode_newpfd_list(const uint32_t *docs, uint32_t n, uint32_t bs, float frac, uint32_t *words,
                              uint32_t *off, uint32_t *head, uint32_t *median);
int64_t or_encode_parapfd_segs(const uint32_t *docs, uint32_t n, uint32_t nseg, const uint32_t *start, float frac,
                               uint32_t *words, uint32_t *off, uint32_t *head, uint32_t *median);
int64_t or_encode_residual_list(int codec, const uint32_t *docs, uint32_t n, uint32_t nseg, const uint32_t *start,
                                float frac, uint32_t *words, uint32_t *off, uint32_t *head, uint32_t *reg,
                                int32_t *base, uint32_t *listreg);
uint32_t or_hs_partition(const uint32_t *docs, uint32_t n, uint32_t ebs, uint32_t kbits, uint32_t ubits,
                         uint32_t *shift_out, uint32_t *bnd);
uint64_t or_intersect(uint32_t k, const uint32_t *const *lists, const uint64_t *lens, uint32_t *out);

/* ---------------------------------------------------------------------------
 * PRNG
 * ------------------------------------------------------------------------- */
typedef struct {
    uint64_t s[4];
} wl_rng;

static uint64_t wl_splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static void wl_seed(wl_rng *r, uint64_t seed) {
    for (int i = 0; i < 4; ++i) r->s[i] = wl_splitmix(&seed);
}

static inline uint64_t wl_rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t wl_next(wl_rng *r) {
    uint64_t *s = r->s;
    const uint64_t out = wl_rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = wl_rotl(s[3], 45);
    return out;
}

/* uniform in [0, n): the high 64 bits of next() * n */
static uint64_t wl_below(wl_rng *r, uint64_t n) { return (uint64_t)(((unsigned __int128)wl_next(r) * n) >> 64); }

/* uniform double in [0, 1) from the top 53 bits */
static double wl_unit(wl_rng *r) { return (double)(wl_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* Geometric on {1, 2, ...} with the given mean, by inversion */
static uint64_t wl_geom(wl_rng *r, double mean) {
    if (mean <= 1.0) return 1;
    const double p = 1.0 / mean;
    const double u = wl_unit(r);
    return 1 + (uint64_t)floor(log1p(-u) / log1p(-p));
}

static uint64_t wl_sub_seed(uint64_t seed, uint64_t a, uint64_t b) {
    uint64_t x = seed ^ (a * 0x9e3779b97f4a7c15ull) ^ (b * 0xc2b2ae3d27d4eb4full);
    return wl_splitmix(&x);
}

/* log-uniform value in [a, b], truncated */
static uint32_t wl_logu(wl_rng *r, double a, double b) {
    return (uint32_t)exp(log(a) + wl_unit(r) * (log(b) - log(a)));
}

/* ---------------------------------------------------------------------------
 * Growable u32 arrays, sorting and set operations
 * ------------------------------------------------------------------------- */
typedef struct {
    uint32_t *v;
    size_t n, cap;
} wl_vec;

static void wl_reserve(wl_vec *a, size_t c) {
    if (c <= a->cap) return;
    size_t nc = a->cap ? a->cap : 16;
    while (nc < c) nc *= 2;
    a->v = (uint32_t *)realloc(a->v, nc * 4);
    a->cap = nc;
}

static void wl_push(wl_vec *a, uint32_t x) {
    if (a->n == a->cap) wl_reserve(a, a->n + 1);
    a->v[a->n++] = x;
}

static void wl_free(wl_vec *a) {
    free(a->v);
    a->v = NULL;
    a->n = a->cap = 0;
}

/* ascending sort: insertion for short arrays, else LSD radix on 3 x 11 bits */
static void wl_sort(uint32_t *a, size_t n) {
    if (n < 64) {
        for (size_t i = 1; i < n; ++i) {
            uint32_t x = a[i];
            size_t j = i;
            while (j && a[j - 1] > x) {
                a[j] = a[j - 1];
                --j;
            }
            a[j] = x;
        }
        return;
    }
    uint32_t *tmp = (uint32_t *)malloc(n * 4);
    uint32_t *src = a, *dst = tmp;
    for (int pass = 0; pass < 3; ++pass) {
        const int sh = 11 * pass;
        size_t cnt[2049];
        memset(cnt, 0, sizeof cnt);
        for (size_t i = 0; i < n; ++i) ++cnt[((src[i] >> sh) & 2047u) + 1];
        for (int d = 0; d < 2048; ++d) cnt[d + 1] += cnt[d];
        for (size_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 2047u]++] = src[i];
        uint32_t *t = src;
        src = dst;
        dst = t;
    }
    /* three passes: the sorted data is in tmp */
    memcpy(a, src, n * 4);
    free(tmp);
}

/* out = sorted distinct union of two sorted arrays (either may hold duplicates) */
static void wl_union(const uint32_t *a, size_t na, const uint32_t *b, size_t nb, wl_vec *out) {
    wl_vec r = {0};
    wl_reserve(&r, na + nb + 1);
    size_t i = 0, j = 0;
    while (i < na || j < nb) {
        uint32_t x;
        if (j >= nb || (i < na && a[i] <= b[j])) x = a[i++];
        else x = b[j++];
        if (r.n == 0 || r.v[r.n - 1] != x) r.v[r.n++] = x;
    }
    wl_free(out);
    *out = r;
}

/* k distinct values of [0, N), sorted: draw rounds of the missing count, sort,
 * merge, drop repeats, until k are held (the complement when k > N / 2) */
static void wl_uniform_sorted(wl_rng *r, uint64_t N, uint64_t k, wl_vec *out) {
    out->n = 0;
    if (k == 0) return;
    if (k > N) k = N;
    if (k > N / 2) {
        wl_vec comp = {0};
        wl_uniform_sorted(r, N, N - k, &comp);
        wl_reserve(out, k);
        uint64_t j = 0;
        for (uint64_t v = 0; v < N; ++v) {
            if (j < comp.n && comp.v[j] == v) {
                ++j;
                continue;
            }
            out->v[out->n++] = (uint32_t)v;
        }
        wl_free(&comp);
        return;
    }
    wl_vec draw = {0};
    while (out->n < k) {
        const uint64_t need = k - out->n;
        draw.n = 0;
        wl_reserve(&draw, need);
        for (uint64_t i = 0; i < need; ++i) draw.v[draw.n++] = (uint32_t)wl_below(r, N);
        wl_sort(draw.v, draw.n);
        wl_vec merged = {0};
        wl_union(out->v, out->n, draw.v, draw.n, &merged);
        wl_free(out);
        *out = merged;
    }
    wl_free(&draw);
}

/* exactly n docIDs of [0, U): 70% in runs (length ~ Geometric(run_mean), gaps
 * ~ Geometric(g), g shrunk when the runs would not fit the universe), the rest
 * uniform, topped up with uniform values after duplicates are dropped */
static void wl_clustered_sorted(wl_rng *r, uint64_t U, uint64_t n, double run_mean, double gap_mean, wl_vec *out) {
    out->n = 0;
    if (n > U) n = U;
    const uint64_t nrun = (uint64_t)(0.7 * (double)n);
    double runs = (double)nrun / run_mean;
    if (runs < 1.0) runs = 1.0;
    const double fit = (double)U / runs - run_mean;
    double g = fit * 0.9 < gap_mean ? fit * 0.9 : gap_mean;
    if (g < 1.0) g = 1.0;
    wl_vec a = {0};
    wl_reserve(&a, nrun + 1);
    uint64_t pos = wl_below(r, (uint64_t)g > 1 ? (uint64_t)g : 1);
    while (a.n < nrun) {
        const uint64_t len = wl_geom(r, run_mean);
        for (uint64_t i = 0; i < len && a.n < nrun; ++i) {
            wl_push(&a, (uint32_t)(pos % U));
            ++pos;
        }
        pos += wl_geom(r, g);
    }
    wl_vec u = {0};
    wl_uniform_sorted(r, U, n - a.n, &u);
    wl_sort(a.v, a.n);
    wl_union(a.v, a.n, u.v, u.n, out);
    while (out->n < n) {
        wl_vec extra = {0}, m = {0};
        wl_uniform_sorted(r, U, n - out->n, &extra);
        wl_union(out->v, out->n, extra.v, extra.n, &m);
        wl_free(out);
        *out = m;
        wl_free(&extra);
    }
    if (out->n > n) {
        uint8_t *drop = (uint8_t *)calloc(out->n, 1);
        uint64_t extra = out->n - n;
        while (extra) {
            const uint64_t i = wl_below(r, out->n);
            if (!drop[i]) {
                drop[i] = 1;
                --extra;
            }
        }
        size_t w = 0;
        for (size_t i = 0; i < out->n; ++i)
            if (!drop[i]) out->v[w++] = out->v[i];
        out->n = w;
        free(drop);
    }
    wl_free(&a);
    wl_free(&u);
}

/* first index i with cdf[i] > u (n when none) */
static size_t wl_upper_bound(const double *cdf, size_t n, double u) {
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) >> 1;
        if (cdf[mid] <= u) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* gaps ~ Zipf(s) on {1 .. cap} (cdf of the unnormalised weights) from a start
 * below 1024 up to the universe end */
static void wl_zipfgap_sorted(wl_rng *r, uint64_t U, uint32_t cap, const double *cdf, wl_vec *out) {
    out->n = 0;
    uint64_t pos = wl_below(r, 1024);
    while (pos < U) {
        wl_push(out, (uint32_t)pos);
        const double u = wl_unit(r) * cdf[cap - 1];
        uint64_t g = (uint64_t)wl_upper_bound(cdf, cap, u) + 1;
        pos += g < cap ? g : cap;
    }
}

/* ---------------------------------------------------------------------------
 * Workload sets
 * ------------------------------------------------------------------------- */
typedef struct {
    wl_vec docs;      /* concatenated lists */
    uint64_t *loff;   /* nlists + 1 */
    uint32_t nlists;
    wl_vec terms;
    wl_vec toff;      /* nq + 1 */
    uint8_t *codecs;  /* per list, or NULL */
    double *info;
    uint32_t ninfo;
} or_workload;

/* per-list generation on host threads; lists[l] receives list l */
typedef void (*wl_gen_fn)(void *ctx, uint32_t l, wl_vec *out);
typedef struct {
    wl_gen_fn fn;
    void *ctx;
    uint32_t nl;
    wl_vec *lists;
    uint32_t next;
    pthread_mutex_t mu;
} wl_pool;

static void *wl_pool_worker(void *arg) {
    wl_pool *p = (wl_pool *)arg;
    for (;;) {
        pthread_mutex_lock(&p->mu);
        const uint32_t l = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (l >= p->nl) break;
        p->fn(p->ctx, l, &p->lists[l]);
    }
    return NULL;
}

static wl_vec *wl_parallel(uint32_t nl, uint32_t threads, wl_gen_fn fn, void *ctx) {
    wl_pool p;
    p.fn = fn;
    p.ctx = ctx;
    p.nl = nl;
    p.lists = (wl_vec *)calloc(nl ? nl : 1, sizeof(wl_vec));
    p.next = 0;
    pthread_mutex_init(&p.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, wl_pool_worker, &p);
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&p.mu);
    return p.lists;
}

static or_workload *wl_new(void) {
    or_workload *w = (or_workload *)calloc(1, sizeof(or_workload));
    wl_push(&w->toff, 0);
    return w;
}

/* appends lists[0 .. nl) to the set (and frees them) */
static void wl_append(or_workload *w, wl_vec *lists, uint32_t nl) {
    size_t tot = w->docs.n;
    for (uint32_t l = 0; l < nl; ++l) tot += lists[l].n;
    wl_reserve(&w->docs, tot + 1);
    w->loff = (uint64_t *)realloc(w->loff, sizeof(uint64_t) * (w->nlists + nl + 1));
    if (w->nlists == 0) w->loff[0] = 0;
    for (uint32_t l = 0; l < nl; ++l) {
        memcpy(w->docs.v + w->docs.n, lists[l].v, lists[l].n * 4);
        w->docs.n += lists[l].n;
        w->loff[w->nlists + l + 1] = w->docs.n;
        wl_free(&lists[l]);
    }
    w->nlists += nl;
}

static int wl_has(const uint32_t *t, size_t n, uint32_t c) {
    for (size_t i = 0; i < n; ++i)
        if (t[i] == c) return 1;
    return 0;
}

static void wl_end_query(or_workload *w) { wl_push(&w->toff, (uint32_t)w->terms.n); }

/* queries of qmin..qmax distinct terms drawn with probability proportional to
 * sqrt(df) (cdf: running sums of sqrt(df[r]), acc: the total) */
static void wl_df_queries(or_workload *w, wl_rng *r, uint32_t nq, uint32_t qmin, uint32_t qmax, const double *cdf,
                          double acc, uint32_t nterms) {
    uint32_t t[64];
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = qmin + (uint32_t)wl_below(r, qmax - qmin + 1);
        uint32_t n = 0;
        while (n < k) {
            const double u = wl_unit(r) * acc;
            uint32_t id = (uint32_t)wl_upper_bound(cdf, nterms, u);
            const uint32_t c = id < nterms - 1 ? id : nterms - 1;
            if (!wl_has(t, n, c)) t[n++] = c;
        }
        for (uint32_t i = 0; i < n; ++i) wl_push(&w->terms, t[i]);
        wl_end_query(w);
    }
}

typedef struct {
    uint64_t seed, U;
    uint64_t a;  /* sub-seed stream */
    const uint32_t *len;
    uint32_t short_len, long_len;
    double run_mean, gap_mean;
    uint32_t nclust, zcap;
    const double *zcdf;
} wl_ctx;

static void wl_gen_pair(void *c, uint32_t l, wl_vec *out) {
    wl_ctx *x = (wl_ctx *)c;
    wl_rng r;
    wl_seed(&r, wl_sub_seed(x->seed, 1, l));
    wl_uniform_sorted(&r, x->U, (l & 1) ? x->long_len : x->short_len, out);
}

/* config 1: npairs (short, long) uniform lists; query i = lists (2i, 2i+1) */
or_workload *or_wl_pairs(uint64_t seed, uint32_t npairs, uint32_t short_len, uint32_t long_len, uint32_t ubits,
                         uint32_t threads) {
    or_workload *w = wl_new();
    wl_ctx x = {0};
    x.seed = seed;
    x.U = 1ull << ubits;
    x.short_len = short_len;
    x.long_len = long_len;
    wl_vec *lists = wl_parallel(2 * npairs, threads, wl_gen_pair, &x);
    wl_append(w, lists, 2 * npairs);
    free(lists);
    for (uint32_t i = 0; i < npairs; ++i) {
        wl_push(&w->terms, 2 * i);
        wl_push(&w->terms, 2 * i + 1);
        wl_end_query(w);
    }
    return w;
}

static void wl_gen_uniform_len(void *c, uint32_t l, wl_vec *out) {
    wl_ctx *x = (wl_ctx *)c;
    wl_rng r;
    wl_seed(&r, wl_sub_seed(x->seed, x->a, l));
    wl_uniform_sorted(&r, x->U, x->len[l], out);
}

/* config 2: df_r = min(cap, round(cap / r)) over ndocs documents; nq queries
 * of qmin..qmax terms ~ df^0.5 */
or_workload *or_wl_zipf_corpus(uint64_t seed, uint32_t ndocs, uint32_t nterms, uint32_t cap, uint32_t nq,
                               uint32_t qmin, uint32_t qmax, uint32_t threads) {
    or_workload *w = wl_new();
    uint32_t *df = (uint32_t *)malloc(sizeof(uint32_t) * (nterms ? nterms : 1));
    for (uint32_t r = 0; r < nterms; ++r) {
        double v = round((double)cap / (double)(r + 1));
        if (v > (double)cap) v = (double)cap;
        if (v < 1.0) v = 1.0;
        df[r] = (uint32_t)v;
    }
    wl_ctx x = {0};
    x.seed = seed;
    x.U = ndocs;
    x.a = 2;
    x.len = df;
    wl_vec *lists = wl_parallel(nterms, threads, wl_gen_uniform_len, &x);
    wl_append(w, lists, nterms);
    free(lists);
    double *cdf = (double *)malloc(sizeof(double) * (nterms ? nterms : 1));
    double acc = 0;
    for (uint32_t r = 0; r < nterms; ++r) cdf[r] = (acc += sqrt((double)df[r]));
    wl_rng rq;
    wl_seed(&rq, wl_sub_seed(seed, 3, 0));
    wl_df_queries(w, &rq, nq, qmin, qmax, cdf, acc, nterms);
    free(cdf);
    free(df);
    return w;
}

static void wl_gen_clustered(void *c, uint32_t l, wl_vec *out) {
    wl_ctx *x = (wl_ctx *)c;
    wl_rng r;
    wl_seed(&r, wl_sub_seed(x->seed, x->a, l));
    wl_clustered_sorted(&r, x->U, x->len[l], x->run_mean, x->gap_mean, out);
}

/* config 3: npool long clustered lists and one short clustered list per query
 * (list npool + q) ANDed with 1..3 distinct pool lists */
or_workload *or_wl_skewed(uint64_t seed, uint32_t ubits, uint32_t npool, uint32_t long_min, uint32_t long_max,
                          uint32_t nq, uint32_t short_min, uint32_t short_max, double run_mean, double gap_mean,
                          uint32_t threads) {
    or_workload *w = wl_new();
    uint32_t *len = (uint32_t *)malloc(sizeof(uint32_t) * (npool + nq + 1));
    wl_rng lr;
    wl_seed(&lr, wl_sub_seed(seed, 4, 0));
    for (uint32_t i = 0; i < npool; ++i) len[i] = wl_logu(&lr, long_min, long_max);
    for (uint32_t q = 0; q < nq; ++q) len[npool + q] = wl_logu(&lr, short_min, short_max);
    wl_ctx x = {0};
    x.seed = seed;
    x.U = 1ull << ubits;
    x.a = 5;
    x.len = len;
    x.run_mean = run_mean;
    x.gap_mean = gap_mean;
    wl_vec *lists = wl_parallel(npool + nq, threads, wl_gen_clustered, &x);
    wl_append(w, lists, npool + nq);
    free(lists);
    wl_rng r;
    wl_seed(&r, wl_sub_seed(seed, 6, 0));
    uint32_t t[8];
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t k = 1 + (uint32_t)wl_below(&r, 3);
        uint32_t n = 0;
        t[n++] = npool + q;
        while (n < k + 1) {
            const uint32_t c = (uint32_t)wl_below(&r, npool);
            if (!wl_has(t, n, c)) t[n++] = c;
        }
        for (uint32_t i = 0; i < n; ++i) wl_push(&w->terms, t[i]);
        wl_end_query(w);
    }
    free(len);
    return w;
}

static void wl_gen_target(void *c, uint32_t l, wl_vec *out) {
    wl_ctx *x = (wl_ctx *)c;
    wl_rng r;
    wl_seed(&r, wl_sub_seed(x->seed, 8, l));
    if (l < x->nclust) wl_clustered_sorted(&r, x->U, x->len[l], 64.0, 4096.0, out);
    else wl_zipfgap_sorted(&r, x->U, x->zcap, x->zcdf, out);
}

typedef struct {
    uint64_t seed, U;
    const wl_vec *targets;
    const uint32_t *tgt, *klen;
} wl_kctx;

static void wl_gen_keys(void *c, uint32_t q, wl_vec *out) {
    wl_kctx *x = (wl_kctx *)c;
    wl_rng r;
    wl_seed(&r, wl_sub_seed(x->seed, 10, q));
    const wl_vec *L = &x->targets[x->tgt[q]];
    uint64_t want = x->klen[q];
    if (want > L->n + x->U / 2) want = L->n + x->U / 2;
    uint64_t half = want / 2;
    if (half > L->n) half = L->n;
    wl_vec pick = {0}, a = {0}, u = {0};
    wl_uniform_sorted(&r, L->n, half, &pick);
    wl_reserve(&a, pick.n + 1);
    for (size_t i = 0; i < pick.n; ++i) a.v[a.n++] = L->v[pick.v[i]];
    wl_uniform_sorted(&r, x->U, want - half, &u);
    wl_union(a.v, a.n, u.v, u.n, out);
    wl_free(&pick);
    wl_free(&a);
    wl_free(&u);
}

/* config 4: nclust clustered and nzipf Zipf-gap target lists, then nq
 * probe-key lists (half drawn from the target, half uniform); query q =
 * (target, key list nt + q); info = target lengths */
or_workload *or_wl_learned(uint64_t seed, uint32_t ubits, uint32_t nclust, uint32_t nzipf, uint32_t lmin, uint32_t lmax,
                           double zipf_s, uint32_t zipf_cap, uint32_t nq, uint32_t kmin, uint32_t kmax,
                           uint32_t threads) {
    or_workload *w = wl_new();
    const uint64_t U = 1ull << ubits;
    const uint32_t nt = nclust + nzipf;
    uint32_t *len = (uint32_t *)calloc(nt + 1, sizeof(uint32_t));
    wl_rng lr;
    wl_seed(&lr, wl_sub_seed(seed, 7, 0));
    for (uint32_t i = 0; i < nclust; ++i) len[i] = wl_logu(&lr, lmin, lmax);
    double *cdf = (double *)malloc(sizeof(double) * (zipf_cap ? zipf_cap : 1));
    double acc = 0;
    for (uint32_t g = 1; g <= zipf_cap; ++g) cdf[g - 1] = (acc += pow((double)g, -zipf_s));
    wl_ctx x = {0};
    x.seed = seed;
    x.U = U;
    x.len = len;
    x.nclust = nclust;
    x.zcap = zipf_cap;
    x.zcdf = cdf;
    wl_vec *lists = wl_parallel(nt, threads, wl_gen_target, &x);
    uint32_t *tgt = (uint32_t *)malloc(sizeof(uint32_t) * (nq + 1)), *klen = (uint32_t *)malloc(sizeof(uint32_t) * (nq + 1));
    wl_rng qr;
    wl_seed(&qr, wl_sub_seed(seed, 9, 0));
    for (uint32_t q = 0; q < nq; ++q) {
        tgt[q] = (uint32_t)wl_below(&qr, nt);
        klen[q] = wl_logu(&qr, kmin, kmax);
    }
    wl_kctx kx = {seed, U, lists, tgt, klen};
    wl_vec *keys = wl_parallel(nq, threads, wl_gen_keys, &kx);
    w->ninfo = nt;
    w->info = (double *)malloc(sizeof(double) * (nt ? nt : 1));
    for (uint32_t l = 0; l < nt; ++l) w->info[l] = (double)lists[l].n;
    wl_append(w, lists, nt);
    wl_append(w, keys, nq);
    for (uint32_t q = 0; q < nq; ++q) {
        wl_push(&w->terms, tgt[q]);
        wl_push(&w->terms, nt + q);
        wl_end_query(w);
    }
    free(lists);
    free(keys);
    free(tgt);
    free(klen);
    free(cdf);
    free(len);
    return w;
}

/* config 5: Zipf(1) dfs scaled to `total` postings over 2^ubits; codec per
 * list ParaPFD (0) below pfd_below postings, else SegLRC (3); queries of
 * qmin..qmax terms ~ df^0.5 */
or_workload *or_wl_serving(uint64_t seed, uint32_t ubits, uint32_t nterms, uint64_t total, uint32_t nq, uint32_t qmin,
                           uint32_t qmax, uint32_t pfd_below, uint32_t threads) {
    or_workload *w = wl_new();
    const uint64_t U = 1ull << ubits;
    double H = 0;
    for (uint32_t r = 1; r <= nterms; ++r) H += 1.0 / r;
    uint32_t *df = (uint32_t *)malloc(sizeof(uint32_t) * (nterms ? nterms : 1));
    for (uint32_t r = 0; r < nterms; ++r) {
        double v = round((double)total / (H * (r + 1)));
        if (v > (double)U) v = (double)U;
        if (v < 1.0) v = 1.0;
        df[r] = (uint32_t)v;
    }
    wl_ctx x = {0};
    x.seed = seed;
    x.U = U;
    x.a = 11;
    x.len = df;
    wl_vec *lists = wl_parallel(nterms, threads, wl_gen_uniform_len, &x);
    wl_append(w, lists, nterms);
    free(lists);
    w->codecs = (uint8_t *)malloc(nterms ? nterms : 1);
    for (uint32_t r = 0; r < nterms; ++r) w->codecs[r] = df[r] < pfd_below ? 0 : 3;
    double *cdf = (double *)malloc(sizeof(double) * (nterms ? nterms : 1));
    double acc = 0;
    for (uint32_t r = 0; r < nterms; ++r) cdf[r] = (acc += sqrt((double)df[r]));
    wl_rng rq;
    wl_seed(&rq, wl_sub_seed(seed, 12, 0));
    wl_df_queries(w, &rq, nq, qmin, qmax, cdf, acc, nterms);
    free(cdf);
    free(df);
    return w;
}

void or_wl_free(or_workload *w) {
    if (!w) return;
    wl_free(&w->docs);
    wl_free(&w->terms);
    wl_free(&w->toff);
    free(w->loff);
    free(w->codecs);
    free(w->info);
    free(w);
}

uint64_t or_wl_ndocs(const or_workload *w) { return w->docs.n; }
uint32_t or_wl_nlists(const or_workload *w) { return w->nlists; }
uint32_t or_wl_nqueries(const or_workload *w) { return (uint32_t)w->toff.n - 1; }
uint64_t or_wl_nterms(const or_workload *w) { return w->terms.n; }
uint32_t or_wl_ninfo(const or_workload *w) { return w->ninfo; }
const uint32_t *or_wl_docs(const or_workload *w) { return w->docs.v; }
const uint64_t *or_wl_loff(const or_workload *w) { return w->loff; }
const uint32_t *or_wl_terms(const or_workload *w) { return w->terms.v; }
const uint32_t *or_wl_toff(const or_workload *w) { return w->toff.v; }
const uint8_t *or_wl_codecs(const or_workload *w) { return w->codecs; }
const double *or_wl_info(const or_workload *w) { return w->info; }

/* ---------------------------------------------------------------------------
 * Whole-corpus encoder (compressed image of the CPU path)
 *
 * Per list l with codec c[l] (0 ParaPFD, 1 LRC, 2 LRCSeg, 3 SegLRC,
 * 4 HS_SegLRC, 5 HS_ParaPFD, 6 NewPFD): segments of `block` postings, or the
 * reference's hash buckets (HS_SegLRC_Generator.cu:503-594: non-empty buckets
 * for HS_SegLRC, blocks of `block` inside each bucket for HS_ParaPFD). Two
 * calls: or_corpus_plan gives every list's segment count, then
 * or_corpus_encode writes into arrays the caller sized from the plan.
 * ------------------------------------------------------------------------- */
static uint32_t wl_hs_starts(const uint32_t *d, uint32_t n, int codec, uint32_t block, uint32_t bucket,
                             uint32_t kbits, uint32_t ubits, uint32_t *starts) {
    uint32_t nbmax = kbits ? (uint32_t)((uint64_t)d[n - 1] >> (ubits > kbits ? ubits - kbits : 0)) + 2u
                           : 2u * n + 4u;
    uint32_t *bnd = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)nbmax + 2));
    uint32_t sh = 0;
    const uint32_t nb = or_hs_partition(d, n, bucket, kbits, ubits, &sh, bnd);
    uint32_t ns = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t lo = bnd[b], hi = bnd[b + 1];
        const uint32_t step = codec == 5 ? block : (hi > lo ? hi - lo : 1u);
        for (uint32_t k = lo; k < hi; k += step) {
            if (starts) starts[ns] = k;
            ++ns;
        }
    }
    free(bnd);
    return ns;
}

typedef struct {
    const uint32_t *docs;
    const uint64_t *loff;
    const uint8_t *codecs;
    uint32_t nlists, block, bucket, kbits, ubits;
    float frac;
    /* outputs (encode pass) */
    const uint64_t *seg_base;  /* nlists + 1 */
    const uint64_t *word_cap;  /* per list word slot base (upper bounds), nlists + 1 */
    uint32_t *nseg, *nwords;
    uint32_t *words, *head, *rec, *sreg, *lreg;
    int *err;
    uint32_t next;
    pthread_mutex_t mu;
    int plan;
} wl_corpus;

static void *wl_corpus_worker(void *arg) {
    wl_corpus *c = (wl_corpus *)arg;
    for (;;) {
        pthread_mutex_lock(&c->mu);
        const uint32_t l = c->next++;
        pthread_mutex_unlock(&c->mu);
        if (l >= c->nlists) break;
        const uint32_t *d = c->docs + c->loff[l];
        const uint32_t n = (uint32_t)(c->loff[l + 1] - c->loff[l]);
        const int codec = c->codecs[l];
        if (n == 0) {
            c->nseg[l] = 0;
            continue;
        }
        const int hs = codec == 4 || codec == 5;
        if (c->plan) {
            c->nseg[l] = hs ? wl_hs_starts(d, n, codec, c->block, c->bucket, c->kbits, c->ubits, NULL)
                            : (n + c->block - 1) / c->block;
            continue;
        }
        const uint32_t ns = c->nseg[l];
        const uint64_t s0 = c->seg_base[l];
        uint32_t *starts = (uint32_t *)malloc(sizeof(uint32_t) * ns);
        if (hs) wl_hs_starts(d, n, codec, c->block, c->bucket, c->kbits, c->ubits, starts);
        else
            for (uint32_t s = 0; s < ns; ++s) starts[s] = s * c->block;
        uint32_t *off = (uint32_t *)malloc(sizeof(uint32_t) * ns), *aux = (uint32_t *)calloc(ns, 4);
        uint32_t *reg = (uint32_t *)calloc((size_t)ns * 4, 4);
        uint32_t listreg[4] = {0, 0, 0, 0};
        uint32_t *wout = c->words + c->word_cap[l];
        int64_t w;
        if (codec == 6) w = or_encode_newpfd_list(d, n, c->block, c->frac, wout, off, c->head + s0, aux);
        else if (codec == 0) w = or_encode_parapfd_list(d, n, c->block, c->frac, wout, off, c->head + s0, aux);
        else if (codec == 5) w = or_encode_parapfd_segs(d, n, ns, starts, c->frac, wout, off, c->head + s0, aux);
        else
            w = or_encode_residual_list(codec, d, n, ns, starts, c->frac, wout, off, c->head + s0, reg,
                                        (int32_t *)aux, listreg);
        if (w < 0) {
            *c->err = 1;
            w = 0;
        }
        c->nwords[l] = (uint32_t)w;
        for (uint32_t s = 0; s < ns; ++s) {
            uint32_t *r = c->rec + 4 * (s0 + s);
            r[0] = starts[s];
            r[1] = off[s];
            r[2] = aux[s];
            r[3] = (s + 1 < ns ? starts[s + 1] : n) - starts[s];
            memcpy(c->sreg + 4 * (s0 + s), reg + 4 * (size_t)s, 16);
        }
        memcpy(c->lreg + 4 * (size_t)l, listreg, 16);
        free(starts);
        free(off);
        free(aux);
        free(reg);
    }
    return NULL;
}

static void wl_corpus_run(wl_corpus *c, uint32_t threads) {
    c->next = 0;
    pthread_mutex_init(&c->mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (uint32_t t = 0; t < threads; ++t) pthread_create(&th[t], NULL, wl_corpus_worker, c);
    for (uint32_t t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&c->mu);
}

/* segments of every list (nseg[nlists]) */
void or_corpus_plan(const uint32_t *docs, const uint64_t *loff, uint32_t nlists, const uint8_t *codecs,
                    uint32_t block, uint32_t bucket, uint32_t kbits, uint32_t ubits, uint32_t threads,
                    uint32_t *nseg) {
    wl_corpus c;
    memset(&c, 0, sizeof c);
    c.docs = docs;
    c.loff = loff;
    c.codecs = codecs;
    c.nlists = nlists;
    c.block = block;
    c.bucket = bucket;
    c.kbits = kbits;
    c.ubits = ubits;
    c.nseg = nseg;
    c.plan = 1;
    wl_corpus_run(&c, threads);
}

/* Encodes every list: list l's blocks go to words[word_cap[l] ..] (the caller
 * sizes each slot as 3 n + 8 nseg + 8 words), nwords[l] receives its word
 * count; per segment head, rec {start, off, aux, count} and sreg {a, b, L, R};
 * per list lreg (the list-level regression). Returns 0, or -1 when a list is
 * not representable in its format. */
int or_corpus_encode(const uint32_t *docs, const uint64_t *loff, uint32_t nlists, const uint8_t *codecs,
                     uint32_t block, float frac, uint32_t bucket, uint32_t kbits, uint32_t ubits, uint32_t threads,
                     const uint32_t *nseg, const uint64_t *seg_base, const uint64_t *word_cap, uint32_t *words,
                     uint32_t *nwords, uint32_t *head, uint32_t *rec, uint32_t *sreg, uint32_t *lreg) {
    wl_corpus c;
    memset(&c, 0, sizeof c);
    int err = 0;
    c.docs = docs;
    c.loff = loff;
    c.codecs = codecs;
    c.nlists = nlists;
    c.block = block;
    c.frac = frac;
    c.bucket = bucket;
    c.kbits = kbits;
    c.ubits = ubits;
    c.nseg = (uint32_t *)nseg;
    c.seg_base = seg_base;
    c.word_cap = word_cap;
    c.nwords = nwords;
    c.words = words;
    c.head = head;
    c.rec = rec;
    c.sreg = sreg;
    c.lreg = lreg;
    c.err = &err;
    c.plan = 0;
    wl_corpus_run(&c, threads);
    return err ? -1 : 0;
}

/* ---------------------------------------------------------------------------
 * Exact answer of a batch on host threads: pass 1 counts (counts[q]), pass 2
 * writes each query's sorted result at offsets[q] (exclusive prefix of the
 * counts, computed by the caller) into out.
 * ------------------------------------------------------------------------- */
typedef struct {
    const uint32_t *docs;
    const uint64_t *loff;
    const uint32_t *terms;
    const uint64_t *toff;
    uint32_t nq;
    uint64_t *counts;
    const uint64_t *offsets;
    uint32_t *out;
    uint32_t *scratch;
    uint32_t *next;
    pthread_mutex_t *mu;
} wl_ans;

static void *wl_ans_worker(void *arg) {
    wl_ans *a = (wl_ans *)arg;
    const uint32_t *lp[64];
    uint64_t ln[64];
    for (;;) {
        pthread_mutex_lock(a->mu);
        const uint32_t q0 = *a->next;
        *a->next += 64;
        pthread_mutex_unlock(a->mu);
        if (q0 >= a->nq) break;
        const uint32_t q1 = q0 + 64 < a->nq ? q0 + 64 : a->nq;
        for (uint32_t q = q0; q < q1; ++q) {
            uint32_t k = (uint32_t)(a->toff[q + 1] - a->toff[q]);
            if (k > 64) k = 64;
            for (uint32_t t = 0; t < k; ++t) {
                const uint32_t term = a->terms[a->toff[q] + t];
                lp[t] = a->docs + a->loff[term];
                ln[t] = a->loff[term + 1] - a->loff[term];
            }
            uint32_t *dst = a->offsets ? a->out + a->offsets[q] : a->scratch;
            const uint64_t c = k ? or_intersect(k, lp, ln, dst) : 0;
            if (!a->offsets) a->counts[q] = c;
        }
    }
    return NULL;
}

void or_answer_pass(const uint32_t *docs, const uint64_t *loff, const uint32_t *terms, const uint64_t *toff,
                    uint32_t nq, uint32_t threads, uint64_t max_list, uint64_t *counts, const uint64_t *offsets,
                    uint32_t *out) {
    if (threads < 1) threads = 1;
    uint32_t next = 0;
    pthread_mutex_t mu;
    pthread_mutex_init(&mu, NULL);
    wl_ans *jobs = (wl_ans *)malloc(sizeof(wl_ans) * threads);
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * threads);
    for (uint32_t t = 0; t < threads; ++t) {
        wl_ans *j = &jobs[t];
        j->docs = docs;
        j->loff = loff;
        j->terms = terms;
        j->toff = toff;
        j->nq = nq;
        j->counts = counts;
        j->offsets = offsets;
        j->out = out;
        j->scratch = offsets ? NULL : (uint32_t *)malloc((max_list ? max_list : 1) * 4);
        j->next = &next;
        j->mu = &mu;
        pthread_create(&th[t], NULL, wl_ans_worker, j);
    }
    for (uint32_t t = 0; t < threads; ++t) {
        pthread_join(th[t], NULL);
        free(jobs[t].scratch);
    }
    free(jobs);
    free(th);
    pthread_mutex_destroy(&mu);
}
