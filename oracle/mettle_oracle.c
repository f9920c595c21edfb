/*
 * mettle_oracle.c — CPU oracle for the offloaded SQL subset.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline
 * ("port" of the reference path). Nothing in the product links it. The
 * semantics restated here are listed in mettle_oracle.h; each function below
 * names the reference code it follows.
 */
#include "mettle_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef __int128 i128;

int32_t orc_threads(void) {
#ifdef _OPENMP
    return (int32_t)omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------- dates */

/* Civil date -> days since epoch; the same civil algorithm as
 * src/plan/parser.rs:426-449 (parse_date_to_days_since_epoch). */
int32_t orc_days_from_civil(int32_t y, int32_t m, int32_t d) {
    int32_t ay = y - (m <= 2);
    int32_t era = (ay >= 0 ? ay : ay - 399) / 400;
    int32_t yoe = ay - era * 400;
    int32_t mo = m + (m > 2 ? -3 : 9);
    int32_t doy = (153 * mo + 2) / 5 + d - 1;
    int32_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return era * 146097 + doe - 719468;
}

void orc_civil_from_days(int32_t z, int32_t *y, int32_t *m, int32_t *d) {
    z += 719468;
    int32_t era = (z >= 0 ? z : z - 146096) / 146097;
    int32_t doe = z - era * 146097;
    int32_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
    int32_t yy = yoe + era * 400;
    int32_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
    int32_t mp = (5 * doy + 2) / 153;
    int32_t dd = doy - (153 * mp + 2) / 5 + 1;
    int32_t mm = mp + (mp < 10 ? 3 : -9);
    *y = yy + (mm <= 2);
    *m = mm;
    *d = dd;
}

/* -------------------------------------------------------------- filter */

/* One predicate, op codes of kernels.metal:70-173 (compare_*_scalar). */
static inline int cmp_i64(int64_t x, int op, int64_t k) {
    switch (op) {
    case 0: return x == k;
    case 1: return x < k;
    case 2: return x <= k;
    case 3: return x > k;
    case 4: return x >= k;
    default: return 0;
    }
}
static inline int cmp_f64(double x, int op, double k) {
    switch (op) {
    case 0: return x == k;
    case 1: return x < k;
    case 2: return x <= k;
    case 3: return x > k;
    case 4: return x >= k;
    default: return 0;
    }
}
static inline int cmp_f32(float x, int op, float k) {
    switch (op) {
    case 0: return x == k;
    case 1: return x < k;
    case 2: return x <= k;
    case 3: return x > k;
    case 4: return x >= k;
    default: return 0;
    }
}

static inline int row_passes(int32_t np, const void *const *cols, const int32_t *types,
                             const int32_t *ops, const int64_t *il, const double *fl, int64_t i) {
    for (int32_t p = 0; p < np; ++p) {
        int ok;
        switch (types[p]) {
        case ORC_I32: ok = cmp_i64(((const int32_t *)cols[p])[i], ops[p], il[p]); break;
        case ORC_I64: ok = cmp_i64(((const int64_t *)cols[p])[i], ops[p], il[p]); break;
        case ORC_F32: ok = cmp_f32(((const float *)cols[p])[i], ops[p], (float)fl[p]); break;
        case ORC_F64: ok = cmp_f64(((const double *)cols[p])[i], ops[p], fl[p]); break;
        default: ok = 0;
        }
        if (!ok) return 0;
    }
    return 1;
}

/* Conjunctive filter to an ascending selection vector: the semantics of the
 * reference's compare_* -> and_masks -> filter_to_indices chain
 * (kernels.metal:70-173, 673, 684; gather_ops.rs:23-159), with the row order
 * made deterministic. Two passes: per-chunk counts, prefix, write. */
int64_t orc_filter(int32_t np, const void *const *cols, const int32_t *types, const int32_t *ops,
                   const int64_t *il, const double *fl, int64_t n, int64_t *out) {
    int nt = orc_threads();
    int64_t *counts = (int64_t *)calloc((size_t)nt + 1, sizeof(int64_t));
    int64_t chunk = (n + nt - 1) / (nt > 0 ? nt : 1);
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        int64_t lo = (int64_t)t * chunk, hi = lo + chunk;
        if (hi > n) hi = n;
        int64_t c = 0;
        for (int64_t i = lo; i < hi; ++i) c += row_passes(np, cols, types, ops, il, fl, i);
        counts[t + 1] = c;
#pragma omp barrier
#pragma omp single
        for (int k = 0; k < nt; ++k) counts[k + 1] += counts[k];
        int64_t o = counts[t];
        for (int64_t i = lo; i < hi; ++i)
            if (row_passes(np, cols, types, ops, il, fl, i)) out[o++] = i;
    }
    int64_t total = counts[nt];
    free(counts);
    return total;
}

/* ---------------------------------------------------------- projections */

int32_t orc_gather_i32(const int32_t *col, const int64_t *rows, int64_t s, int32_t *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s; ++i) out[i] = col[rows[i]];
    return 0;
}
int32_t orc_gather_i64(const int64_t *col, const int64_t *rows, int64_t s, int64_t *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s; ++i) out[i] = col[rows[i]];
    return 0;
}
int32_t orc_gather_f32(const float *col, const int64_t *rows, int64_t s, float *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s; ++i) out[i] = col[rows[i]];
    return 0;
}
/* INTEGER * INTEGER -> INTEGER with DuckDB's overflow error. */
int32_t orc_gather_i32_mul(const int32_t *col, const int64_t *rows, int64_t s, int32_t k, int32_t *out) {
    int32_t ovf = 0;
#pragma omp parallel for schedule(static) reduction(| : ovf)
    for (int64_t i = 0; i < s; ++i) {
        int64_t r = (int64_t)col[rows[i]] * (int64_t)k;
        if (r > INT32_MAX || r < INT32_MIN) ovf |= 1;
        out[i] = (int32_t)r;
    }
    return ovf;
}
int32_t orc_gather_i32_add(const int32_t *col, const int64_t *rows, int64_t s, int32_t k, int32_t *out) {
    int32_t ovf = 0;
#pragma omp parallel for schedule(static) reduction(| : ovf)
    for (int64_t i = 0; i < s; ++i) {
        int64_t r = (int64_t)col[rows[i]] + (int64_t)k;
        if (r > INT32_MAX || r < INT32_MIN) ovf |= 1;
        out[i] = (int32_t)r;
    }
    return ovf;
}
int32_t orc_gather_i64_add(const int64_t *col, const int64_t *rows, int64_t s, int64_t k, int64_t *out) {
    int32_t ovf = 0;
#pragma omp parallel for schedule(static) reduction(| : ovf)
    for (int64_t i = 0; i < s; ++i) {
        int64_t r;
        if (__builtin_add_overflow(col[rows[i]], k, &r)) ovf |= 1;
        out[i] = r;
    }
    return ovf;
}
int32_t orc_gather_i64_mul(const int64_t *col, const int64_t *rows, int64_t s, int64_t k, int64_t *out) {
    int32_t ovf = 0;
#pragma omp parallel for schedule(static) reduction(| : ovf)
    for (int64_t i = 0; i < s; ++i) {
        int64_t r;
        if (__builtin_mul_overflow(col[rows[i]], k, &r)) ovf |= 1;
        out[i] = r;
    }
    return ovf;
}
/* FLOAT * k -> FLOAT (binary32 product). */
int32_t orc_gather_f32_mul(const float *col, const int64_t *rows, int64_t s, float k, float *out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s; ++i) {
        volatile float x = col[rows[i]];
        out[i] = x * k;
    }
    return 0;
}

/* ----------------------------------------------------------------- sort */

/* Stable LSD radix sort of (key, row) by a biased unsigned key. */
static void radix_sort_u64_rows(uint64_t *keys, int64_t *rows, int64_t s, int key_bytes) {
    uint64_t *k2 = (uint64_t *)malloc((size_t)(s ? s : 1) * sizeof(uint64_t));
    int64_t *r2 = (int64_t *)malloc((size_t)(s ? s : 1) * sizeof(int64_t));
    for (int pass = 0; pass < key_bytes * 8 / 16; ++pass) {
        int shift = pass * 16;
        int64_t *hist = (int64_t *)calloc(65536, sizeof(int64_t));
        for (int64_t i = 0; i < s; ++i) hist[(keys[i] >> shift) & 0xFFFF]++;
        int64_t acc = 0;
        for (int b = 0; b < 65536; ++b) {
            int64_t c = hist[b];
            hist[b] = acc;
            acc += c;
        }
        for (int64_t i = 0; i < s; ++i) {
            int64_t d = hist[(keys[i] >> shift) & 0xFFFF]++;
            k2[d] = keys[i];
            r2[d] = rows[i];
        }
        memcpy(keys, k2, (size_t)s * sizeof(uint64_t));
        memcpy(rows, r2, (size_t)s * sizeof(int64_t));
        free(hist);
    }
    free(k2);
    free(r2);
}

/* ORDER BY key [DESC] over a selection vector; ties keep row order. The
 * reference sorts the materialized batch on the CPU (src/plan/helpers.rs:627-667). */
void orc_sort_rows_i32(const int32_t *key, int64_t *rows, int64_t s, int32_t desc) {
    uint64_t *k = (uint64_t *)malloc((size_t)(s ? s : 1) * sizeof(uint64_t));
    for (int64_t i = 0; i < s; ++i) {
        uint32_t u = (uint32_t)key[rows[i]] ^ 0x80000000u;
        k[i] = desc ? (uint64_t)(~u) : (uint64_t)u;
    }
    radix_sort_u64_rows(k, rows, s, 4);
    free(k);
}
void orc_sort_rows_i64(const int64_t *key, int64_t *rows, int64_t s, int32_t desc) {
    uint64_t *k = (uint64_t *)malloc((size_t)(s ? s : 1) * sizeof(uint64_t));
    for (int64_t i = 0; i < s; ++i) {
        uint64_t u = (uint64_t)key[rows[i]] ^ 0x8000000000000000ull;
        k[i] = desc ? ~u : u;
    }
    radix_sort_u64_rows(k, rows, s, 8);
    free(k);
}

/* ------------------------------------------------------------- group-by */

double orc_avg_i128(uint64_t lo, int64_t hi, int64_t count) {
    i128 s = ((i128)hi << 64) | (i128)lo;
    long double ls;
    /* Hugeint -> long double: exact below 2^64 in magnitude. */
    if (s >= 0) {
        ls = (long double)(uint64_t)(s >> 64) * 18446744073709551616.0L + (long double)(uint64_t)s;
    } else {
        i128 m = -s;
        ls = -((long double)(uint64_t)(m >> 64) * 18446744073709551616.0L + (long double)(uint64_t)m);
    }
    long double q = ls / (long double)count;
    return (double)q;
}

typedef struct {
    int64_t key;
    int64_t count;
    i128 sumv;
    int64_t minv, maxv;
    long double sumf;
    float minf, maxf;
    int32_t used;
} c3_group;

static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

typedef struct {
    c3_group *slots;
    int64_t cap, used;
} c3_table;

static void c3_grow(c3_table *t) {
    int64_t ncap = t->cap ? t->cap * 2 : 1024;
    c3_group *ns = (c3_group *)calloc((size_t)ncap, sizeof(c3_group));
    for (int64_t i = 0; i < t->cap; ++i) {
        if (!t->slots[i].used) continue;
        uint64_t h = mix64((uint64_t)t->slots[i].key) & (uint64_t)(ncap - 1);
        while (ns[h].used) h = (h + 1) & (uint64_t)(ncap - 1);
        ns[h] = t->slots[i];
    }
    free(t->slots);
    t->slots = ns;
    t->cap = ncap;
}

static inline c3_group *c3_find(c3_table *t, int64_t key) {
    if (2 * (t->used + 1) > t->cap) c3_grow(t);
    uint64_t h = mix64((uint64_t)key) & (uint64_t)(t->cap - 1);
    for (;;) {
        c3_group *g = &t->slots[h];
        if (!g->used) {
            g->used = 1;
            g->key = key;
            g->minv = INT64_MAX;
            g->maxv = INT64_MIN;
            g->minf = INFINITY;
            g->maxf = -INFINITY;
            t->used++;
            return g;
        }
        if (g->key == key) return g;
        h = (h + 1) & (uint64_t)(t->cap - 1);
    }
}

/* ORDER BY SUM(v) DESC, k ASC. */
static int c3_before(const c3_group *a, const c3_group *b) {
    if (a->sumv != b->sumv) return a->sumv > b->sumv;
    return a->key < b->key;
}
static int c3_cmp_rank(const void *x, const void *y) {
    const c3_group *a = (const c3_group *)x, *b = (const c3_group *)y;
    if (c3_before(a, b)) return -1;
    if (c3_before(b, a)) return 1;
    return 0;
}
static int c3_cmp_key(const void *x, const void *y) {
    const c3_group *a = (const c3_group *)x, *b = (const c3_group *)y;
    return (a->key > b->key) - (a->key < b->key);
}

/* Keep the best `k` groups of `src` in heap order (worst at index 0). */
static void heap_sift(c3_group *h, int64_t n, int64_t i) {
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, w = i;
        /* worst-first heap: parent is "after" children in rank order */
        if (l < n && c3_before(&h[w], &h[l])) w = l;
        if (r < n && c3_before(&h[w], &h[r])) w = r;
        if (w == i) return;
        c3_group t = h[i];
        h[i] = h[w];
        h[w] = t;
        i = w;
    }
}

/* Grouped aggregate of config 3. The reference's GPU path cannot take a
 * BIGINT key (src/plan/helpers.rs:136) and runs the CPU HashMap aggregate
 * of src/plan/aggregate.rs:88-236 in f64; this restates the exact DuckDB
 * result types instead. Hash-partitioned: each thread owns a key partition. */
int64_t orc_groupby_c3(const int64_t *k, const int64_t *v, const float *f, int64_t n, int64_t limit,
                       int64_t *n_groups, int64_t *o_key, uint64_t *o_sumv_lo, int64_t *o_sumv_hi,
                       int64_t *o_count, int64_t *o_minv, int64_t *o_maxv, double *o_avgv,
                       double *o_sumf, float *o_minf, float *o_maxf, double *o_avgf) {
    int nt = orc_threads();
    int P = 1;
    while (P < 4 * nt) P <<= 1;
    int pbits = 0;
    while ((1 << pbits) < P) pbits++;
    /* partition row ids by key hash: count, prefix, scatter (stable) */
    int64_t chunk = (n + nt - 1) / nt;
    int64_t *cnt = (int64_t *)calloc((size_t)nt * P, sizeof(int64_t));
    uint32_t *order = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    int64_t *pstart = (int64_t *)calloc((size_t)P + 1, sizeof(int64_t));
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        int64_t lo = (int64_t)t * chunk, hi = lo + chunk;
        if (hi > n) hi = n;
        int64_t *c = cnt + (size_t)t * P;
        for (int64_t i = lo; i < hi; ++i) c[mix64((uint64_t)k[i]) >> (64 - pbits)]++;
#pragma omp barrier
#pragma omp single
        {
            int64_t acc = 0;
            for (int p = 0; p < P; ++p) {
                pstart[p] = acc;
                for (int q = 0; q < nt; ++q) {
                    int64_t x = cnt[(size_t)q * P + p];
                    cnt[(size_t)q * P + p] = acc;
                    acc += x;
                }
            }
            pstart[P] = acc;
        }
        for (int64_t i = lo; i < hi; ++i) order[c[mix64((uint64_t)k[i]) >> (64 - pbits)]++] = (uint32_t)i;
    }
    free(cnt);
    c3_table *tabs = (c3_table *)calloc((size_t)P, sizeof(c3_table));
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int p = 0; p < P; ++p) {
        c3_table *t = &tabs[p];
        for (int64_t j = pstart[p]; j < pstart[p + 1]; ++j) {
            int64_t i = order[j];
            c3_group *g = c3_find(t, k[i]);
            g->count++;
            g->sumv += (i128)v[i];
            if (v[i] < g->minv) g->minv = v[i];
            if (v[i] > g->maxv) g->maxv = v[i];
            g->sumf += (long double)f[i];
            if (f[i] < g->minf) g->minf = f[i];
            if (f[i] > g->maxf) g->maxf = f[i];
        }
    }
    free(order);
    free(pstart);
    int64_t total = 0;
    for (int p = 0; p < P; ++p) total += tabs[p].used;
    *n_groups = total;

    c3_group *sel;
    int64_t nsel;
    if (limit < 0) {
        sel = (c3_group *)malloc((size_t)(total ? total : 1) * sizeof(c3_group));
        nsel = 0;
        for (int p = 0; p < P; ++p)
            for (int64_t i = 0; i < tabs[p].cap; ++i)
                if (tabs[p].slots[i].used) sel[nsel++] = tabs[p].slots[i];
        qsort(sel, (size_t)nsel, sizeof(c3_group), c3_cmp_key);
    } else {
        int64_t K = limit < total ? limit : total;
        /* per-partition bounded heaps, then a final merge */
        c3_group *heaps = (c3_group *)malloc((size_t)P * (size_t)(K ? K : 1) * sizeof(c3_group));
        int64_t *hn = (int64_t *)calloc((size_t)P, sizeof(int64_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int p = 0; p < P; ++p) {
            c3_group *h = heaps + (size_t)p * (size_t)(K ? K : 1);
            int64_t m = 0;
            if (K == 0) continue;
            for (int64_t i = 0; i < tabs[p].cap; ++i) {
                const c3_group *g = &tabs[p].slots[i];
                if (!g->used) continue;
                if (m < K) {
                    h[m++] = *g;
                    if (m == K)
                        for (int64_t q = K / 2; q >= 0; --q) heap_sift(h, K, q);
                } else if (c3_before(g, &h[0])) {
                    h[0] = *g;
                    heap_sift(h, K, 0);
                }
            }
            hn[p] = m;
        }
        int64_t all = 0;
        for (int p = 0; p < P; ++p) all += hn[p];
        sel = (c3_group *)malloc((size_t)(all ? all : 1) * sizeof(c3_group));
        nsel = 0;
        for (int p = 0; p < P; ++p)
            for (int64_t i = 0; i < hn[p]; ++i) sel[nsel++] = heaps[(size_t)p * (size_t)(K ? K : 1) + i];
        free(heaps);
        free(hn);
        qsort(sel, (size_t)nsel, sizeof(c3_group), c3_cmp_rank);
        if (nsel > K) nsel = K;
    }
    for (int64_t i = 0; i < nsel; ++i) {
        const c3_group *g = &sel[i];
        o_key[i] = g->key;
        o_sumv_lo[i] = (uint64_t)g->sumv;
        o_sumv_hi[i] = (int64_t)(g->sumv >> 64);
        o_count[i] = g->count;
        o_minv[i] = g->minv;
        o_maxv[i] = g->maxv;
        o_avgv[i] = orc_avg_i128((uint64_t)g->sumv, (int64_t)(g->sumv >> 64), g->count);
        o_sumf[i] = (double)g->sumf;
        o_minf[i] = g->minf;
        o_maxf[i] = g->maxf;
        o_avgf[i] = (double)(g->sumf / (long double)g->count);
    }
    free(sel);
    for (int p = 0; p < P; ++p) free(tabs[p].slots);
    free(tabs);
    return nsel;
}

/* ------------------------------------------------------------------ Q3 */

/* int32 key -> int32 value open-addressing map (value -1 = absent). */
typedef struct {
    int32_t *keys;
    int32_t *vals;
    uint8_t *used;
    int64_t cap;
} i32map;

static void i32map_init(i32map *m, int64_t n) {
    int64_t cap = 16;
    while (cap < 2 * n) cap <<= 1;
    m->cap = cap;
    m->keys = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    m->vals = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    m->used = (uint8_t *)calloc((size_t)cap, 1);
}
static void i32map_free(i32map *m) {
    free(m->keys);
    free(m->vals);
    free(m->used);
}
static inline uint64_t h32(int32_t k) { return mix64((uint64_t)(uint32_t)k); }
/* Insert; returns 0 if the key was already present (duplicate build key). */
static int i32map_put(i32map *m, int32_t k, int32_t v) {
    uint64_t h = h32(k) & (uint64_t)(m->cap - 1);
    while (m->used[h]) {
        if (m->keys[h] == k) return 0;
        h = (h + 1) & (uint64_t)(m->cap - 1);
    }
    m->used[h] = 1;
    m->keys[h] = k;
    m->vals[h] = v;
    return 1;
}
static inline int32_t i32map_get(const i32map *m, int32_t k) {
    uint64_t h = h32(k) & (uint64_t)(m->cap - 1);
    while (m->used[h]) {
        if (m->keys[h] == k) return m->vals[h];
        h = (h + 1) & (uint64_t)(m->cap - 1);
    }
    return -1;
}

typedef struct {
    int32_t key, date, prio;
    int32_t ord_row;
    i128 rev;
} q3_group;

/* ORDER BY revenue DESC, o_orderdate ASC, then l_orderkey ASC. */
static int q3_before(const q3_group *a, const q3_group *b) {
    if (a->rev != b->rev) return a->rev > b->rev;
    if (a->date != b->date) return a->date < b->date;
    return a->key < b->key;
}
static int q3_cmp(const void *x, const void *y) {
    const q3_group *a = (const q3_group *)x, *b = (const q3_group *)y;
    if (q3_before(a, b)) return -1;
    if (q3_before(b, a)) return 1;
    return 0;
}

/* Config-4 pipeline. The reference runs it as filter -> hash/dense join per
 * step -> compact -> reindex -> revenue -> group-by-representative-row ->
 * top-K (src/plan/executor/fast_path/,  kernels.metal:996-1118) in f32;
 * here the same relational result with exact scale-4 revenue. */
int64_t orc_q3(const int32_t *c_custkey, const int32_t *c_segment, int64_t n_cust,
               const int32_t *o_orderkey, const int32_t *o_custkey, const int32_t *o_orderdate,
               const int32_t *o_shippriority, int64_t n_ord, const int32_t *l_orderkey,
               const int64_t *l_price, const int64_t *l_discount, const int32_t *l_shipdate,
               int64_t n_li, int32_t segment, int32_t date, int64_t limit, int64_t *n_groups,
               int32_t *o_key, uint64_t *o_rev_lo, int64_t *o_rev_hi, int32_t *o_date, int32_t *o_prio) {
    int nt = orc_threads();
    /* customer: qualifying custkeys */
    i32map cust;
    i32map_init(&cust, n_cust);
    for (int64_t i = 0; i < n_cust; ++i)
        if (c_segment[i] == segment) i32map_put(&cust, c_custkey[i], (int32_t)i);
    /* orders: qualifying orderkey -> dense group slot */
    int32_t *slot_of_row = (int32_t *)malloc((size_t)(n_ord ? n_ord : 1) * sizeof(int32_t));
    int64_t n_q = 0;
    for (int64_t i = 0; i < n_ord; ++i) {
        slot_of_row[i] = -1;
        if (o_orderdate[i] < date && i32map_get(&cust, o_custkey[i]) >= 0) slot_of_row[i] = (int32_t)n_q++;
    }
    i32map ord;
    i32map_init(&ord, n_q);
    q3_group *groups = (q3_group *)calloc((size_t)(n_q ? n_q : 1), sizeof(q3_group));
    for (int64_t i = 0; i < n_ord; ++i) {
        int32_t s = slot_of_row[i];
        if (s < 0) continue;
        i32map_put(&ord, o_orderkey[i], s);
        groups[s].key = o_orderkey[i];
        groups[s].date = o_orderdate[i];
        groups[s].prio = o_shippriority ? o_shippriority[i] : 0;
        groups[s].ord_row = (int32_t)i;
    }
    free(slot_of_row);
    /* lineitem: probe + exact revenue; per-thread partial sums, then merge */
    uint8_t *hit = (uint8_t *)calloc((size_t)(n_q ? n_q : 1), 1);
    i128 **part = (i128 **)calloc((size_t)nt, sizeof(i128 *));
    int64_t chunk = (n_li + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        int64_t lo = (int64_t)t * chunk, hi = lo + chunk;
        if (hi > n_li) hi = n_li;
        i128 *acc = NULL;
        for (int64_t i = lo; i < hi; ++i) {
            if (!(l_shipdate[i] > date)) continue;
            int32_t s = i32map_get(&ord, l_orderkey[i]);
            if (s < 0) continue;
            if (!acc) acc = (i128 *)calloc((size_t)(n_q ? n_q : 1), sizeof(i128));
            acc[s] += (i128)l_price[i] * (i128)(100 - l_discount[i]);
            hit[s] = 1;
        }
        part[t] = acc;
    }
    for (int t = 0; t < nt; ++t) {
        if (!part[t]) continue;
        for (int64_t s = 0; s < n_q; ++s) groups[s].rev += part[t][s];
        free(part[t]);
    }
    free(part);
    /* live groups only: a group exists when at least one lineitem joined */
    int64_t live = 0;
    for (int64_t s = 0; s < n_q; ++s)
        if (hit[s]) groups[live++] = groups[s];
    free(hit);
    *n_groups = live;
    qsort(groups, (size_t)live, sizeof(q3_group), q3_cmp);
    int64_t m = (limit >= 0 && limit < live) ? limit : live;
    for (int64_t i = 0; i < m; ++i) {
        o_key[i] = groups[i].key;
        o_rev_lo[i] = (uint64_t)groups[i].rev;
        o_rev_hi[i] = (int64_t)(groups[i].rev >> 64);
        o_date[i] = groups[i].date;
        o_prio[i] = groups[i].prio;
    }
    free(groups);
    i32map_free(&cust);
    i32map_free(&ord);
    return m;
}
