/*
 * CPU restatement of the MNMGDatalog fixpoint programs -- TEST INFRASTRUCTURE.
 * (Declarations and contract in dl_oracle.h.)
 *
 * The restatement keeps the reference's relational steps one for one so the
 * per-iteration delta counts are comparable: hash join (a multimap keyed by
 * the first column, common/hash_table.cu + common/join.cu), thrust
 * sort(set_cmp)+unique(is_equal), set_difference(set_cmp), merge(set_cmp),
 * unique(is_equal_key). Tuples are held as 64-bit words whose unsigned order
 * equals set_cmp order (common/utils.cu:114-124): the signed key is biased by
 * 2^31 into the high half and the signed value into the low half.
 */
#include "dl_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;

static inline u64 pk(int32_t k, int32_t v) {
    return ((u64) ((uint32_t) k ^ 0x80000000u) << 32) | (u64) ((uint32_t) v ^ 0x80000000u);
}
static inline int32_t pk_key(u64 p) { return (int32_t) ((uint32_t) (p >> 32) ^ 0x80000000u); }
static inline int32_t pk_val(u64 p) { return (int32_t) ((uint32_t) p ^ 0x80000000u); }
static inline u64 pk_swap(u64 p) { return (p << 32) | (p >> 32); }

static void *xmalloc(size_t n) {
    void *p = malloc(n ? n : 1);
    if (!p) { fprintf(stderr, "oracle: out of host memory (%zu bytes)\n", n); abort(); }
    return p;
}

void oracle_free(void *p) { free(p); }

/* Sorting helper for the oracle: LSD radix over 16-bit digits, skipping
 * digits on which every key agrees. Produces set_cmp order. */
static void sort_keys(u64 *a, int64_t n) {
    if (n < 2) return;
    u64 orv = 0, andv = ~(u64) 0;
    for (int64_t i = 0; i < n; ++i) { orv |= a[i]; andv &= a[i]; }
    u64 diff = orv ^ andv;
    u64 *tmp = (u64 *) xmalloc((size_t) n * 8);
    int64_t *cnt = (int64_t *) xmalloc(65536 * sizeof(int64_t));
    u64 *src = a, *dst = tmp;
    for (int sh = 0; sh < 64; sh += 16) {
        if (((diff >> sh) & 0xFFFF) == 0) continue;
        memset(cnt, 0, 65536 * sizeof(int64_t));
        for (int64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xFFFF]++;
        int64_t s = 0;
        for (int d = 0; d < 65536; ++d) { int64_t c = cnt[d]; cnt[d] = s; s += c; }
        for (int64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        u64 *t = src; src = dst; dst = t;
    }
    if (src != a) memcpy(a, src, (size_t) n * 8);
    free(tmp);
    free(cnt);
}

/* thrust::unique(is_equal) on sorted input (e.g. tc.cu:251-253). */
static int64_t unique_keys(u64 *a, int64_t n) {
    if (n == 0) return 0;
    int64_t k = 1;
    for (int64_t i = 1; i < n; ++i)
        if (a[i] != a[k - 1]) a[k++] = a[i];
    return k;
}

static int64_t sort_unique(u64 *a, int64_t n) {
    sort_keys(a, n);
    return unique_keys(a, n);
}

/* thrust::unique(is_equal_key): keeps the first tuple of every key run
 * (wcc.cu:219-221, 320-323). */
static int64_t unique_by_key(u64 *a, int64_t n) {
    if (n == 0) return 0;
    int64_t k = 1;
    for (int64_t i = 1; i < n; ++i)
        if ((a[i] >> 32) != (a[k - 1] >> 32)) a[k++] = a[i];
    return k;
}

/* thrust::set_difference(set_cmp) (tc.cu:260-263, wcc.cu:336-339). Multiset
 * semantics; `out` may alias `a`. */
static int64_t set_difference(const u64 *a, int64_t na, const u64 *b, int64_t nb, u64 *out) {
    int64_t i = 0, j = 0, k = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) out[k++] = a[i++];
        else if (b[j] < a[i]) ++j;
        else { ++i; ++j; }
    }
    while (i < na) out[k++] = a[i++];
    return k;
}

/* thrust::merge(set_cmp) (tc.cu:276-279, wcc.cu:308-312); ties take `a`
 * first, duplicates are kept. */
static void merge(const u64 *a, int64_t na, const u64 *b, int64_t nb, u64 *out) {
    int64_t i = 0, j = 0, k = 0;
    while (i < na && j < nb) {
        if (b[j] < a[i]) out[k++] = b[j++];
        else out[k++] = a[i++];
    }
    while (i < na) out[k++] = a[i++];
    while (j < nb) out[k++] = b[j++];
}

/* The join index: the hash-table relation sorted by (key, value). Probing
 * it yields, per probe key, the same multiset of matches as the reference's
 * linear-probe multimap (common/hash_table.cu:1-22, common/join.cu:1-48). */
typedef struct {
    u64 *rel;
    int64_t n;
} join_index;

static join_index index_build(const u64 *rel, int64_t n) {
    join_index ix;
    ix.rel = (u64 *) xmalloc((size_t) n * 8);
    memcpy(ix.rel, rel, (size_t) n * 8);
    sort_keys(ix.rel, n);
    ix.n = n;
    return ix;
}

static int64_t index_lower(const join_index *ix, uint32_t khi) {
    int64_t lo = 0, hi = ix->n;
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if ((uint32_t) (ix->rel[mid] >> 32) < khi) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* get_join (common/join.cu:51-87): for probe tuple (k, v) and every
 * relation tuple (k, w) emit (w, v). Two passes like the reference: size,
 * then write. */
static u64 *join(const join_index *ix, const u64 *probe, int64_t np, int64_t *out_n) {
    int64_t total = 0;
    for (int64_t i = 0; i < np; ++i) {
        uint32_t khi = (uint32_t) (probe[i] >> 32);
        for (int64_t j = index_lower(ix, khi); j < ix->n && (uint32_t) (ix->rel[j] >> 32) == khi; ++j) ++total;
    }
    u64 *out = (u64 *) xmalloc((size_t) total * 8);
    int64_t k = 0;
    for (int64_t i = 0; i < np; ++i) {
        uint32_t khi = (uint32_t) (probe[i] >> 32);
        u64 vlo = probe[i] & 0xFFFFFFFFull;
        for (int64_t j = index_lower(ix, khi); j < ix->n && (uint32_t) (ix->rel[j] >> 32) == khi; ++j)
            out[k++] = (ix->rel[j] << 32) | vlo;
    }
    *out_n = total;
    return out;
}

typedef struct {
    int64_t *v;
    int64_t n, cap;
} i64vec;

static void vec_push(i64vec *x, int64_t v) {
    if (x->n == x->cap) {
        x->cap = x->cap ? 2 * x->cap : 64;
        x->v = (int64_t *) realloc(x->v, (size_t) x->cap * sizeof(int64_t));
        if (!x->v) abort();
    }
    x->v[x->n++] = v;
}

/* delta <- set_difference(delta, full); full <- merge(full, delta).
 * tc.cu:260-286, sg.cu:349-368. Returns the new |delta|. */
static int64_t diff_and_merge(u64 **delta, int64_t nd, u64 **full, int64_t *nfull) {
    nd = set_difference(*delta, nd, *full, *nfull, *delta);
    u64 *nf = (u64 *) xmalloc((size_t) (*nfull + nd) * 8);
    merge(*full, *nfull, *delta, nd, nf);
    free(*full);
    *full = nf;
    *nfull += nd;
    return nd;
}

int oracle_tc(const int32_t *edges, int64_t rows, int32_t **out, int64_t *out_rows,
              int32_t *iterations, int64_t **deltas) {
    /* tc.cu:132-133 create_entity_ar / create_entity_ar_reverse */
    u64 *e = (u64 *) xmalloc((size_t) rows * 8);
    u64 *delta = (u64 *) xmalloc((size_t) rows * 8);
    for (int64_t i = 0; i < rows; ++i) {
        e[i] = pk(edges[2 * i], edges[2 * i + 1]);
        delta[i] = pk(edges[2 * i + 1], edges[2 * i]);
    }
    /* tc.cu:178-181 dedup delta; 188-189 full = delta */
    int64_t nd = sort_unique(delta, rows);
    int64_t nfull = nd;
    u64 *full = (u64 *) xmalloc((size_t) nd * 8);
    memcpy(full, delta, (size_t) nd * 8);
    /* tc.cu:210 hash table over the edge relation keyed by source */
    join_index ix = index_build(e, rows);
    free(e);
    i64vec dv = {0, 0, 0};
    int32_t it = 0;
    for (;;) { /* tc.cu:216-314 */
        int64_t nj;
        u64 *j = join(&ix, delta, nd, &nj); /* (y,x) x edge(y,z) -> (z,x) */
        free(delta);
        delta = j;
        nd = sort_unique(delta, nj);
        int64_t old = nfull;
        nd = diff_and_merge(&delta, nd, &full, &nfull);
        ++it;
        vec_push(&dv, nd);
        if (old == nfull) break;
    }
    free(delta);
    free(ix.rel);
    /* tc.cu:324 reverse_t_full: rows (x, z) in (z, x) order */
    int32_t *o = (int32_t *) xmalloc((size_t) nfull * 8);
    for (int64_t i = 0; i < nfull; ++i) {
        o[2 * i] = pk_val(full[i]);
        o[2 * i + 1] = pk_key(full[i]);
    }
    free(full);
    *out = o;
    *out_rows = nfull;
    *iterations = it;
    *deltas = dv.v;
    return 0;
}

int oracle_tc_nl(const int32_t *edges, int64_t rows, int32_t **out, int64_t *out_rows,
                 int32_t *iterations, int64_t **deltas) {
    /* tc_nl.cu differs from tc.cu only in deduplicating the edge relation
     * (tc_nl.cu:182-185) and probing it by binary search (common/join.cu:89-180);
     * both leave every derived set unchanged. */
    return oracle_tc(edges, rows, out, out_rows, iterations, deltas);
}

int oracle_sg(const int32_t *edges, int64_t rows, int32_t **out, int64_t *out_rows,
              int32_t *iterations, int64_t **deltas) {
    /* sg.cu:117 create_entity_ar; 150-153 dedup into t_delta */
    u64 *delta = (u64 *) xmalloc((size_t) rows * 8);
    for (int64_t i = 0; i < rows; ++i) delta[i] = pk(edges[2 * i], edges[2 * i + 1]);
    int64_t nd = sort_unique(delta, rows);
    /* sg.cu:162 hash table over the deduplicated edges */
    join_index ix = index_build(delta, nd);
    /* sg.cu:170-179 base rule: e(p,x), e(p,y), x != y */
    int64_t nb;
    u64 *base = join(&ix, delta, nd, &nb);
    int64_t k = 0;
    for (int64_t i = 0; i < nb; ++i)
        if ((base[i] >> 32) != (base[i] & 0xFFFFFFFFull)) base[k++] = base[i];
    free(delta);
    delta = base;
    nd = sort_unique(delta, k); /* sg.cu:216-217 */
    int64_t nfull = nd;
    u64 *full = (u64 *) xmalloc((size_t) nd * 8);
    memcpy(full, delta, (size_t) nd * 8);
    i64vec dv = {0, 0, 0};
    int32_t it = 0;
    for (;;) { /* sg.cu:244-390 */
        int64_t n1, n2;
        u64 *j1 = join(&ix, delta, nd, &n1); /* sg(a,b), e(a,x) -> (x,b) */
        for (int64_t i = 0; i < n1; ++i) j1[i] = pk_swap(j1[i]); /* sg.cu:253 -> (b,x) */
        n1 = sort_unique(j1, n1);                                 /* sg.cu:282-287 */
        u64 *j2 = join(&ix, j1, n1, &n2);                         /* (b,x), e(b,y) -> (y,x) */
        for (int64_t i = 0; i < n2; ++i) j2[i] = pk_swap(j2[i]); /* sg.cu:301 -> (x,y) */
        n2 = sort_unique(j2, n2);                                 /* sg.cu:330-335 */
        free(j1);
        free(delta);
        delta = j2;
        int64_t old = nfull;
        nd = diff_and_merge(&delta, n2, &full, &nfull); /* sg.cu:349-368 */
        ++it;
        vec_push(&dv, nd);
        if (old == nfull) break; /* sg.cu:383-389 */
    }
    free(delta);
    free(ix.rel);
    int32_t *o = (int32_t *) xmalloc((size_t) nfull * 8); /* sg.cu:400 rows (x, y) */
    for (int64_t i = 0; i < nfull; ++i) {
        o[2 * i] = pk_key(full[i]);
        o[2 * i + 1] = pk_val(full[i]);
    }
    free(full);
    *out = o;
    *out_rows = nfull;
    *iterations = it;
    *deltas = dv.v;
    return 0;
}

int oracle_wcc(const int32_t *edges, int64_t rows, int32_t stop_mode,
               int32_t **comp_rows, int64_t *n_comp, int64_t *largest,
               int32_t *iterations, int64_t **deltas,
               int32_t **node_ids, int32_t **labels, int64_t *n_nodes) {
    /* wcc.cu:140-167: edge = dedup(E u E^T) */
    u64 *edge = (u64 *) xmalloc((size_t) (2 * rows) * 8);
    for (int64_t i = 0; i < rows; ++i) {
        edge[i] = pk(edges[2 * i], edges[2 * i + 1]);
        edge[rows + i] = pk(edges[2 * i + 1], edges[2 * i]);
    }
    int64_t ne = sort_unique(edge, 2 * rows);
    /* wcc.cu:211-221: cc(n, n), one per node */
    u64 *cc = (u64 *) xmalloc((size_t) ne * 8);
    for (int64_t i = 0; i < ne; ++i) cc[i] = (edge[i] & 0xFFFFFFFF00000000ull) | (edge[i] >> 32);
    sort_keys(cc, ne);
    int64_t ncc = unique_by_key(cc, ne);
    /* wcc.cu:228-231: delta = cc */
    int64_t nd = ncc;
    u64 *delta = (u64 *) xmalloc((size_t) nd * 8);
    memcpy(delta, cc, (size_t) nd * 8);
    int64_t global_delta = nd;
    join_index ix = index_build(edge, ne); /* wcc.cu:247 */
    free(edge);
    i64vec dv = {0, 0, 0};
    int32_t it = 0;
    for (;;) { /* wcc.cu:255-387 */
        int64_t nj;
        u64 *jr = join(&ix, delta, nd, &nj); /* (node,label), edge(node,nbr) -> (nbr,label) */
        nj = sort_unique(jr, nj);            /* wcc.cu:286-291 */
        u64 *ncc_buf = (u64 *) xmalloc((size_t) (ncc + nj) * 8);
        merge(cc, ncc, jr, nj, ncc_buf);                    /* wcc.cu:308-312 */
        int64_t nn = unique_by_key(ncc_buf, ncc + nj);      /* wcc.cu:320-323 */
        u64 *nd_buf = (u64 *) xmalloc((size_t) nn * 8);
        nd = set_difference(ncc_buf, nn, cc, ncc, nd_buf); /* wcc.cu:336-339 */
        free(delta);
        delta = nd_buf;
        free(cc);
        cc = ncc_buf;
        ncc = nn;
        free(jr);
        int64_t old = global_delta;
        global_delta = nd;
        ++it;
        vec_push(&dv, nd);
        if (stop_mode == ORACLE_WCC_STOP_REFERENCE) {
            if (old == global_delta) break; /* wcc.cu:366-383 */
        } else if (nd == 0) {
            break;
        }
    }
    free(delta);
    free(ix.rel);
    /* wcc.cu:389-472: component ids, sizes, largest */
    int32_t *ids = (int32_t *) xmalloc((size_t) ncc * 4);
    int32_t *lab = (int32_t *) xmalloc((size_t) ncc * 4);
    u64 *comp = (u64 *) xmalloc((size_t) ncc * 8);
    for (int64_t i = 0; i < ncc; ++i) {
        ids[i] = pk_key(cc[i]);
        lab[i] = pk_val(cc[i]);
        comp[i] = pk(lab[i], 0); /* replace_key_by_value: (label, 0) */
    }
    sort_keys(comp, ncc);
    int64_t best = 0, run = 0;
    for (int64_t i = 0; i < ncc; ++i) {
        run = (i > 0 && comp[i] == comp[i - 1]) ? run + 1 : 1;
        if (run > best) best = run;
    }
    int64_t nc = unique_by_key(comp, ncc);
    int32_t *rowsout = (int32_t *) xmalloc((size_t) nc * 8);
    for (int64_t i = 0; i < nc; ++i) {
        rowsout[2 * i] = pk_key(comp[i]);
        rowsout[2 * i + 1] = 0;
    }
    free(comp);
    free(cc);
    *comp_rows = rowsout;
    *n_comp = nc;
    *largest = best;
    *iterations = it;
    *deltas = dv.v;
    *node_ids = ids;
    *labels = lab;
    *n_nodes = ncc;
    return 0;
}

void oracle_generate_rows(int64_t rows, int32_t rand_range, int32_t *out) {
    /* common/parallel_io.cu:87-97 with rank 0: seed = rank + 1 */
    srand(1u);
    for (int64_t i = 0; i < 2 * rows; ++i) out[i] = (rand() % rand_range) + 1;
}

int oracle_single_join(int64_t rows, int32_t rand_range, int32_t **out, int64_t *out_rows) {
    int32_t *data = (int32_t *) xmalloc((size_t) rows * 8);
    oracle_generate_rows(rows, rand_range, data);
    u64 *rel = (u64 *) xmalloc((size_t) rows * 8);
    u64 *rev = (u64 *) xmalloc((size_t) rows * 8);
    for (int64_t i = 0; i < rows; ++i) {
        rel[i] = pk(data[2 * i], data[2 * i + 1]);
        rev[i] = pk(data[2 * i + 1], data[2 * i]);
    }
    free(data);
    int64_t nrel = sort_unique(rel, rows); /* single_join.cu:165-168 */
    int64_t nrev = sort_unique(rev, rows); /* single_join.cu:200-203 */
    join_index ix = index_build(rel, nrel);
    free(rel);
    int64_t nj;
    u64 *j = join(&ix, rev, nrev, &nj); /* (b,a), rel(b,c) -> (c,a) */
    free(rev);
    free(ix.rel);
    nj = sort_unique(j, nj); /* single_join.cu:259-264 */
    int32_t *o = (int32_t *) xmalloc((size_t) nj * 8);
    for (int64_t i = 0; i < nj; ++i) { /* get_reverse_int_ar_from_entity_ar: rows (a, c) */
        o[2 * i] = pk_val(j[i]);
        o[2 * i + 1] = pk_key(j[i]);
    }
    free(j);
    *out = o;
    *out_rows = nj;
    return 0;
}
