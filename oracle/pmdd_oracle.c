/*
 * pmdd_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A plain-C, single-threaded restatement of rahulptel/PMDD's CPU enumeration over a
 * decision diagram, operating on the flat DD layout of include/pmdd.h.  It is the
 * checker for the CUDA engine: tests, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may call it; nothing shipped links or calls it.
 *
 * Parity of this restatement is pinned against the reference's own binary (built by
 * oracle/Makefile into oracle/_ref/) on the committed fixtures in tests/golden/.
 *
 * What each function restates:
 *   front_merge_shift   ParetoFrontier::merge(frontier, shift)
 *                       src/pmdd/enum/pareto_frontier.hpp:237-303 (weak-dominance insert:
 *                       an incoming point equal to a kept one is dropped; a kept point
 *                       weakly dominated by an incoming one is replaced / erased)
 *   oracle_topdown      topdown_cpu_enumerate + expand_layer_topdown_cpu
 *                       src/pmdd/enum/cpu/enum.cpp:14-76, src/pmdd/enum/cpu/topdown.cpp:12-33
 *                       (incoming arcs merged in stored order: the flat DD lists 1-arcs
 *                       first, as the maximising CPU loop does)
 *   oracle_bottomup     bottomup_cpu_enumerate  src/pmdd/enum/cpu/enum.cpp:122-229
 *   oracle_coupled      coupled_cpu_enumerate / coupled_mdd_cpu_enumerate
 *                       src/pmdd/enum/cpu/enum.cpp:231-554 with the layer-value
 *                       heuristics of src/pmdd/enum/cpu/couple.cpp:15-48 and
 *                       ParetoFrontier::convolute (pareto_frontier.hpp:353-365)
 *   knapsack state dominance
 *                       filter_dominance_knapsack_cpu  src/pmdd/enum/cpu/dominance.cpp:24-86
 *   set-packing state dominance
 *                       filter_dominance_setpacking_cpu  src/pmdd/enum/cpu/dominance.cpp:88-173
 *                       (applied on top-down layers by methods 1 and 3,
 *                       src/pmdd/enum/cpu/enum.cpp:43-49 and :275-285)
 *   oracle_nd_keep      the GPU filter's keep rule dominates_or_tie_before
 *                       src/pmdd/enum/gpu/dominance_utils.cuh:10-23 (first duplicate kept)
 *
 * One deliberate difference: the reference marks erased points by writing the
 * sentinel -9999999 into their first objective; this restatement keeps an explicit
 * flag instead, which only differs if a real objective value equals the sentinel.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/pmdd.h"

typedef struct {
    int32_t *pts;   /* n * d values */
    int64_t n;
    int64_t cap;
} front_t;

static int front_reserve(front_t *f, int64_t n, int d) {
    if (n <= f->cap) return 0;
    int64_t cap = f->cap ? f->cap : 16;
    while (cap < n) cap *= 2;
    int32_t *p = (int32_t *)realloc(f->pts, (size_t)cap * (size_t)d * sizeof(int32_t));
    if (!p) return -1;
    f->pts = p;
    f->cap = cap;
    return 0;
}

static void front_free(front_t *f) {
    free(f->pts);
    f->pts = NULL;
    f->n = f->cap = 0;
}

/* ParetoFrontier::merge(frontier, shift): insert every src point + shift. */
static int front_merge_shift(front_t *dst, const int32_t *src, int64_t src_n, const int32_t *shift,
                             int d, uint8_t **erased_buf, int64_t *erased_cap) {
    const int64_t end = dst->n;
    int32_t aux[8];
    if (front_reserve(dst, dst->n + src_n, d)) return -1;
    if (*erased_cap < dst->n + src_n) {
        int64_t c = dst->n + src_n + 64;
        uint8_t *e = (uint8_t *)realloc(*erased_buf, (size_t)c);
        if (!e) return -1;
        *erased_buf = e;
        *erased_cap = c;
    }
    uint8_t *erased = *erased_buf;
    memset(erased, 0, (size_t)(dst->n + src_n));
    for (int64_t j = 0; j < src_n; ++j) {
        for (int o = 0; o < d; ++o) aux[o] = src[j * d + o] + shift[o];
        int must_add = 1;
        for (int64_t i = 0; i < end; ++i) {
            if (erased[i]) continue;
            const int32_t *s = dst->pts + i * d;
            int dominates = 1, dominated = 1;
            for (int o = 0; o < d && (dominates || dominated); ++o) {
                dominates &= (aux[o] >= s[o]);
                dominated &= (aux[o] <= s[o]);
            }
            if (dominated) {
                must_add = 0;
                break;
            } else if (dominates) {
                if (must_add) {
                    memcpy(dst->pts + i * d, aux, sizeof(int32_t) * (size_t)d);
                    must_add = 0;
                } else {
                    erased[i] = 1;
                }
            }
        }
        if (must_add) {
            memcpy(dst->pts + dst->n * d, aux, sizeof(int32_t) * (size_t)d);
            dst->n++;
        }
    }
    /* remove_empty(): compact (order of survivors is irrelevant to the set) */
    int64_t w = 0;
    for (int64_t i = 0; i < dst->n; ++i) {
        if (erased[i]) continue;
        if (w != i) memcpy(dst->pts + w * d, dst->pts + i * d, sizeof(int32_t) * (size_t)d);
        ++w;
    }
    dst->n = w;
    return 0;
}

static int64_t sum_points(const front_t *f, int d) {
    int64_t s = 0;
    for (int64_t i = 0; i < f->n * d; ++i) s += f->pts[i];
    return s;
}

/* Out-arc CSR (transpose of the in-arc CSR), arcs grouped by tail node. */
typedef struct {
    int32_t *off;  /* N+1 */
    int32_t *arc;  /* A: index of the in-arc record */
} out_csr_t;

static int build_out_csr(const pmdd_dd *dd, out_csr_t *o) {
    const int32_t N = dd->num_nodes, A = dd->num_arcs;
    o->off = (int32_t *)calloc((size_t)N + 1, sizeof(int32_t));
    o->arc = (int32_t *)malloc((size_t)(A > 0 ? A : 1) * sizeof(int32_t));
    if (!o->off || !o->arc) return -1;
    for (int32_t a = 0; a < A; ++a) o->off[dd->arc_src[a] + 1]++;
    for (int32_t v = 0; v < N; ++v) o->off[v + 1] += o->off[v];
    int32_t *fill = (int32_t *)malloc((size_t)(N > 0 ? N : 1) * sizeof(int32_t));
    if (!fill) return -1;
    memcpy(fill, o->off, (size_t)N * sizeof(int32_t));
    for (int32_t v = 0; v < N; ++v)
        for (int32_t a = dd->in_arc_offsets[v]; a < dd->in_arc_offsets[v + 1]; ++a)
            o->arc[fill[dd->arc_src[a]]++] = a;
    free(fill);
    return 0;
}

static void free_out_csr(out_csr_t *o) {
    free(o->off);
    free(o->arc);
}

static int32_t *arc_head_table(const pmdd_dd *dd) {
    int32_t *head = (int32_t *)malloc((size_t)(dd->num_arcs > 0 ? dd->num_arcs : 1) * sizeof(int32_t));
    if (!head) return NULL;
    for (int32_t v = 0; v < dd->num_nodes; ++v)
        for (int32_t a = dd->in_arc_offsets[v]; a < dd->in_arc_offsets[v + 1]; ++a) head[a] = v;
    return head;
}

static const int32_t *sd_keys;
static int cmp_min_weight_desc(const void *a, const void *b) {
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    if (sd_keys[x] != sd_keys[y]) return sd_keys[x] > sd_keys[y] ? -1 : 1;
    return x < y ? -1 : (x > y);
}

/* filter_dominance_knapsack_cpu (src/pmdd/enum/cpu/dominance.cpp:24-86) on layer l:
 * non-empty nodes ordered by min_weight, largest first (ties: stable by node id here;
 * the reference's std::sort leaves tie order unspecified); each label of node i is
 * dropped if a label of one of the next two nodes is >= on every objective, skipping
 * the pair when both nodes have one parent, the same one, through different arcs. */
static int64_t knapsack_state_dominance(const pmdd_dd *dd, int l, front_t *fr) {
    const int d = dd->nobjs;
    const int32_t b = dd->layer_offsets[l], e = dd->layer_offsets[l + 1];
    const int32_t cnt = e - b;
    if (cnt <= 1 || dd->min_weight == NULL) return 0;
    int32_t *order = (int32_t *)malloc((size_t)cnt * sizeof(int32_t));
    int32_t m = 0;
    for (int32_t v = b; v < e; ++v)
        if (fr[v].n > 0) order[m++] = v;
    /* min_weight descending, ties by node id (stable) */
    sd_keys = dd->min_weight;
    qsort(order, (size_t)m, sizeof(int32_t), cmp_min_weight_desc);
    int64_t removed = 0;
    uint8_t *dead = NULL;
    for (int32_t i = 0; i + 1 < m; ++i) {
        const int32_t n1 = order[i];
        const int32_t p1 = dd->in_arc_offsets[n1 + 1] - dd->in_arc_offsets[n1] == 1 ? dd->in_arc_offsets[n1] : -1;
        dead = (uint8_t *)realloc(dead, (size_t)(fr[n1].n > 0 ? fr[n1].n : 1));
        memset(dead, 0, (size_t)fr[n1].n);
        int64_t num_dead = 0;
        for (int32_t j = i + 1; j < m && j < i + 3; ++j) {
            const int32_t n2 = order[j];
            const int32_t p2 = dd->in_arc_offsets[n2 + 1] - dd->in_arc_offsets[n2] == 1 ? dd->in_arc_offsets[n2] : -1;
            /* BDD arc type: weight row 0 is the 0-arc row, any other row a 1-arc */
            if (p1 >= 0 && p2 >= 0 && dd->arc_src[p1] == dd->arc_src[p2] &&
                (dd->arc_weight[p1] != 0) != (dd->arc_weight[p2] != 0))
                continue;
            for (int64_t s1 = 0; s1 < fr[n1].n; ++s1) {
                if (dead[s1]) continue;
                const int32_t *x = fr[n1].pts + s1 * d;
                for (int64_t s2 = 0; s2 < fr[n2].n; ++s2) {
                    const int32_t *y = fr[n2].pts + s2 * d;
                    int dom = 1;
                    for (int o = 0; o < d && dom; ++o) dom = (y[o] >= x[o]);
                    if (dom) {
                        dead[s1] = 1;
                        ++num_dead;
                        break;
                    }
                }
            }
        }
        if (num_dead > 0) {
            int64_t w = 0;
            for (int64_t s = 0; s < fr[n1].n; ++s) {
                if (dead[s]) continue;
                if (w != s) memcpy(fr[n1].pts + w * d, fr[n1].pts + s * d, sizeof(int32_t) * d);
                ++w;
            }
            fr[n1].n = w;
            removed += num_dead;
        }
    }
    free(dead);
    free(order);
    return removed;
}

/* Drops the labels of node n1 that a label of node n2 weakly dominates (>= on every
 * objective); returns how many. */
static int64_t drop_dominated_labels(front_t *fr, int32_t n1, int32_t n2, int d) {
    int64_t w = 0, dropped = 0;
    for (int64_t s1 = 0; s1 < fr[n1].n; ++s1) {
        const int32_t *x = fr[n1].pts + s1 * d;
        int dom = 0;
        for (int64_t s2 = 0; s2 < fr[n2].n && !dom; ++s2) {
            const int32_t *y = fr[n2].pts + s2 * d;
            dom = 1;
            for (int o = 0; o < d && dom; ++o) dom = (y[o] >= x[o]);
        }
        if (dom) {
            ++dropped;
            continue;
        }
        if (w != s1) memcpy(fr[n1].pts + w * d, x, sizeof(int32_t) * d);
        ++w;
    }
    fr[n1].n = w;
    return dropped;
}

static int lowest_vertex(const uint64_t *s, int W) {
    for (int w = 0; w < W; ++w)
        if (s[w]) return w * 64 + __builtin_ctzll(s[w]);
    return -1;
}

/* filter_dominance_setpacking_cpu (src/pmdd/enum/cpu/dominance.cpp:88-173) on layer l:
 * the layer's nodes (labels or not) are bucketed by state size, buckets 0 ..
 * num_layers-2, each in layer order.  For a bucket b1 (b1 < num_layers-2) holding two or
 * more nodes, only the next non-empty bucket b2 is searched: each node of b1 takes the
 * first node of b2 that has the same lowest vertex, is not its single-parent sibling
 * through a different arc type, and whose state contains the node's state, and loses
 * the labels that a label of that node weakly dominates.  A node is only compared with
 * nodes of larger buckets, which are pruned later, so every comparison sees the labels
 * as they were before the pass. */
static int64_t setpacking_state_dominance(const pmdd_dd *dd, int l, front_t *fr) {
    const int d = dd->nobjs, W = dd->state_words, nb = dd->num_layers - 1;
    const int32_t b = dd->layer_offsets[l], e = dd->layer_offsets[l + 1];
    const int32_t cnt = e - b;
    if (cnt <= 1 || dd->node_state == NULL || W <= 0) return 0;
    int32_t *bucket = (int32_t *)malloc((size_t)cnt * sizeof(int32_t));
    int32_t *start = (int32_t *)calloc((size_t)nb + 2, sizeof(int32_t));
    int32_t *list = (int32_t *)malloc((size_t)cnt * sizeof(int32_t));
    for (int32_t i = 0; i < cnt; ++i) {
        const uint64_t *s = dd->node_state + (size_t)(b + i) * W;
        int pc = 0;
        for (int w = 0; w < W; ++w) pc += __builtin_popcountll(s[w]);
        bucket[i] = pc < nb ? pc : nb; /* sizes >= nb take no part */
        start[bucket[i] + 1]++;
    }
    for (int k = 0; k <= nb; ++k) start[k + 1] += start[k];
    {
        int32_t *fill = (int32_t *)malloc(((size_t)nb + 1) * sizeof(int32_t));
        memcpy(fill, start, ((size_t)nb + 1) * sizeof(int32_t));
        for (int32_t i = 0; i < cnt; ++i) list[fill[bucket[i]]++] = i; /* layer order within a bucket */
        free(fill);
    }
    int64_t removed = 0;
    for (int b1 = 0; b1 + 1 < nb; ++b1) {
        if (start[b1 + 1] - start[b1] <= 1) continue;
        int b2 = b1 + 1;
        while (b2 < nb && start[b2 + 1] == start[b2]) ++b2;
        if (b2 >= nb) continue;
        for (int32_t p = start[b1]; p < start[b1 + 1]; ++p) {
            const int32_t n1 = b + list[p];
            const uint64_t *s1 = dd->node_state + (size_t)n1 * W;
            const int32_t a1 = dd->in_arc_offsets[n1 + 1] - dd->in_arc_offsets[n1] == 1 ? dd->in_arc_offsets[n1] : -1;
            for (int32_t q = start[b2]; q < start[b2 + 1]; ++q) {
                const int32_t n2 = b + list[q];
                const uint64_t *s2 = dd->node_state + (size_t)n2 * W;
                if (lowest_vertex(s1, W) != lowest_vertex(s2, W)) continue;
                const int32_t a2 =
                    dd->in_arc_offsets[n2 + 1] - dd->in_arc_offsets[n2] == 1 ? dd->in_arc_offsets[n2] : -1;
                if (a1 >= 0 && a2 >= 0 && dd->arc_src[a1] == dd->arc_src[a2] &&
                    (dd->arc_weight[a1] != 0) != (dd->arc_weight[a2] != 0))
                    continue;
                int subset = 1;
                for (int w = 0; w < W && subset; ++w) subset = (s1[w] & ~s2[w]) == 0;
                if (!subset) continue;
                removed += drop_dominated_labels(fr, n1, n2, d);
                break;
            }
        }
    }
    free(bucket);
    free(start);
    free(list);
    return removed;
}

/* filter_dominance_cpu (src/pmdd/enum/cpu/dominance.cpp:12-22) dispatches on the problem
 * type; here the DD says which: knapsack BDDs carry min_weight, set-packing BDDs their
 * node states, TSP MDDs neither (no state dominance, as in the reference). */
static int64_t layer_state_dominance(const pmdd_dd *dd, int l, front_t *fr) {
    if (dd->min_weight != NULL) return knapsack_state_dominance(dd, l, fr);
    if (dd->node_state != NULL) return setpacking_state_dominance(dd, l, fr);
    return 0;
}

static int validate(const pmdd_dd *dd) {
    if (!dd || dd->nobjs < 1 || dd->nobjs > 8 || dd->num_layers < 2) return PMDD_ERR_INVALID;
    if (dd->layer_offsets[1] != 1 || dd->layer_offsets[dd->num_layers] - dd->layer_offsets[dd->num_layers - 1] != 1)
        return PMDD_ERR_INVALID;
    return PMDD_OK;
}

static int take_result(front_t *f, int d, int32_t **out, int64_t *n_out) {
    *n_out = f->n;
    *out = (int32_t *)malloc((size_t)(f->n > 0 ? f->n : 1) * (size_t)d * sizeof(int32_t));
    if (!*out) return PMDD_ERR_OOM;
    memcpy(*out, f->pts, (size_t)f->n * (size_t)d * sizeof(int32_t));
    return PMDD_OK;
}

typedef struct {
    int64_t candidates_total;
    int64_t survivors_total;
    int64_t dominance_filtered_total;
    int64_t join_products_total;
    int32_t layer_coupling;
    int32_t pad;
} oracle_stats;

/* Method 1: top-down (optionally with knapsack state dominance). */
int oracle_topdown(const pmdd_dd *dd, int state_dominance, int32_t **out, int64_t *n_out, oracle_stats *st) {
    int rc = validate(dd);
    if (rc) return rc;
    const int d = dd->nobjs;
    const int32_t N = dd->num_nodes;
    front_t *fr = (front_t *)calloc((size_t)N, sizeof(front_t));
    uint8_t *erased = NULL;
    int64_t erased_cap = 0;
    if (!fr) return PMDD_ERR_OOM;
    front_reserve(&fr[0], 1, d);
    memset(fr[0].pts, 0, sizeof(int32_t) * d);
    fr[0].n = 1;
    for (int l = 1; l < dd->num_layers; ++l) {
        for (int32_t v = dd->layer_offsets[l]; v < dd->layer_offsets[l + 1]; ++v) {
            for (int32_t a = dd->in_arc_offsets[v]; a < dd->in_arc_offsets[v + 1]; ++a) {
                const front_t *p = &fr[dd->arc_src[a]];
                if (st) st->candidates_total += p->n;
                if (front_merge_shift(&fr[v], p->pts, p->n, dd->weights + (size_t)dd->arc_weight[a] * d, d, &erased,
                                      &erased_cap))
                    return PMDD_ERR_OOM;
            }
        }
        if (state_dominance > 0) {
            const int64_t r = layer_state_dominance(dd, l, fr);
            if (st) st->dominance_filtered_total += r;
        }
        for (int32_t v = dd->layer_offsets[l]; v < dd->layer_offsets[l + 1]; ++v)
            if (st) st->survivors_total += fr[v].n;
        for (int32_t u = dd->layer_offsets[l - 1]; u < dd->layer_offsets[l]; ++u) front_free(&fr[u]);
    }
    const int32_t term = N - 1;
    rc = take_result(&fr[term], d, out, n_out);
    for (int32_t v = 0; v < N; ++v) front_free(&fr[v]);
    free(fr);
    free(erased);
    return rc;
}

/* Method 2: bottom-up. */
int oracle_bottomup(const pmdd_dd *dd, int32_t **out, int64_t *n_out) {
    int rc = validate(dd);
    if (rc) return rc;
    const int d = dd->nobjs;
    const int32_t N = dd->num_nodes;
    out_csr_t oc;
    if (build_out_csr(dd, &oc)) return PMDD_ERR_OOM;
    int32_t *head = arc_head_table(dd);
    if (!head) return PMDD_ERR_OOM;
    front_t *fr = (front_t *)calloc((size_t)N, sizeof(front_t));
    uint8_t *erased = NULL;
    int64_t erased_cap = 0;
    front_reserve(&fr[N - 1], 1, d);
    memset(fr[N - 1].pts, 0, sizeof(int32_t) * d);
    fr[N - 1].n = 1;
    for (int l = dd->num_layers - 2; l >= 0; --l) {
        for (int32_t u = dd->layer_offsets[l]; u < dd->layer_offsets[l + 1]; ++u) {
            for (int32_t k = oc.off[u]; k < oc.off[u + 1]; ++k) {
                const int32_t a = oc.arc[k];
                const front_t *c = &fr[head[a]];
                if (front_merge_shift(&fr[u], c->pts, c->n, dd->weights + (size_t)dd->arc_weight[a] * d, d, &erased,
                                      &erased_cap))
                    return PMDD_ERR_OOM;
            }
        }
        for (int32_t v = dd->layer_offsets[l + 1]; v < dd->layer_offsets[l + 2]; ++v) front_free(&fr[v]);
    }
    rc = take_result(&fr[0], d, out, n_out);
    for (int32_t v = 0; v < N; ++v) front_free(&fr[v]);
    free(fr);
    free(head);
    free(erased);
    free_out_csr(&oc);
    return rc;
}

/* Method 3: dynamic layer cutset.  Layer choice: expand top-down while the top-down
 * value <= the bottom-up value.  Top-down value of a node = |F_td| x (number of
 * outgoing arcs); bottom-up value = (int)(1.5 x |F_bu| x (number of incoming arcs)),
 * truncated per node as src/pmdd/enum/cpu/couple.cpp:15-48 does.  At the meeting
 * layer every node's top-down and bottom-up frontiers are convoluted into one
 * running frontier. */
int oracle_coupled(const pmdd_dd *dd, int state_dominance, int32_t **out, int64_t *n_out, oracle_stats *st) {
    int rc = validate(dd);
    if (rc) return rc;
    const int d = dd->nobjs;
    const int32_t N = dd->num_nodes;
    out_csr_t oc;
    if (build_out_csr(dd, &oc)) return PMDD_ERR_OOM;
    int32_t *head = arc_head_table(dd);
    front_t *td = (front_t *)calloc((size_t)N, sizeof(front_t));
    front_t *bu = (front_t *)calloc((size_t)N, sizeof(front_t));
    uint8_t *erased = NULL;
    int64_t erased_cap = 0;
    if (!td || !bu || !head) return PMDD_ERR_OOM;
    front_reserve(&td[0], 1, d);
    memset(td[0].pts, 0, sizeof(int32_t) * d);
    td[0].n = 1;
    front_reserve(&bu[N - 1], 1, d);
    memset(bu[N - 1].pts, 0, sizeof(int32_t) * d);
    bu[N - 1].n = 1;
    int layer_td = 0, layer_bu = dd->num_layers - 1;
    int64_t val_td = 0, val_bu = 0;
    while (layer_td != layer_bu) {
        if (val_td <= val_bu) {
            ++layer_td;
            const int l = layer_td;
            val_td = 0;
            for (int32_t v = dd->layer_offsets[l]; v < dd->layer_offsets[l + 1]; ++v) {
                for (int32_t a = dd->in_arc_offsets[v]; a < dd->in_arc_offsets[v + 1]; ++a) {
                    const front_t *p = &td[dd->arc_src[a]];
                    if (st) st->candidates_total += p->n;
                    if (front_merge_shift(&td[v], p->pts, p->n, dd->weights + (size_t)dd->arc_weight[a] * d, d,
                                          &erased, &erased_cap))
                        return PMDD_ERR_OOM;
                }
                val_td += (int64_t)td[v].n * (oc.off[v + 1] - oc.off[v]);
            }
            /* state dominance after the layer value, before the survivor count
             * (src/pmdd/enum/cpu/enum.cpp:266-285) */
            if (state_dominance > 0) {
                const int64_t r = layer_state_dominance(dd, l, td);
                if (st) st->dominance_filtered_total += r;
            }
            for (int32_t v = dd->layer_offsets[l]; v < dd->layer_offsets[l + 1]; ++v)
                if (st) st->survivors_total += td[v].n;
            for (int32_t u = dd->layer_offsets[l - 1]; u < dd->layer_offsets[l]; ++u) front_free(&td[u]);
        } else {
            --layer_bu;
            const int l = layer_bu;
            val_bu = 0;
            for (int32_t u = dd->layer_offsets[l]; u < dd->layer_offsets[l + 1]; ++u) {
                for (int32_t k = oc.off[u]; k < oc.off[u + 1]; ++k) {
                    const int32_t a = oc.arc[k];
                    const front_t *c = &bu[head[a]];
                    if (st) st->candidates_total += c->n;
                    if (front_merge_shift(&bu[u], c->pts, c->n, dd->weights + (size_t)dd->arc_weight[a] * d, d,
                                          &erased, &erased_cap))
                        return PMDD_ERR_OOM;
                }
                const int64_t in_arcs = dd->in_arc_offsets[u + 1] - dd->in_arc_offsets[u];
                val_bu += (int64_t)(1.5 * (double)(bu[u].n * in_arcs));
                if (st) st->survivors_total += bu[u].n;
            }
            for (int32_t v = dd->layer_offsets[l + 1]; v < dd->layer_offsets[l + 2]; ++v) front_free(&bu[v]);
        }
    }
    if (st) st->layer_coupling = layer_td;
    front_t res = {0};
    const int l = layer_td;
    for (int32_t v = dd->layer_offsets[l]; v < dd->layer_offsets[l + 1]; ++v) {
        const front_t *A = &td[v], *B = &bu[v];
        if (st) st->join_products_total += A->n * B->n;
        /* convolute: shift the larger frontier by each point of the smaller one */
        const front_t *small = A->n < B->n ? A : B;
        const front_t *big = A->n < B->n ? B : A;
        for (int64_t j = 0; j < small->n; ++j)
            if (front_merge_shift(&res, big->pts, big->n, small->pts + j * d, d, &erased, &erased_cap))
                return PMDD_ERR_OOM;
    }
    (void)sum_points;
    /* the joined frontier counts as survivors too (src/pmdd/enum/cpu/enum.cpp:393-395) */
    if (st) st->survivors_total += res.n;
    rc = take_result(&res, d, out, n_out);
    front_free(&res);
    for (int32_t v = 0; v < N; ++v) {
        front_free(&td[v]);
        front_free(&bu[v]);
    }
    free(td);
    free(bu);
    free(head);
    free(erased);
    free_out_csr(&oc);
    return rc;
}

/* Keep rule of the GPU filter (dominates_or_tie_before): point i survives unless some
 * j has pts[j] >= pts[i] on every objective and (pts[j] != pts[i] or j < i). */
void oracle_nd_keep(const int32_t *pts, int64_t n, int d, uint8_t *keep) {
    for (int64_t i = 0; i < n; ++i) {
        const int32_t *x = pts + i * d;
        int k = 1;
        for (int64_t j = 0; j < n && k; ++j) {
            if (j == i) continue;
            const int32_t *y = pts + j * d;
            int ge = 1, eq = 1;
            for (int o = 0; o < d; ++o) {
                ge &= (y[o] >= x[o]);
                eq &= (y[o] == x[o]);
            }
            if (ge && (!eq || j < i)) k = 0;
        }
        keep[i] = (uint8_t)k;
    }
}

void oracle_free(void *p) { free(p); }
