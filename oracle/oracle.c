/*
 * oracle.c -- CPU restatement of graph-gpu's serial algorithms.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Written as plain, serial C so that
 * each function can be read against the reference source it restates; the
 * citation above each function names that source (paths inside the reference
 * project).  Parity of this file with the reference is checked by
 * tests/test_oracle.py against oracle/_ref (the reference's own CPU code built
 * from its sources) and against the committed fixtures in tests/golden/.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

/* ------------------------------------------------------------------ utils */

static void* xmalloc(size_t bytes) {
    void* p = malloc(bytes ? bytes : 1);
    if (!p) abort();
    return p;
}

static orc_csr* csr_alloc(uint64_t n, uint64_t m, uint32_t flags) {
    orc_csr* g = (orc_csr*)xmalloc(sizeof *g);
    g->n = n;
    g->m = m;
    g->flags = flags;
    g->row_ptr = (uint32_t*)xmalloc((n + 1) * sizeof(uint32_t));
    g->col_idx = (uint32_t*)xmalloc(m * sizeof(uint32_t));
    return g;
}

void orc_csr_free(orc_csr* g) {
    if (!g) return;
    free(g->row_ptr);
    free(g->col_idx);
    free(g);
}

static uint32_t deg(const orc_csr* g, uint64_t v) { return g->row_ptr[v + 1] - g->row_ptr[v]; }

/* SplitMix64: src/util/rng.hpp:13-18 (next), :20-22 (below, multiply-shift),
 * :24 (uniform, 53-bit mantissa). */
uint64_t orc_rng_next(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t orc_rng_below(uint64_t* s, uint64_t bound) {
    return (uint64_t)(((unsigned __int128)orc_rng_next(s) * bound) >> 64);
}

double orc_rng_uniform(uint64_t* s) {
    return (double)(orc_rng_next(s) >> 11) * (1.0 / 9007199254740992.0);
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

/* ------------------------------------------------------------ CSR builders */

/* src/graph/csr.cpp:112-144 (compactAdjacency): sort each list, drop
 * self-loops and duplicates, slide the lists left, rebuild row_ptr. */
static void compact_adjacency(uint64_t n, uint32_t* rp, uint32_t* ci) {
    uint64_t pos = 0;
    for (uint64_t v = 0; v < n; ++v) {
        uint32_t b = rp[v], e = rp[v + 1];
        qsort(ci + b, e - b, sizeof(uint32_t), cmp_u32);
        uint64_t start = pos;
        for (uint32_t i = b; i < e; ++i) {
            uint32_t x = ci[i];
            if (x == (uint32_t)v) continue;
            if (pos > start && ci[pos - 1] == x) continue;
            ci[pos++] = x; /* pos <= i: never overwrites unread entries */
        }
        rp[v] = (uint32_t)start;
    }
    rp[n] = (uint32_t)pos;
}

/* src/graph/csr.cpp:146-163 (fromEdgeList): count, scatter, compact. */
orc_csr* orc_from_edge_list(uint64_t n, const uint32_t* eu, const uint32_t* ev, uint64_t ne,
                            int directed) {
    uint32_t* rp = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    for (uint64_t i = 0; i < ne; ++i) {
        rp[eu[i] + 1]++;
        if (!directed) rp[ev[i] + 1]++;
    }
    for (uint64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
    uint32_t* ci = (uint32_t*)xmalloc((uint64_t)rp[n] * sizeof(uint32_t));
    uint32_t* cur = (uint32_t*)xmalloc((n + 1) * sizeof(uint32_t));
    memcpy(cur, rp, n * sizeof(uint32_t));
    for (uint64_t i = 0; i < ne; ++i) {
        ci[cur[eu[i]]++] = ev[i];
        if (!directed) ci[cur[ev[i]]++] = eu[i];
    }
    free(cur);
    compact_adjacency(n, rp, ci);
    orc_csr* g = (orc_csr*)xmalloc(sizeof *g);
    g->n = n;
    g->m = rp[n];
    g->flags = (directed ? ORC_FLAG_DIRECTED : 0u) | ORC_FLAG_SORTED | ORC_FLAG_DEDUP;
    g->row_ptr = rp;
    g->col_idx = ci;
    return g;
}

typedef struct {
    uint32_t *u, *v;
    uint64_t size, cap;
} edge_list;

static void el_push(edge_list* e, uint32_t u, uint32_t v) {
    if (e->size == e->cap) {
        e->cap = e->cap ? 2 * e->cap : 1024;
        e->u = (uint32_t*)realloc(e->u, e->cap * sizeof(uint32_t));
        e->v = (uint32_t*)realloc(e->v, e->cap * sizeof(uint32_t));
    }
    e->u[e->size] = u;
    e->v[e->size] = v;
    e->size++;
}

static orc_csr* el_build(edge_list* e, uint64_t n, int directed) {
    orc_csr* g = orc_from_edge_list(n, e->u, e->v, e->size, directed);
    free(e->u);
    free(e->v);
    return g;
}

/* src/graph/generators.cpp:8-12 */
orc_csr* orc_gen_path(uint32_t n) {
    edge_list e = {0};
    for (uint32_t i = 0; i + 1 < n; ++i) el_push(&e, i, i + 1);
    return el_build(&e, n, 0);
}

/* src/graph/generators.cpp:14-18 */
orc_csr* orc_gen_star(uint32_t leaves) {
    edge_list e = {0};
    for (uint32_t i = 1; i <= leaves; ++i) el_push(&e, 0, i);
    return el_build(&e, (uint64_t)leaves + 1, 0);
}

/* src/graph/generators.cpp:20-25 */
orc_csr* orc_gen_complete(uint32_t n) {
    edge_list e = {0};
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j) el_push(&e, i, j);
    return el_build(&e, n, 0);
}

/* src/graph/generators.cpp:27-34 (addGrid) */
static void add_grid(edge_list* e, uint32_t base, uint32_t rows, uint32_t cols) {
    for (uint32_t r = 0; r < rows; ++r)
        for (uint32_t c = 0; c < cols; ++c) {
            uint32_t v = base + r * cols + c;
            if (c + 1 < cols) el_push(e, v, v + 1);
            if (r + 1 < rows) el_push(e, v, v + cols);
        }
}

/* src/graph/generators.cpp:36-41 */
orc_csr* orc_gen_two_components(void) {
    edge_list e = {0};
    for (uint32_t i = 0; i + 1 < 300; ++i) el_push(&e, i, i + 1);
    add_grid(&e, 300, 10, 10);
    return el_build(&e, 400, 0);
}

/* src/graph/generators.cpp:43 */
orc_csr* orc_gen_empty(uint32_t n) { return orc_from_edge_list(n, NULL, NULL, 0, 0); }

/* src/graph/generators.cpp:45-49 */
orc_csr* orc_gen_grid2d(uint32_t rows, uint32_t cols) {
    edge_list e = {0};
    add_grid(&e, 0, rows, cols);
    return el_build(&e, (uint64_t)rows * cols, 0);
}

/* src/graph/generators.cpp:51-75: per edge, `scale` quadrant draws with
 * a = .57, b = .19, c = .19 from one SplitMix64 stream.  The raw endpoint
 * pairs, before fromEdgeList (the reference's gen::rmat takes only an integer
 * edge factor; this takes any edge count on the same stream). */
void orc_rmat_draw(uint32_t scale, uint64_t m, uint64_t seed, uint32_t* eu, uint32_t* ev) {
    const double a = 0.57, b = 0.19, c = 0.19;
    /* edge i takes draws i*scale+1 .. i*scale+scale of the stream, whose state
     * before them is seed + i*scale*golden: edges are independent */
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < m; ++i) {
        uint64_t s = seed + i * (uint64_t)scale * 0x9E3779B97F4A7C15ull;
        uint32_t u = 0, v = 0;
        for (uint32_t bit = 0; bit < scale; ++bit) {
            double r = orc_rng_uniform(&s);
            uint32_t ub = 0, vb = 0;
            if (r < a) {
            } else if (r < a + b) {
                vb = 1;
            } else if (r < a + b + c) {
                ub = 1;
            } else {
                ub = 1;
                vb = 1;
            }
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        eu[i] = u;
        ev[i] = v;
    }
}

orc_csr* orc_gen_rmat_edges(uint32_t scale, uint64_t m, int directed, uint64_t seed) {
    const uint64_t n = 1ull << scale;
    uint32_t* eu = (uint32_t*)xmalloc((m ? m : 1) * sizeof(uint32_t));
    uint32_t* ev = (uint32_t*)xmalloc((m ? m : 1) * sizeof(uint32_t));
    orc_rmat_draw(scale, m, seed, eu, ev);
    orc_csr* g = orc_from_edge_list(n, eu, ev, m, directed);
    free(eu);
    free(ev);
    return g;
}

orc_csr* orc_gen_rmat(uint32_t scale, uint32_t edgefactor, int directed, uint64_t seed) {
    return orc_gen_rmat_edges(scale, (uint64_t)edgefactor << scale, directed, seed);
}

/* ------------------------------------------------------------- transforms */

/* src/graph/transform.cpp:9-24: count, prefix, scatter in source order. */
orc_csr* orc_transpose(const orc_csr* g) {
    orc_csr* t = csr_alloc(g->n, g->m, g->flags);
    memset(t->row_ptr, 0, (g->n + 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < g->m; ++i) t->row_ptr[g->col_idx[i] + 1]++;
    for (uint64_t v = 0; v < g->n; ++v) t->row_ptr[v + 1] += t->row_ptr[v];
    uint32_t* cur = (uint32_t*)xmalloc((g->n + 1) * sizeof(uint32_t));
    memcpy(cur, t->row_ptr, g->n * sizeof(uint32_t));
    for (uint64_t u = 0; u < g->n; ++u)
        for (uint32_t i = g->row_ptr[u]; i < g->row_ptr[u + 1]; ++i)
            t->col_idx[cur[g->col_idx[i]]++] = (uint32_t)u;
    free(cur);
    return t;
}

static orc_csr* csr_copy(const orc_csr* g) {
    orc_csr* c = csr_alloc(g->n, g->m, g->flags);
    memcpy(c->row_ptr, g->row_ptr, (g->n + 1) * sizeof(uint32_t));
    memcpy(c->col_idx, g->col_idx, g->m * sizeof(uint32_t));
    return c;
}

/* Merge of two sorted lists without duplicates (src/graph/transform.cpp:33-45). */
static uint32_t merge_lists(const uint32_t* a, const uint32_t* ae, const uint32_t* b,
                            const uint32_t* be, uint32_t* out) {
    uint32_t k = 0;
    while (a != ae || b != be) {
        uint32_t x;
        if (b == be || (a != ae && *a < *b)) x = *a++;
        else if (a == ae || *b < *a) x = *b++;
        else { x = *a++; ++b; }
        if (out) out[k] = x;
        ++k;
    }
    return k;
}

/* src/graph/transform.cpp:26-57: undirected inputs unchanged; directed ones
 * become the union of G and its transpose, flagged sorted + dedup. */
orc_csr* orc_symmetrize(const orc_csr* g) {
    if (!(g->flags & ORC_FLAG_DIRECTED)) return csr_copy(g);
    orc_csr* t = orc_transpose(g);
    const uint64_t n = g->n;
    uint32_t* rp = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    for (uint64_t v = 0; v < n; ++v)
        rp[v + 1] = rp[v] + merge_lists(g->col_idx + g->row_ptr[v], g->col_idx + g->row_ptr[v + 1],
                                        t->col_idx + t->row_ptr[v], t->col_idx + t->row_ptr[v + 1],
                                        NULL);
    uint32_t* ci = (uint32_t*)xmalloc((uint64_t)rp[n] * sizeof(uint32_t));
    for (uint64_t v = 0; v < n; ++v)
        merge_lists(g->col_idx + g->row_ptr[v], g->col_idx + g->row_ptr[v + 1],
                    t->col_idx + t->row_ptr[v], t->col_idx + t->row_ptr[v + 1], ci + rp[v]);
    orc_csr_free(t);
    orc_csr* s = (orc_csr*)xmalloc(sizeof *s);
    s->n = n;
    s->m = rp[n];
    s->flags = ORC_FLAG_SORTED | ORC_FLAG_DEDUP;
    s->row_ptr = rp;
    s->col_idx = ci;
    return s;
}

/* src/graph/transform.cpp:59-76: vertex v becomes perm[v]; lists re-sorted. */
orc_csr* orc_permute(const orc_csr* g, const uint32_t* perm) {
    const uint64_t n = g->n;
    uint32_t* inv = (uint32_t*)xmalloc((n + 1) * sizeof(uint32_t));
    for (uint64_t v = 0; v < n; ++v) inv[perm[v]] = (uint32_t)v;
    orc_csr* p = csr_alloc(n, g->m, g->flags);
    p->row_ptr[0] = 0;
    for (uint64_t nv = 0; nv < n; ++nv) p->row_ptr[nv + 1] = p->row_ptr[nv] + deg(g, inv[nv]);
    for (uint64_t nv = 0; nv < n; ++nv) {
        uint32_t* out = p->col_idx + p->row_ptr[nv];
        uint32_t k = 0, old = inv[nv];
        for (uint32_t i = g->row_ptr[old]; i < g->row_ptr[old + 1]; ++i) out[k++] = perm[g->col_idx[i]];
        qsort(out, k, sizeof(uint32_t), cmp_u32);
    }
    free(inv);
    return p;
}

/* src/graph/reorder.cpp:20-25: Fisher-Yates with the project RNG. */
void orc_random_perm(uint64_t n, uint64_t seed, uint32_t* p) {
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; ++i) p[i] = (uint32_t)i;
    for (uint64_t i = n; i > 1; --i) {
        uint64_t j = orc_rng_below(&s, i);
        uint32_t t = p[i - 1];
        p[i - 1] = p[j];
        p[j] = t;
    }
}

/* Orderings of src/graph/reorder.cpp:30-90, on a symmetric graph. */
static const orc_csr* g_sort_graph; /* qsort has no context argument */
static uint32_t deg_of(const orc_csr* g, uint32_t v) { return g->row_ptr[v + 1] - g->row_ptr[v]; }

static int cmp_deg_desc_id(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    uint32_t dx = deg_of(g_sort_graph, x), dy = deg_of(g_sort_graph, y);
    if (dx != dy) return dx > dy ? -1 : 1;
    return x < y ? -1 : x > y;
}

static int cmp_deg_asc_id(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    uint32_t dx = deg_of(g_sort_graph, x), dy = deg_of(g_sort_graph, y);
    if (dx != dy) return dx < dy ? -1 : 1;
    return x < y ? -1 : x > y;
}

/* degreePerm (reorder.cpp:27-38): new ids by descending degree, ties by id
 * (a stable sort of the identity). */
void orc_reorder_degree(const orc_csr* g, uint32_t* perm) {
    uint32_t* order = (uint32_t*)xmalloc(g->n * sizeof(uint32_t) + 4);
    for (uint64_t v = 0; v < g->n; ++v) order[v] = (uint32_t)v;
    g_sort_graph = g;
    qsort(order, g->n, sizeof(uint32_t), cmp_deg_desc_id);
    for (uint64_t i = 0; i < g->n; ++i) perm[order[i]] = (uint32_t)i;
    free(order);
}

/* cmBfs (reorder.cpp:40-62): breadth-first from start over unmarked
 * vertices; each vertex's newly marked neighbours are appended sorted by
 * (degree, id).  Appends to out[*len]; returns where the last level begins. */
static uint64_t cm_bfs(const orc_csr* g, uint32_t start, uint8_t* mark, uint32_t* out, uint64_t* len,
                       uint32_t* scratch) {
    uint64_t head = *len, last = head;
    out[(*len)++] = start;
    mark[start] = 1;
    g_sort_graph = g;
    while (head < *len) {
        const uint64_t level_end = *len;
        last = head;
        for (; head < level_end; ++head) {
            const uint32_t u = out[head];
            uint64_t k = 0;
            for (uint32_t i = g->row_ptr[u]; i < g->row_ptr[u + 1]; ++i) {
                const uint32_t w = g->col_idx[i];
                if (!mark[w]) {
                    mark[w] = 1;
                    scratch[k++] = w;
                }
            }
            qsort(scratch, k, sizeof(uint32_t), cmp_deg_asc_id);
            memcpy(out + *len, scratch, k * sizeof(uint32_t));
            *len += k;
        }
    }
    return last;
}

/* rcmPerm (reorder.cpp:64-92): components in the order of their first vertex
 * by (degree, id); per component one probe pass from that vertex, whose last
 * level's first lowest-degree vertex starts the real pass; the whole order
 * reversed at the end. */
void orc_reorder_rcm(const orc_csr* g, uint32_t* perm) {
    const uint64_t n = g->n;
    uint32_t* by_degree = (uint32_t*)xmalloc(n * sizeof(uint32_t) + 4);
    uint32_t* order = (uint32_t*)xmalloc(n * sizeof(uint32_t) + 4);
    uint32_t* tmp = (uint32_t*)xmalloc(n * sizeof(uint32_t) + 4);
    uint32_t* scratch = (uint32_t*)xmalloc(n * sizeof(uint32_t) + 4);
    uint8_t* mark = (uint8_t*)calloc(n + 1, 1);
    uint8_t* probe = (uint8_t*)calloc(n + 1, 1);
    for (uint64_t v = 0; v < n; ++v) by_degree[v] = (uint32_t)v;
    g_sort_graph = g;
    qsort(by_degree, n, sizeof(uint32_t), cmp_deg_asc_id);
    uint64_t len = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t s = by_degree[i];
        if (mark[s]) continue;
        uint64_t tl = 0;
        const uint64_t last = cm_bfs(g, s, probe, tmp, &tl, scratch);
        uint32_t start = tmp[last];
        for (uint64_t j = last; j < tl; ++j)
            if (deg_of(g, tmp[j]) < deg_of(g, start)) start = tmp[j];
        cm_bfs(g, start, mark, order, &len, scratch);
    }
    for (uint64_t i = 0; i < n; ++i) perm[order[i]] = (uint32_t)(n - 1 - i);
    free(by_degree);
    free(order);
    free(tmp);
    free(scratch);
    free(mark);
    free(probe);
}

/* locality (reorder.cpp:111-125): mean |u - v| over stored entries and the
 * fraction with u / 64 == v / 64. */
void orc_locality(const orc_csr* g, double* mean_gap, double* same_block64) {
    double gap = 0;
    uint64_t same = 0;
    for (uint64_t u = 0; u < g->n; ++u)
        for (uint32_t i = g->row_ptr[u]; i < g->row_ptr[u + 1]; ++i) {
            const uint64_t w = g->col_idx[i];
            gap += u > w ? (double)(u - w) : (double)(w - u);
            same += (u >> 6) == (w >> 6);
        }
    *mean_gap = g->m ? gap / (double)g->m : 0;
    *same_block64 = g->m ? (double)same / (double)g->m : 0;
}

/* src/graph/csr.cpp:86-104 */
int orc_validate(const orc_csr* g) {
    if (g->m >= (1ull << 32)) return 1;
    if (g->row_ptr[0] != 0) return 2;
    if (g->row_ptr[g->n] != g->m) return 3;
    int strict = (g->flags & ORC_FLAG_SORTED) && (g->flags & ORC_FLAG_DEDUP);
    for (uint64_t v = 0; v < g->n; ++v) {
        uint32_t b = g->row_ptr[v], e = g->row_ptr[v + 1];
        if (e < b) return 4;
        for (uint32_t i = b; i < e; ++i) {
            uint32_t u = g->col_idx[i];
            if (u >= g->n) return 5;
            if (strict) {
                if (u == v) return 6;
                if (i > b && g->col_idx[i - 1] >= u) return 7;
            }
        }
    }
    return 0;
}

/* -------------------------------------------------------------------- BFS */

/* src/cpu/bfs_cpu.cpp:27-45: queue BFS, the exactness oracle. */
void orc_bfs_serial(const orc_csr* g, uint32_t source, uint32_t* dist) {
    for (uint64_t v = 0; v < g->n; ++v) dist[v] = ORC_UNREACHED;
    uint32_t* q = (uint32_t*)xmalloc(g->n * sizeof(uint32_t));
    uint64_t head = 0, tail = 0;
    dist[source] = 0;
    q[tail++] = source;
    while (head < tail) {
        uint32_t u = q[head++];
        uint32_t du = dist[u] + 1;
        for (uint32_t i = g->row_ptr[u]; i < g->row_ptr[u + 1]; ++i) {
            uint32_t w = g->col_idx[i];
            if (dist[w] == ORC_UNREACHED) {
                dist[w] = du;
                q[tail++] = w;
            }
        }
    }
    free(q);
}

static void trace_push(orc_level* tr, int cap, int* count, uint32_t level, char dir,
                       uint64_t frontier, uint64_t edges) {
    if (tr && *count < cap) {
        tr[*count].level = level;
        tr[*count].direction = (uint32_t)dir;
        tr[*count].frontier = frontier;
        tr[*count].edges = edges;
    }
    (*count)++;
}

/* src/cpu/bfs_cpu.cpp:227-283 (bfsDO) with the level steps of :87-115
 * (top-down) and :137-157 (bottom-up), run serially: the frontier sets and
 * every counter the direction rule reads are the same in any schedule. */
int orc_bfs_do(const orc_csr* g, uint32_t source, uint32_t* dist, double alpha, double beta,
               orc_level* trace, int cap) {
    const uint64_t n = g->n, words = (n + 63) / 64;
    for (uint64_t v = 0; v < n; ++v) dist[v] = ORC_UNREACHED;
    uint32_t* queue = (uint32_t*)xmalloc(n * sizeof(uint32_t));
    uint32_t* nextq = (uint32_t*)xmalloc(n * sizeof(uint32_t));
    uint64_t* front = (uint64_t*)calloc(words + 1, sizeof(uint64_t));
    uint64_t* next = (uint64_t*)calloc(words + 1, sizeof(uint64_t));
    dist[source] = 0;
    queue[0] = source;
    uint64_t fsize = 1, edges_to_check = g->m, scout = deg(g, source);
    uint32_t level = 0;
    int count = 0;
    while (fsize > 0) {
        if ((double)scout > (double)edges_to_check / alpha) {
            memset(front, 0, words * sizeof(uint64_t));
            for (uint64_t i = 0; i < fsize; ++i) front[queue[i] >> 6] |= 1ull << (queue[i] & 63);
            uint64_t awake = fsize, old_awake;
            do {
                old_awake = awake;
                memset(next, 0, words * sizeof(uint64_t));
                uint64_t found = 0, examined = 0;
                for (uint64_t v = 0; v < n; ++v) {
                    if (dist[v] != ORC_UNREACHED) continue;
                    uint32_t b = g->row_ptr[v], e = g->row_ptr[v + 1], p = b;
                    for (; p != e; ++p) {
                        uint32_t u = g->col_idx[p];
                        if ((front[u >> 6] >> (u & 63)) & 1) {
                            dist[v] = level + 1;
                            next[v >> 6] |= 1ull << (v & 63);
                            ++found;
                            ++p;
                            break;
                        }
                    }
                    examined += p - b;
                }
                trace_push(trace, cap, &count, level, 'B', old_awake, examined);
                awake = found;
                uint64_t* t = front;
                front = next;
                next = t;
                ++level;
            } while (awake >= old_awake || (double)awake > (double)n / beta);
            fsize = 0;
            for (uint64_t w = 0; w < words; ++w) {
                uint64_t word = front[w];
                while (word) {
                    uint64_t v = w * 64 + (uint64_t)__builtin_ctzll(word);
                    word &= word - 1;
                    if (v < n) queue[fsize++] = (uint32_t)v;
                }
            }
            scout = 1;
        } else {
            edges_to_check -= edges_to_check < scout ? edges_to_check : scout;
            uint64_t nsize = 0, nscout = 0, examined = 0;
            for (uint64_t i = 0; i < fsize; ++i) {
                uint32_t u = queue[i];
                examined += deg(g, u);
                for (uint32_t k = g->row_ptr[u]; k < g->row_ptr[u + 1]; ++k) {
                    uint32_t w = g->col_idx[k];
                    if (dist[w] == ORC_UNREACHED) {
                        dist[w] = level + 1;
                        nscout += deg(g, w);
                        nextq[nsize++] = w;
                    }
                }
            }
            trace_push(trace, cap, &count, level, 'T', fsize, examined);
            scout = nscout;
            uint32_t* t = queue;
            queue = nextq;
            nextq = t;
            fsize = nsize;
            ++level;
        }
    }
    free(queue);
    free(nextq);
    free(front);
    free(next);
    return count;
}

/* src/bench/main.cpp:130-149 (largestComponent): component ids by BFS from
 * each unassigned vertex in id order; the first largest one wins. */
static uint8_t* largest_component(const orc_csr* g) {
    const uint64_t n = g->n;
    uint32_t* comp = (uint32_t*)xmalloc((n + 1) * sizeof(uint32_t));
    uint32_t* q = (uint32_t*)xmalloc((n + 1) * sizeof(uint32_t));
    for (uint64_t v = 0; v < n; ++v) comp[v] = ORC_UNREACHED;
    uint32_t best = 0, id = 0;
    uint64_t best_size = 0;
    for (uint64_t r = 0; r < n; ++r) {
        if (comp[r] != ORC_UNREACHED) continue;
        uint64_t head = 0, tail = 0;
        comp[r] = id;
        q[tail++] = (uint32_t)r;
        while (head < tail) {
            uint32_t u = q[head++];
            for (uint32_t i = g->row_ptr[u]; i < g->row_ptr[u + 1]; ++i)
                if (comp[g->col_idx[i]] == ORC_UNREACHED) {
                    comp[g->col_idx[i]] = id;
                    q[tail++] = g->col_idx[i];
                }
        }
        if (tail > best_size) {
            best_size = tail;
            best = id;
        }
        ++id;
    }
    uint8_t* mask = (uint8_t*)xmalloc(n + 1);
    for (uint64_t v = 0; v < n; ++v) mask[v] = comp[v] == best;
    free(comp);
    free(q);
    return mask;
}

/* src/bench/main.cpp:155-169 (pickSources): distinct uniform picks with
 * degree > 0 inside the largest component, from SplitMix64(seed). */
int orc_pick_sources(const orc_csr* g, int count, uint64_t seed, int any_component, uint32_t* out) {
    const uint64_t n = g->n;
    uint8_t* ok;
    if (any_component) {
        ok = (uint8_t*)xmalloc(n + 1);
        memset(ok, 1, n + 1);
    } else {
        ok = largest_component(g);
    }
    uint64_t candidates = 0;
    for (uint64_t v = 0; v < n; ++v) candidates += ok[v] && deg(g, v) > 0;
    if ((uint64_t)count > candidates) count = (int)candidates;
    uint8_t* used = (uint8_t*)calloc(n + 1, 1);
    uint64_t s = seed;
    int k = 0;
    while (k < count) {
        uint32_t v = (uint32_t)orc_rng_below(&s, n);
        if (ok[v] && deg(g, v) > 0 && !used[v]) {
            used[v] = 1;
            out[k++] = v;
        }
    }
    free(ok);
    free(used);
    return count;
}

/* src/bench/main.cpp:329-332: TEPS denominator. */
uint64_t orc_component_edges(const orc_csr* g, const uint32_t* dist) {
    uint64_t s = 0;
    for (uint64_t v = 0; v < g->n; ++v)
        if (dist[v] != ORC_UNREACHED) s += deg(g, v);
    return s / 2;
}

/* --------------------------------------------------------------- PageRank */

/* src/cpu/pagerank_cpu.cpp:9-13 */
void orc_out_degrees(const orc_csr* g, uint32_t* od) {
    for (uint64_t v = 0; v < g->n; ++v) od[v] = deg(g, v);
}

/* src/cpu/pagerank_cpu.cpp:20-53 (pagerank, serial): Jacobi pull in double,
 * r0 = 1/n, dangling mass redistributed uniformly, L1 change per iteration. */
int orc_pagerank_serial(const orc_csr* in, const uint32_t* outdeg, double* r, double d, int iters,
                        double tol, double* last_delta) {
    const uint64_t n = in->n;
    if (last_delta) *last_delta = 0;
    if (n == 0) return 0;
    const double base = (1.0 - d) / (double)n;
    double* contrib = (double*)xmalloc(n * sizeof(double));
    double* next = (double*)xmalloc(n * sizeof(double));
    for (uint64_t v = 0; v < n; ++v) r[v] = 1.0 / (double)n;
    int done = 0;
    for (int it = 0; it < iters; ++it) {
        double dangling = 0;
        for (uint64_t u = 0; u < n; ++u) {
            if (outdeg[u]) contrib[u] = r[u] / outdeg[u];
            else {
                contrib[u] = 0;
                dangling += r[u];
            }
        }
        const double add = base + d * dangling / (double)n;
        double delta = 0;
        for (uint64_t v = 0; v < n; ++v) {
            double s = 0;
            for (uint32_t i = in->row_ptr[v]; i < in->row_ptr[v + 1]; ++i) s += contrib[in->col_idx[i]];
            next[v] = add + d * s;
            delta += fabs(next[v] - r[v]);
        }
        memcpy(r, next, n * sizeof(double));
        done = it + 1;
        if (last_delta) *last_delta = delta;
        if (tol > 0 && delta < tol) break;
    }
    free(contrib);
    free(next);
    return done;
}

static const double* g_sort_ref;
static int cmp_rank_desc(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    if (g_sort_ref[x] > g_sort_ref[y]) return -1;
    if (g_sort_ref[x] < g_sort_ref[y]) return 1;
    return x < y ? -1 : x > y;
}

/* src/cpu/pagerank_cpu.hpp:42-60 (checkRanks): L1, sum, and the max relative
 * error over the reference's top-1000 vertices (ties broken by id here). */
static void check_ranks(const double* ref, const float* gf, const double* gd, uint64_t n, double* l1,
                        double* max_rel, double* sum) {
    double a = 0, s = 0, mr = 0;
    for (uint64_t v = 0; v < n; ++v) {
        double x = gf ? (double)gf[v] : gd[v];
        a += fabs(ref[v] - x);
        s += x;
    }
    uint64_t k = n < 1000 ? n : 1000;
    if (k) {
        uint32_t* idx = (uint32_t*)xmalloc(n * sizeof(uint32_t));
        for (uint64_t v = 0; v < n; ++v) idx[v] = (uint32_t)v;
        g_sort_ref = ref;
        qsort(idx, n, sizeof(uint32_t), cmp_rank_desc);
        for (uint64_t i = 0; i < k; ++i) {
            uint32_t v = idx[i];
            double x = gf ? (double)gf[v] : gd[v];
            double e = fabs(ref[v] - x) / ref[v];
            if (e > mr) mr = e;
        }
        free(idx);
    }
    *l1 = a;
    *sum = s;
    *max_rel = mr;
}

void orc_check_ranks_f32(const double* ref, const float* got, uint64_t n, double* l1, double* mr,
                         double* sum) {
    check_ranks(ref, got, NULL, n, l1, mr, sum);
}

void orc_check_ranks_f64(const double* ref, const double* got, uint64_t n, double* l1, double* mr,
                         double* sum) {
    check_ranks(ref, NULL, got, n, l1, mr, sum);
}

/* src/cpu/pagerank_cpu.hpp:80-84 (gsNoWorseThanJacobi) */
int orc_gs_no_worse(double gs_l1, double gs_rel, double gs_sum, double j_l1, double j_rel) {
    const double budget = j_l1 > 1e-4 ? j_l1 : 1e-4;
    const double relb = j_rel * (1 + 1e-4) > 1e-3 ? j_rel * (1 + 1e-4) : 1e-3;
    return gs_l1 <= budget && fabs(gs_sum - 1.0) <= budget && gs_rel <= relb;
}

/* ------------------------------------------------------- selector MLP (ref) */

/* Straightforward double-precision forward/backward of
 *   out = W3 relu(W2 relu(W1 x + b1) + b2) + b3,
 *   loss = sum(mask * (out - y)^2) / max(1, sum(mask)).
 * No counterpart in the reference (the selector is new); it is the CPU check
 * for the GPU training kernels. */
double orc_mlp_loss_grad(int nf, int nh, int no, const float* P, int batch, const float* x,
                         const float* y, const float* mask, float* G) {
    const float *w1 = P, *b1 = w1 + nh * nf, *w2 = b1 + nh, *b2 = w2 + nh * nh, *w3 = b2 + nh,
                *b3 = w3 + no * nh;
    const size_t np = (size_t)nh * nf + nh + (size_t)nh * nh + nh + (size_t)no * nh + no;
    double* g = (double*)calloc(np, sizeof(double));
    double *gw1 = g, *gb1 = gw1 + nh * nf, *gw2 = gb1 + nh, *gb2 = gw2 + nh * nh, *gw3 = gb2 + nh,
           *gb3 = gw3 + no * nh;
    double* h1 = (double*)xmalloc(nh * sizeof(double));
    double* h2 = (double*)xmalloc(nh * sizeof(double));
    double* dh1 = (double*)xmalloc(nh * sizeof(double));
    double* dh2 = (double*)xmalloc(nh * sizeof(double));
    double* dout = (double*)xmalloc(no * sizeof(double));
    double msum = 0, loss = 0;
    for (int b = 0; b < batch; ++b)
        for (int o = 0; o < no; ++o) msum += mask[b * no + o];
    const double scale = msum > 1 ? 1.0 / msum : 1.0;
    for (int b = 0; b < batch; ++b) {
        const float* xb = x + (size_t)b * nf;
        for (int j = 0; j < nh; ++j) {
            double s = b1[j];
            for (int f = 0; f < nf; ++f) s += (double)w1[j * nf + f] * xb[f];
            h1[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < nh; ++j) {
            double s = b2[j];
            for (int k = 0; k < nh; ++k) s += (double)w2[j * nh + k] * h1[k];
            h2[j] = s > 0 ? s : 0;
        }
        for (int o = 0; o < no; ++o) {
            double s = b3[o];
            for (int k = 0; k < nh; ++k) s += (double)w3[o * nh + k] * h2[k];
            double mk = mask[b * no + o], e = s - y[b * no + o];
            loss += mk * e * e;
            dout[o] = 2.0 * mk * e * scale;
        }
        for (int k = 0; k < nh; ++k) dh2[k] = 0;
        for (int o = 0; o < no; ++o) {
            gb3[o] += dout[o];
            for (int k = 0; k < nh; ++k) {
                gw3[o * nh + k] += dout[o] * h2[k];
                dh2[k] += dout[o] * w3[o * nh + k];
            }
        }
        for (int k = 0; k < nh; ++k) dh2[k] = h2[k] > 0 ? dh2[k] : 0;
        for (int k = 0; k < nh; ++k) dh1[k] = 0;
        for (int j = 0; j < nh; ++j) {
            gb2[j] += dh2[j];
            for (int k = 0; k < nh; ++k) {
                gw2[j * nh + k] += dh2[j] * h1[k];
                dh1[k] += dh2[j] * w2[j * nh + k];
            }
        }
        for (int k = 0; k < nh; ++k) dh1[k] = h1[k] > 0 ? dh1[k] : 0;
        for (int j = 0; j < nh; ++j) {
            gb1[j] += dh1[j];
            for (int f = 0; f < nf; ++f) gw1[j * nf + f] += dh1[j] * xb[f];
        }
    }
    for (size_t i = 0; i < np; ++i) G[i] = (float)g[i];
    free(g);
    free(h1);
    free(h2);
    free(dh1);
    free(dh2);
    free(dout);
    return loss * scale;
}

void orc_mlp_forward(int nf, int nh, int no, const float* P, int batch, const float* x, float* out) {
    const float *w1 = P, *b1 = w1 + nh * nf, *w2 = b1 + nh, *b2 = w2 + nh * nh, *w3 = b2 + nh,
                *b3 = w3 + no * nh;
    double* h1 = (double*)xmalloc(nh * sizeof(double));
    double* h2 = (double*)xmalloc(nh * sizeof(double));
    for (int b = 0; b < batch; ++b) {
        const float* xb = x + (size_t)b * nf;
        for (int j = 0; j < nh; ++j) {
            double s = b1[j];
            for (int f = 0; f < nf; ++f) s += (double)w1[j * nf + f] * xb[f];
            h1[j] = s > 0 ? s : 0;
        }
        for (int j = 0; j < nh; ++j) {
            double s = b2[j];
            for (int k = 0; k < nh; ++k) s += (double)w2[j * nh + k] * h1[k];
            h2[j] = s > 0 ? s : 0;
        }
        for (int o = 0; o < no; ++o) {
            double s = b3[o];
            for (int k = 0; k < nh; ++k) s += (double)w3[o * nh + k] * h2[k];
            out[(size_t)b * no + o] = (float)s;
        }
    }
    free(h1);
    free(h2);
}

/* ------------------------------------------------------------ SNAP text */

/* The whole (decompressed) file; gzread passes plain text through unchanged. */
static char* read_all(const char* path, uint64_t* len, int* io_err) {
    gzFile f = gzopen(path, "rb");
    *io_err = 0;
    if (!f) {
        *io_err = 1;
        return NULL;
    }
    uint64_t cap = 1 << 20, n = 0;
    char* buf = (char*)xmalloc(cap);
    for (;;) {
        if (cap - n < (1 << 20)) {
            cap *= 2;
            buf = (char*)realloc(buf, cap);
            if (!buf) abort();
        }
        int got = gzread(f, buf + n, (unsigned)(cap - n > (1u << 30) ? (1u << 30) : cap - n));
        if (got < 0) {
            *io_err = 2;
            break;
        }
        if (got == 0) break;
        n += (uint64_t)got;
    }
    gzclose(f);
    *len = n;
    return buf;
}

static int cmp_u32_snap(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

/* src/graph/snap.cpp:17-81 (forEachEdge: the line rules and the errors, one
 * line at a time; a line of 4 MiB or more before its newline is the
 * reference's "longer than 4 MB" case of its 4 MiB read buffer) and
 * src/graph/snap.cpp:85-149 (convertSnap: dense relabelling in raw-id order,
 * then fromEdgeList's count / scatter / compact). */
int orc_convert_snap(const char* path, int directed, orc_csr** out, orc_convert_stats* st,
                     char* msg, size_t cap) {
    const uint64_t kLongLine = 4u << 20;
    int io = 0;
    uint64_t len = 0;
    char* t = read_all(path, &len, &io);
    *out = NULL;
    memset(st, 0, sizeof *st);
    if (io == 1) {
        snprintf(msg, cap, "cannot open %s", path);
        return 1;
    }
    if (io == 2) {
        free(t);
        snprintf(msg, cap, "gzread failed on %s", path);
        return 1;
    }
    edge_list e = {0};
    uint64_t line_no = 0, pos = 0;
    int bad = 0;
    while (pos < len && !bad) {
        uint64_t end = pos;
        while (end < len && t[end] != '\n') ++end; /* [pos, end): this line */
        ++line_no;
        if (end - pos >= kLongLine) {
            snprintf(msg, cap, "line longer than 4 MB in %s", path);
            bad = 1;
            break;
        }
        uint64_t p = pos;
        const uint64_t next = end + 1;
        pos = next;
        while (p < end && (t[p] == ' ' || t[p] == '\t' || t[p] == '\r')) ++p;
        if (p == end || t[p] == '#' || t[p] == '%') continue; /* blank or comment */
        uint64_t ids[2];
        for (int k = 0; k < 2; ++k) {
            while (p < end && (t[p] == ' ' || t[p] == '\t')) ++p;
            if (p == end || t[p] < '0' || t[p] > '9') {
                snprintf(msg, cap, "%s: malformed line %llu", path, (unsigned long long)line_no);
                bad = 1;
                break;
            }
            uint64_t x = 0; /* wraps modulo 2^64 like the reference's uint64_t */
            while (p < end && t[p] >= '0' && t[p] <= '9') x = x * 10 + (uint64_t)(t[p++] - '0');
            if (x >= 0xFFFFFFFFull) {
                snprintf(msg, cap, "%s: vertex ID too large on line %llu", path,
                         (unsigned long long)line_no);
                bad = 1;
                break;
            }
            ids[k] = x;
        }
        if (bad) break;
        el_push(&e, (uint32_t)ids[0], (uint32_t)ids[1]);
    }
    free(t);
    if (bad) {
        free(e.u);
        free(e.v);
        return 1;
    }
    const uint64_t total = directed ? e.size : 2 * e.size;
    st->lines = e.size;
    st->m_before = total;
    if (total >= 0xFFFFFFFFull) {
        free(e.u);
        free(e.v);
        snprintf(msg, cap, "too many edges for uint32 offsets");
        return 1;
    }
    /* distinct raw ids in increasing order; dense id = rank */
    uint32_t* ids = (uint32_t*)xmalloc(2 * e.size * sizeof(uint32_t));
    for (uint64_t i = 0; i < e.size; ++i) {
        ids[2 * i] = e.u[i];
        ids[2 * i + 1] = e.v[i];
    }
    qsort(ids, 2 * e.size, sizeof(uint32_t), cmp_u32_snap);
    uint64_t n = 0;
    for (uint64_t i = 0; i < 2 * e.size; ++i)
        if (i == 0 || ids[i] != ids[i - 1]) ids[n++] = ids[i];
    for (uint64_t i = 0; i < e.size; ++i) {
        uint32_t* a = (uint32_t*)bsearch(&e.u[i], ids, n, sizeof(uint32_t), cmp_u32_snap);
        uint32_t* b = (uint32_t*)bsearch(&e.v[i], ids, n, sizeof(uint32_t), cmp_u32_snap);
        e.u[i] = (uint32_t)(a - ids);
        e.v[i] = (uint32_t)(b - ids);
    }
    st->raw_max_id = n ? ids[n - 1] : 0;
    st->n = n;
    free(ids);
    *out = orc_from_edge_list(n, e.u, e.v, e.size, directed);
    st->m = (*out)->m;
    free(e.u);
    free(e.v);
    return 0;
}
