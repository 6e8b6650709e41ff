/*
 * sg_oracle.c -- CPU restatement of dsc-nec/subgraph's color-coding counting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it to produce the
 * numbers the CUDA path must reproduce.  Nothing in the product library links
 * or calls it.  It is pinned against the compiled reference (oracle/_ref, built
 * by oracle/build_ref.sh from the reference's own sources) through the golden
 * fixtures in tests/golden/.
 *
 * Every function restates one piece of the reference, cited by file:line of the
 * reference project:
 *   glibc rand() stream ........ CountMat.cpp:979-991 (srand/rand under colorInit)
 *   CSC construction ........... CSCGraph.hpp:95-178
 *   template adjacency ......... Graph.cpp:82-129
 *   DivideTemplates ............ DivideTemplates.cpp:6-327
 *   IndexSys ................... IndexSys.cpp:169-436
 *   per-coloring count ......... CountMat.cpp:268-322, 556-849, 851-977
 *                                DataTableColMajor.cpp:346-400, 553-567
 *   estimate / automorphisms ... CountMat.cpp:199-264, 1498-1572
 *
 * Plain C99, no dependencies.  Sizes are chosen so that the oracle runs in
 * seconds on the graphs the tests use.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_DUMMY 93620 /* Helper.hpp:7 DUMMY_VAL */

/* ------------------------------------------------------------------------- */
/* glibc TYPE_3 additive feedback generator (the default rand() state).       */
/* srandom_r seeds r[0..30] with 16807*r mod (2^31-1) (Schrage form), then    */
/* discards 310 outputs; r[i] = r[i-3] + r[i-31] (mod 2^32); rand() = r>>1.   */
/* ------------------------------------------------------------------------- */
void orc_glibc_rand(uint32_t seed, int64_t n, int32_t *out)
{
    int32_t r[31];
    if (seed == 0) seed = 1;
    int32_t word = (int32_t)seed;
    r[0] = word;
    for (int i = 1; i < 31; ++i) {
        int32_t hi = word / 127773;
        int32_t lo = word % 127773;
        word = 16807 * lo - 2836 * hi;
        if (word < 0) word += 2147483647;
        r[i] = word;
    }
    /* ring buffer of the last 31 values; front pointer f = i-3, rear = i-31 */
    uint32_t ring[31];
    for (int i = 0; i < 31; ++i) ring[i] = (uint32_t)r[i];
    /* r[31..33] = r[0..2] is the same as continuing with fptr/rptr from glibc:
     * val = state[f] += state[r].  Emulate glibc's pointer walk directly. */
    int fptr = 3, rptr = 0;
    int64_t produced = 0;
    for (int64_t step = 0; produced < n; ++step) {
        uint32_t val = ring[fptr] + ring[rptr];
        ring[fptr] = val;
        if (++fptr >= 31) { fptr = 0; ++rptr; }
        else if (++rptr >= 31) rptr = 0;
        if (step >= 310) out[produced++] = (int32_t)(val >> 1);
    }
}

/* CountMat::colorInit (CountMat.cpp:979-991) on one thread: color = rand()%k */
void orc_color(uint32_t seed, int32_t V, int32_t k, int32_t *color)
{
    orc_glibc_rand(seed, V, color);
    for (int32_t v = 0; v < V; ++v) color[v] = color[v] % k;
}

/* ------------------------------------------------------------------------- */
/* CSCGraph::createFromEdgeListFile (CSCGraph.hpp:95-178): both directions    */
/* inserted in edge order, no dedup, rows of each column sorted ascending.    */
/* ------------------------------------------------------------------------- */
static int cmp_i32(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

int orc_csc_build(int32_t V, int32_t E, const int32_t *src, const int32_t *dst,
                  int32_t *indexCol, int32_t *indexRow, int32_t *degList)
{
    for (int32_t i = 0; i < V; ++i) degList[i] = 0;
    for (int32_t i = 0; i < E; ++i) {
        if (src[i] < 0 || src[i] >= V || dst[i] < 0 || dst[i] >= V) return 1;
        degList[dst[i]]++;
        degList[src[i]]++;
    }
    indexCol[0] = 0;
    for (int32_t i = 1; i <= V; ++i) indexCol[i] = indexCol[i - 1] + degList[i - 1];
    int32_t *pos = (int32_t *)malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
    for (int32_t i = 0; i < V; ++i) pos[i] = indexCol[i];
    for (int32_t i = 0; i < E; ++i) {
        indexRow[pos[dst[i]]++] = src[i];
        indexRow[pos[src[i]]++] = dst[i];
    }
    free(pos);
    for (int32_t i = 0; i < V; ++i)
        qsort(indexRow + indexCol[i], (size_t)(indexCol[i + 1] - indexCol[i]), sizeof(int32_t), cmp_i32);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Template graphs (Graph.cpp:82-129): adjacency lists filled in edge order,  */
/* u gets v then v gets u.                                                    */
/* ------------------------------------------------------------------------- */
#define ORC_MAXV 32
#define ORC_MAXSUB 256

typedef struct {
    int nv, ne;                 /* ne = 2 * edges */
    int deg[ORC_MAXV + 1];      /* CSR offsets */
    int adj[2 * ORC_MAXV];
} orc_tgraph;

static void tg_build(orc_tgraph *g, int nv, int nedges, const int *s, const int *d)
{
    int cnt[ORC_MAXV];
    memset(cnt, 0, sizeof(cnt));
    g->nv = nv;
    g->ne = 2 * nedges;
    for (int j = 0; j < nedges; ++j) { cnt[s[j]]++; cnt[d[j]]++; }
    g->deg[0] = 0;
    for (int j = 0; j < nv; ++j) g->deg[j + 1] = g->deg[j] + cnt[j];
    int pos[ORC_MAXV];
    for (int j = 0; j < nv; ++j) pos[j] = g->deg[j];
    for (int j = 0; j < nedges; ++j) {
        g->adj[pos[s[j]]++] = d[j];
        g->adj[pos[d[j]]++] = s[j];
    }
}

/* ------------------------------------------------------------------------- */
/* DivideTemplates (DivideTemplates.cpp:6-327).                               */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;                         /* number of subs */
    orc_tgraph sub[ORC_MAXSUB];
    int node_main[ORC_MAXSUB], node_aux[ORC_MAXSUB], parents[ORC_MAXSUB];
    int cur;
} orc_divider;

static void set_nodes(int *list, int *len, int idx, int val)
{
    while (*len <= idx) list[(*len)++] = ORC_DUMMY;
    list[idx] = val;
}

typedef struct { int len_main, len_aux, len_par; } orc_lens;

/* split_nodes (DivideTemplates.cpp:153-217) + check_val (:219-246) */
static int split_nodes(orc_divider *D, int sub, int root, int rest)
{
    orc_tgraph cur = D->sub[sub];
    int src[2 * ORC_MAXV], dst[2 * ORC_MAXV], ne = 0;
    int added[2 * ORC_MAXV], na = 0;
    added[na++] = root;
    for (int i = 0; i < na; ++i) {
        int a = added[i];
        for (int j = cur.deg[a]; j < cur.deg[a + 1]; ++j) {
            int vid = cur.adj[j];
            int add_edge = 1;
            for (int k = 0; k < ne; ++k)
                if (src[k] == vid && dst[k] == a) { add_edge = 0; break; }
            if (add_edge && vid != rest) {
                src[ne] = a; dst[ne] = vid; ++ne;
                added[na++] = vid;
            }
        }
    }
    int nv;
    if (ne > 0) {
        nv = ne + 1;
        int maxv = 0;
        for (int i = 0; i < ne; ++i) {
            if (src[i] > maxv) maxv = src[i];
            if (dst[i] > maxv) maxv = dst[i];
        }
        int map[2 * ORC_MAXV + 2];
        for (int i = 0; i <= maxv; ++i) map[i] = -1;
        map[root] = 0;
        int next = 1;
        for (int i = 0; i < ne; ++i) {
            if (map[src[i]] == -1) map[src[i]] = next++;
            if (map[dst[i]] == -1) map[dst[i]] = next++;
        }
        for (int i = 0; i < ne; ++i) { src[i] = map[src[i]]; dst[i] = map[dst[i]]; }
    } else {
        nv = 1;
        src[0] = 0;
    }
    int ret = src[0];
    tg_build(&D->sub[D->cur], nv, ne, src, dst);
    D->cur++;
    return ret;
}

static void divide(orc_divider *D, orc_lens *L, int sub, int root)
{
    /* split (DivideTemplates.cpp:128-141): the first neighbour of root */
    int new_node = D->sub[sub].adj[D->sub[sub].deg[root]];
    int root_main = split_nodes(D, sub, root, new_node);
    int root_aux = split_nodes(D, sub, new_node, root);
    int main_index = D->cur - 2, aux_index = D->cur - 1;
    set_nodes(D->node_main, &L->len_main, sub, main_index);
    set_nodes(D->node_aux, &L->len_aux, sub, aux_index);
    set_nodes(D->parents, &L->len_par, main_index, sub);
    set_nodes(D->parents, &L->len_par, aux_index, sub);
    if (D->sub[main_index].nv > 1) divide(D, L, main_index, root_main);
    else {
        set_nodes(D->node_main, &L->len_main, main_index, ORC_DUMMY);
        set_nodes(D->node_aux, &L->len_aux, main_index, ORC_DUMMY);
    }
    if (D->sub[aux_index].nv > 1) divide(D, L, aux_index, root_aux);
    else {
        set_nodes(D->node_main, &L->len_main, aux_index, ORC_DUMMY);
        set_nodes(D->node_aux, &L->len_aux, aux_index, ORC_DUMMY);
    }
}

/* sort_tps (DivideTemplates.cpp:264-327): bubble sort on the parent index */
static void sort_tps(orc_divider *D)
{
    int running = 1;
    int n = D->n;
    int *P = D->parents, *M = D->node_main, *A = D->node_aux;
    while (running) {
        int swapped = 0;
        for (int i = 2; i < n; ++i) {
            if (P[i] < P[i - 1]) {
                orc_tgraph cur_tp = D->sub[i];
                int cp = P[i], cm = M[i], ca = A[i];
                if (M[i] != ORC_DUMMY) P[M[i]] = i - 1;
                if (M[i - 1] != ORC_DUMMY) P[M[i - 1]] = i;
                if (A[i] != ORC_DUMMY) P[A[i]] = i - 1;
                if (A[i - 1] != ORC_DUMMY) P[A[i - 1]] = i;
                if (M[P[i]] == i) M[P[i]] = i - 1;
                else if (A[P[i]] == i) A[P[i]] = i - 1;
                if (M[P[i - 1]] == i - 1) M[P[i - 1]] = i;
                else if (A[P[i - 1]] == i - 1) A[P[i - 1]] = i;
                D->sub[i] = D->sub[i - 1];
                P[i] = P[i - 1]; M[i] = M[i - 1]; A[i] = A[i - 1];
                D->sub[i - 1] = cur_tp;
                P[i - 1] = cp; M[i - 1] = cm; A[i - 1] = ca;
                swapped = 1;
            }
        }
        if (!swapped) running = 0;
    }
}

/* ------------------------------------------------------------------------- */
/* IndexSys (IndexSys.cpp:9-57, 169-436).                                     */
/* ------------------------------------------------------------------------- */
int orc_comb(int n, int k) /* IndexSys.cpp:206-220 */
{
    if (k > n) return 0;
    if (k * 2 > n) k = n - k;
    if (k == 0) return 1;
    int r = n;
    for (int i = 2; i <= k; ++i) { r *= (n - i + 1); r /= i; }
    return r;
}

static void perm_init(int *p, int size) { for (int i = 0; i < size; ++i) p[i] = i + 1; }
static void perm_next(int *p, int size, int colors) /* IndexSys.cpp:228-243 */
{
    for (int i = size - 1; i >= 0; --i) {
        if (p[i] < colors - (size - i - 1)) {
            p[i]++;
            for (int j = i + 1; j < size; ++j) p[j] = p[j - 1] + 1;
            break;
        }
    }
}

static int color_hash(const int *p, int size) /* IndexSys.cpp:303-313 */
{
    int c = 0;
    for (int i = 0; i < size; ++i) c += orc_comb(p[i] - 1, i + 1);
    return c;
}

/* ------------------------------------------------------------------------- */
/* The plan: sub-template list plus index tables.                             */
/* ------------------------------------------------------------------------- */
typedef struct {
    int k;                      /* colors = template size */
    int nsub;
    int size[ORC_MAXSUB];
    int main_[ORC_MAXSUB], aux_[ORC_MAXSUB], parent[ORC_MAXSUB];
    int *c2c[ORC_MAXSUB];       /* comb-to-count: lex index -> column   */
    int *msplit[ORC_MAXSUB];    /* [L_s][S_s] main column per split    */
    int *asplit[ORC_MAXSUB];    /* [L_s][S_s] aux column per split     */
    int nsplit[ORC_MAXSUB];     /* S_s */
    int tlen[ORC_MAXSUB];       /* L_s = C(k, |s|) */
    int aut;                    /* automorphism count */
} orc_plan;

static int automorph_zero(const orc_tgraph *t, const int *map, int nm) /* CountMat.cpp:1510-1546 */
{
    for (int i = 0; i < nm; ++i) {
        int di = t->deg[i + 1] - t->deg[i];
        int dm = t->deg[map[i] + 1] - t->deg[map[i]];
        if (di != dm) return 0;
        const int *adj = t->adj + t->deg[i];
        const int *adjm = t->adj + t->deg[map[i]];
        for (int j = 0; j < di; ++j) {
            int u = adj[j], match = 0;
            for (int k = 0; k < di; ++k)
                if (u == map[adjm[k]]) match = 1;
            if (!match) return 0;
        }
    }
    return 1;
}

static int automorph_rec(const orc_tgraph *t, int *map, int nm, const int *rest, int nr) /* :1548-1572 */
{
    if (nr == 0) return automorph_zero(t, map, nm);
    int count = 0;
    int nrest[ORC_MAXV];
    for (int i = 0; i < nr; ++i) {
        map[nm] = rest[i];
        int q = 0;
        for (int j = 0; j < nr; ++j) if (j != i) nrest[q++] = rest[j];
        count += automorph_rec(t, map, nm + 1, nrest, q);
    }
    return count;
}

orc_plan *orc_plan_create(int nv, int nedges, const int *src, const int *dst, int want_automorphisms)
{
    if (nv < 1 || nv > ORC_MAXV || nedges != nv - 1) return NULL;
    orc_divider *D = (orc_divider *)calloc(1, sizeof(orc_divider));
    orc_lens L = {0, 0, 0};
    tg_build(&D->sub[0], nv, nedges, src, dst);
    D->cur = 1;
    set_nodes(D->parents, &L.len_par, 0, ORC_DUMMY);
    if (nv > 1) divide(D, &L, 0, 0);
    else {
        set_nodes(D->node_main, &L.len_main, 0, ORC_DUMMY);
        set_nodes(D->node_aux, &L.len_aux, 0, ORC_DUMMY);
    }
    D->n = D->cur;
    sort_tps(D);

    orc_plan *P = (orc_plan *)calloc(1, sizeof(orc_plan));
    int k = nv;
    P->k = k;
    P->nsub = D->n;
    for (int s = 0; s < D->n; ++s) {
        P->size[s] = D->sub[s].nv;
        P->main_[s] = D->node_main[s];
        P->aux_[s] = D->node_aux[s];
        P->parent[s] = D->parents[s];
        P->tlen[s] = orc_comb(k, P->size[s]);
    }
    /* index tables, restating gen_index/gen_colors/gen_comb_hash_table */
    for (int s = 0; s < P->nsub; ++s) {
        int sz = P->size[s];
        int L_s = P->tlen[s];
        P->c2c[s] = (int *)malloc(sizeof(int) * L_s);
        int perm[ORC_MAXV];
        perm_init(perm, sz);
        int msz = 0, asz = 0, S = 0;
        if (sz > 1) {
            msz = P->size[P->main_[s]];
            asz = P->size[P->aux_[s]];
            S = orc_comb(sz, msz);
            P->msplit[s] = (int *)malloc(sizeof(int) * L_s * S);
            P->asplit[s] = (int *)malloc(sizeof(int) * L_s * S);
        }
        P->nsplit[s] = S;
        for (int n = 0; n < L_s; ++n) {
            P->c2c[s][n] = color_hash(perm, sz);
            if (sz > 1) {
                /* _index_tmp[sz-2][msz-1] / [asz-1]: lex subsets of positions */
                int pm[ORC_MAXV], pa[ORC_MAXV];
                int colors_main[ORC_MAXV], colors_aux[ORC_MAXV];
                for (int main_itr = 0; main_itr < S; ++main_itr) {
                    int aux_itr = S - 1 - main_itr;
                    perm_init(pm, msz);
                    for (int t = 0; t < main_itr; ++t) perm_next(pm, msz, sz);
                    perm_init(pa, asz);
                    for (int t = 0; t < aux_itr; ++t) perm_next(pa, asz, sz);
                    for (int j = 0; j < msz; ++j) colors_main[j] = perm[pm[j] - 1];
                    for (int j = 0; j < asz; ++j) colors_aux[j] = perm[pa[j] - 1];
                    P->msplit[s][n * S + main_itr] = color_hash(colors_main, msz);
                    P->asplit[s][n * S + main_itr] = color_hash(colors_aux, asz);
                }
            }
            perm_next(perm, sz, k);
        }
    }
    P->aut = 1;
    if (want_automorphisms) {
        int map[ORC_MAXV], rest[ORC_MAXV];
        for (int i = 0; i < nv; ++i) rest[i] = i;
        P->aut = automorph_rec(&D->sub[0], map, 0, rest, nv);
    }
    free(D);
    return P;
}

void orc_plan_destroy(orc_plan *P)
{
    if (!P) return;
    for (int s = 0; s < P->nsub; ++s) {
        free(P->c2c[s]);
        free(P->msplit[s]);
        free(P->asplit[s]);
    }
    free(P);
}

int orc_plan_nsub(const orc_plan *P) { return P->nsub; }
int orc_plan_k(const orc_plan *P) { return P->k; }
int orc_plan_aut(const orc_plan *P) { return P->aut; }
void orc_plan_sub(const orc_plan *P, int s, int *info /* size, main, aux, parent, L_s, S_s */)
{
    info[0] = P->size[s]; info[1] = P->main_[s]; info[2] = P->aux_[s];
    info[3] = P->parent[s]; info[4] = P->tlen[s]; info[5] = P->nsplit[s];
}
void orc_plan_tables(const orc_plan *P, int s, int *c2c, int *msplit, int *asplit)
{
    int L = P->tlen[s], S = P->nsplit[s];
    memcpy(c2c, P->c2c[s], sizeof(int) * L);
    if (S > 0) {
        memcpy(msplit, P->msplit[s], sizeof(int) * L * S);
        memcpy(asplit, P->asplit[s], sizeof(int) * L * S);
    }
}

/* ------------------------------------------------------------------------- */
/* One coloring of the dynamic program.                                       */
/*   mode 0: the reference's default path (isPruned=1, useSPMM=1): FP32      */
/*           tables, first non-bottom sub scaled by 1e-12 through double,    */
/*           root accumulated per vertex in double (CountMat.cpp:556-849,    */
/*           DataTableColMajor.cpp:346-400).                                  */
/*   mode 1: FP64 tables, no scaling (the high-precision oracle).             */
/*   mode 2: isPruned=0 on a CSC graph (CountMat.cpp:851-977): FP32, no      */
/*           scaling, FP32 root; for every output i (lex) and split j one     */
/*           SpMV adds the aux column onto the buffer _bufVec, zeroed only at */
/*           CountMat::initialization (CountMat.cpp:52-59, 931;               */
/*           CSCGraph.hpp:219-239), then obj += bufVec * main                 */
/*           (arrayWiseFMANaive, DataTableColMajor.cpp:502-510).  `state`     */
/*           (V floats, optional) is that buffer, carried in and out.         */
/*   mode 3: isPruned=0 on a CSRGraph: the same, but the SpMV overwrites its  */
/*           output (CSRGraph::SpMVNaiveFull, CSRGraph.cpp:190-208): a fresh */
/*           aggregation for every split.                                     */
/* Tables are column-major [L][V] like DataTableColMajor.                     */
/* root_out (optional) receives the per-vertex root value (double).           */
/* ------------------------------------------------------------------------- */
static double count_original_acc(const int32_t *indexCol, const int32_t *indexRow, int32_t V, const orc_plan *P,
                                 const int32_t *color, float *buf, double *root_out)
{
    int n = P->nsub, k = P->k, bottom = n - 1;
    size_t Vs = (size_t)V;
    float **tf = (float **)calloc((size_t)n, sizeof(float *));
    double countSum = 0.0;
    for (int s = n - 1; s >= 0; --s) {
        int sz = P->size[s];
        if (sz == 1) {
            if (s == bottom) {
                tf[s] = (float *)calloc((size_t)k * Vs, sizeof(float));
                for (int32_t v = 0; v < V; ++v) tf[s][(size_t)P->c2c[s][color[v]] * Vs + v] = 1.0f;
            }
            continue;
        }
        int m = P->main_[s], a = P->aux_[s];
        int mt = P->size[m] == 1 ? bottom : m;
        int at = P->size[a] == 1 ? bottom : a;
        int Ls = P->tlen[s], S = P->nsplit[s];
        float *out = (float *)calloc(s > 0 ? (size_t)Ls * Vs : Vs, sizeof(float));
        for (int i = 0; i < Ls; ++i) {
            float *obj = s > 0 ? out + (size_t)P->c2c[s][i] * Vs : out;
            for (int j = 0; j < S; ++j) {
                const float *x = tf[at] + (size_t)P->asplit[s][i * S + j] * Vs;
                const float *mm = tf[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                for (int32_t v = 0; v < V; ++v) {
                    float b = buf[v];
                    for (int32_t e = indexCol[v]; e < indexCol[v + 1]; ++e) b = b + x[indexRow[e]];
                    buf[v] = b;
                    float prod = b * mm[v];
                    obj[v] = obj[v] + prod;
                }
            }
        }
        if (s > 0) tf[s] = out;
        else {
            for (int32_t v = 0; v < V; ++v) countSum += out[v];
            if (root_out) for (int32_t v = 0; v < V; ++v) root_out[v] = out[v];
            free(out);
        }
        if (P->size[m] > 1) { free(tf[m]); tf[m] = NULL; }
        if (P->size[a] > 1) { free(tf[a]); tf[a] = NULL; }
    }
    for (int s = 0; s < n; ++s) free(tf[s]);
    free(tf);
    return countSum;
}

double orc_count_coloring_state(const int32_t *indexCol, const int32_t *indexRow, int32_t V, const orc_plan *P,
                                const int32_t *color, int mode, float *state, double *root_out);

double orc_count_coloring(const int32_t *indexCol, const int32_t *indexRow, int32_t V,
                          const orc_plan *P, const int32_t *color, int mode, double *root_out)
{
    return orc_count_coloring_state(indexCol, indexRow, V, P, color, mode, NULL, root_out);
}

double orc_count_coloring_state(const int32_t *indexCol, const int32_t *indexRow, int32_t V, const orc_plan *P,
                                const int32_t *color, int mode, float *state, double *root_out)
{
    if (mode == 2) {
        float *buf = state ? state : (float *)calloc((size_t)V + 1, sizeof(float));
        double r = count_original_acc(indexCol, indexRow, V, P, color, buf, root_out);
        if (!state) free(buf);
        return r;
    }
    int n = P->nsub, k = P->k;
    int bottom = n - 1;
    size_t Vs = (size_t)V;
    float **tf = (float **)calloc((size_t)n, sizeof(float *));
    double **td = (double **)calloc((size_t)n, sizeof(double *));
    int scaled = 0;
    double countSum = 0.0;

    for (int s = n - 1; s >= 0; --s) {
        int sz = P->size[s];
        if (sz == 1) {
            if (s == bottom) {
                /* countCurBottom (DataTableColMajor.cpp:553-567) */
                if (mode == 1) {
                    td[s] = (double *)calloc((size_t)k * Vs, sizeof(double));
                    for (int32_t v = 0; v < V; ++v) td[s][(size_t)P->c2c[s][color[v]] * Vs + v] = 1.0;
                } else {
                    tf[s] = (float *)calloc((size_t)k * Vs, sizeof(float));
                    for (int32_t v = 0; v < V; ++v) tf[s][(size_t)P->c2c[s][color[v]] * Vs + v] = 1.0f;
                }
            }
            continue;
        }
        int m = P->main_[s], a = P->aux_[s];
        int mt = P->size[m] == 1 ? bottom : m;
        int at = P->size[a] == 1 ? bottom : a;
        int La = P->tlen[a], Ls = P->tlen[s], S = P->nsplit[s];

        if (mode == 1) {
            double *agg = (double *)calloc((size_t)La * Vs, sizeof(double));
            for (int c = 0; c < La; ++c) {
                const double *x = td[at] + (size_t)c * Vs;
                double *y = agg + (size_t)c * Vs;
                for (int32_t v = 0; v < V; ++v) {
                    double acc = 0.0;
                    for (int32_t e = indexCol[v]; e < indexCol[v + 1]; ++e) acc += x[indexRow[e]];
                    y[v] = acc;
                }
            }
            double *out = NULL;
            if (s > 0) out = (double *)calloc((size_t)Ls * Vs, sizeof(double));
            else out = (double *)calloc(Vs, sizeof(double));
            for (int i = 0; i < Ls; ++i) {
                double *obj = s > 0 ? out + (size_t)P->c2c[s][i] * Vs : out;
                for (int j = 0; j < S; ++j) {
                    const double *mm = td[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                    const double *aa = agg + (size_t)P->asplit[s][i * S + j] * Vs;
                    for (int32_t v = 0; v < V; ++v) obj[v] = obj[v] + aa[v] * mm[v];
                }
            }
            free(agg);
            if (s > 0) td[s] = out;
            else {
                for (int32_t v = 0; v < V; ++v) countSum += out[v];
                if (root_out) memcpy(root_out, out, sizeof(double) * Vs);
                free(out);
            }
        } else {
            /* aggregation: per row, FP32 sequential sum in ascending neighbour
             * order from a zeroed buffer (CSCGraph.hpp:219-307) */
            float *agg = (float *)calloc((size_t)La * Vs, sizeof(float));
            for (int c = 0; c < La; ++c) {
                const float *x = tf[at] + (size_t)c * Vs;
                float *y = agg + (size_t)c * Vs;
                for (int32_t v = 0; v < V; ++v) {
                    float acc = 0.0f;
                    for (int32_t e = indexCol[v]; e < indexCol[v + 1]; ++e) acc = acc + x[indexRow[e]];
                    y[v] = acc;
                }
            }
            if (s > 0) {
                float *out = (float *)calloc((size_t)Ls * Vs, sizeof(float));
                const double scale = (double)(float)1.0e-12; /* float parameter */
                for (int i = 0; i < Ls; ++i) {
                    float *obj = out + (size_t)P->c2c[s][i] * Vs;
                    for (int j = 0; j < S; ++j) {
                        const float *mm = tf[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                        const float *aa = agg + (size_t)P->asplit[s][i * S + j] * Vs;
                        if (mode == 0 && scaled == 0) {
                            for (int32_t v = 0; v < V; ++v)
                                obj[v] = (float)((double)obj[v] + ((double)aa[v] * (double)mm[v]) * scale);
                        } else {
                            for (int32_t v = 0; v < V; ++v) {
                                float prod = aa[v] * mm[v];
                                obj[v] = obj[v] + prod;
                            }
                        }
                    }
                }
                tf[s] = out;
            } else if (mode == 0) {
                double *last = (double *)calloc(Vs, sizeof(double));
                for (int i = 0; i < Ls; ++i)
                    for (int j = 0; j < S; ++j) {
                        const float *mm = tf[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                        const float *aa = agg + (size_t)P->asplit[s][i * S + j] * Vs;
                        for (int32_t v = 0; v < V; ++v) {
                            float prod = aa[v] * mm[v];
                            last[v] = last[v] + (double)prod;
                        }
                    }
                for (int32_t v = 0; v < V; ++v) countSum += last[v];
                countSum *= 1.0e+12; /* CountMat.cpp:820-822: _isScaled is always 1 here */
                if (root_out) memcpy(root_out, last, sizeof(double) * Vs);
                free(last);
            } else {
                float *last = (float *)calloc(Vs, sizeof(float));
                for (int i = 0; i < Ls; ++i)
                    for (int j = 0; j < S; ++j) {
                        const float *mm = tf[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                        const float *aa = agg + (size_t)P->asplit[s][i * S + j] * Vs;
                        for (int32_t v = 0; v < V; ++v) {
                            float prod = aa[v] * mm[v];
                            last[v] = last[v] + prod;
                        }
                    }
                for (int32_t v = 0; v < V; ++v) countSum += last[v];
                if (root_out) for (int32_t v = 0; v < V; ++v) root_out[v] = last[v];
                free(last);
            }
            free(agg);
        }
        scaled = 1;
        /* children freed after their parent (CountMat.cpp:313-316) */
        if (P->size[m] > 1) { free(tf[m]); tf[m] = NULL; free(td[m]); td[m] = NULL; }
        if (P->size[a] > 1) { free(tf[a]); tf[a] = NULL; free(td[a]); td[a] = NULL; }
    }
    for (int s = 0; s < n; ++s) { free(tf[s]); free(td[s]); }
    free(tf);
    free(td);
    return countSum;
}

/* The per-sub table of one coloring in FP32 reference semantics, for table-
 * level parity: runs the DP up to and including sub `upto` and copies its
 * column-major table [L][V] into out. Returns 0 on success. */
int orc_sub_table(const int32_t *indexCol, const int32_t *indexRow, int32_t V,
                  const orc_plan *P, const int32_t *color, int upto, float *out)
{
    int n = P->nsub, k = P->k, bottom = n - 1;
    size_t Vs = (size_t)V;
    if (upto <= 0 || upto >= n) return 1;
    float **tf = (float **)calloc((size_t)n, sizeof(float *));
    int scaled = 0, rc = 1;
    for (int s = n - 1; s >= upto; --s) {
        int sz = P->size[s];
        if (sz == 1) {
            if (s == bottom) {
                tf[s] = (float *)calloc((size_t)k * Vs, sizeof(float));
                for (int32_t v = 0; v < V; ++v) tf[s][(size_t)P->c2c[s][color[v]] * Vs + v] = 1.0f;
            }
            if (s == upto) { memcpy(out, tf[bottom], sizeof(float) * (size_t)k * Vs); rc = 0; }
            continue;
        }
        int m = P->main_[s], a = P->aux_[s];
        int mt = P->size[m] == 1 ? bottom : m;
        int at = P->size[a] == 1 ? bottom : a;
        int La = P->tlen[a], Ls = P->tlen[s], S = P->nsplit[s];
        float *agg = (float *)calloc((size_t)La * Vs, sizeof(float));
        for (int c = 0; c < La; ++c) {
            const float *x = tf[at] + (size_t)c * Vs;
            float *y = agg + (size_t)c * Vs;
            for (int32_t v = 0; v < V; ++v) {
                float acc = 0.0f;
                for (int32_t e = indexCol[v]; e < indexCol[v + 1]; ++e) acc = acc + x[indexRow[e]];
                y[v] = acc;
            }
        }
        float *o = (float *)calloc((size_t)Ls * Vs, sizeof(float));
        const double scale = (double)(float)1.0e-12;
        for (int i = 0; i < Ls; ++i) {
            float *obj = o + (size_t)P->c2c[s][i] * Vs;
            for (int j = 0; j < S; ++j) {
                const float *mm = tf[mt] + (size_t)P->msplit[s][i * S + j] * Vs;
                const float *aa = agg + (size_t)P->asplit[s][i * S + j] * Vs;
                if (scaled == 0) {
                    for (int32_t v = 0; v < V; ++v)
                        obj[v] = (float)((double)obj[v] + ((double)aa[v] * (double)mm[v]) * scale);
                } else {
                    for (int32_t v = 0; v < V; ++v) {
                        float prod = aa[v] * mm[v];
                        obj[v] = obj[v] + prod;
                    }
                }
            }
        }
        free(agg);
        tf[s] = o;
        scaled = 1;
        if (s == upto) { memcpy(out, o, sizeof(float) * (size_t)Ls * Vs); rc = 0; }
        if (P->size[m] > 1) { free(tf[m]); tf[m] = NULL; }
        if (P->size[a] > 1) { free(tf[a]); tf[a] = NULL; }
    }
    for (int s = 0; s < n; ++s) free(tf[s]);
    free(tf);
    return rc;
}

/* CountMat::compute's estimate (CountMat.cpp:246-264): mean raw count over
 * colorings divided by k!/k^k and the automorphism count, rounded. */
static int orc_fact(int n) { return n <= 1 ? 1 : n * orc_fact(n - 1); }
double orc_estimate(const double *raw, int ncol, int k, int aut)
{
    double sum = 0.0;
    for (int i = 0; i < ncol; ++i) sum += raw[i];
    double mean = sum / (double)ncol;
    double prob = orc_fact(k) / (orc_fact(0) * pow(k, k));
    return floor(mean / (prob * (double)aut) + 0.5);
}
