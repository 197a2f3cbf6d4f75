/*
 * CPU oracle for the reordered-SpMV path of Zhangq388/MATRIX-REORDER.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU-baseline leg
 * as the checker / reported baseline, never by the product library.
 * Each function restates one reference algorithm and cites the reference file
 * and lines it follows. Parity of this restatement is pinned against the
 * reference's own code compiled from its sources (oracle/build_ref.sh) and
 * against fixtures in tests/golden/.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ SpMV -- */

void orc_spmv_csr_f64(int n, const int32_t* rowptr, const int32_t* colidx,
                      const float* vals, const float* x, double* y)
{
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            s += (double)vals[k] * (double)x[colidx[k]];
        y[i] = s;
    }
}

int orc_spmv_csr_f32_omp(int n, const int32_t* rowptr, const int32_t* colidx,
                         const float* vals, const float* x, float* y, int threads)
{
    int used = 1;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
    used = threads;
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads)
#endif
    for (int i = 0; i < n; ++i) {
        float s = 0.0f;
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k)
            s += vals[k] * x[colidx[k]];
        y[i] = s;
    }
    return used;
}

/* ---------------------------------------------------------- MERBIT plan -- */

void orc_merbit_sizes(int nrow, int nnz, int sigma, int* lane_num, int* tile_num)
{
    /* include/merbit.cuh:141-142 */
    int ln = (int)(((int64_t)nrow + nnz + sigma - 1) / sigma);
    *lane_num = ln;
    *tile_num = (ln + 31) / 32;
}

/* merge_search, include/merbit.cuh:24-53: binary search along the cross
 * diagonal `diag` of the (row-end offsets, nonzero indices) merge grid. */
static void merge_search(const int32_t* offset, int nrow, int nnz, int diag,
                         int* coord_x, int* coord_y)
{
    int lo = diag - nnz;
    unsigned int y_min = (unsigned int)(lo > 0 ? lo : 0);
    unsigned int y_max = (unsigned int)(diag < nrow ? diag : nrow);
    while (y_min < y_max) {
        int mid = (int)((y_min + y_max) >> 1);
        if (offset[mid + 1] <= diag - mid - 1)
            y_min = (unsigned int)(mid + 1);
        else
            y_max = (unsigned int)mid;
    }
    *coord_x = diag - (int)y_min;
    *coord_y = (int)y_min < nrow ? (int)y_min : nrow;
}

int orc_merbit_plan(const int32_t* rowptr, int nrow, int nnz, int sigma,
                    uint32_t* tile_x, uint32_t* tile_y, uint64_t* lane_desc)
{
    if (sigma < 1 || sigma > 42 || nrow < 0 || nnz < 0) return -1;
    int lane_num, tile_num;
    orc_merbit_sizes(nrow, nnz, sigma, &lane_num, &tile_num);
    /* descriptor layout, include/merbit.cuh:84-86, :104-113 */
    const int wide = sigma >= 15;
    const int sh_flag = wide ? 22 : 18;
    const int sh_dy = wide ? 11 : 9;
    const int64_t items = (int64_t)nnz + nrow;

    for (int tile = 0; tile < tile_num; ++tile) {
        int warp_len = ((tile + 1) * 32 < lane_num) ? 32 : (lane_num - tile * 32);
        int wx0 = 0, wy0 = 0;
        int all_same = 1;
        for (int l = 0; l < warp_len; ++l) {
            int gid = tile * 32 + l;
            int lane_items = ((int64_t)(gid + 1) * sigma < items) ? sigma
                                                                   : (int)(items - (int64_t)gid * sigma);
            int cx, cy;
            merge_search(rowptr, nrow, nnz, gid * sigma, &cx, &cy);
            if (l == 0) { wx0 = cx; wy0 = cy; }
            uint64_t dx = (uint64_t)(uint32_t)(cx - wx0);
            uint64_t dy = (uint64_t)(uint32_t)(cy - wy0);
            uint64_t flags = 0;
            int y_start = cy;
            for (int i = 0; i < lane_items; ++i) {
                if (cx < rowptr[cy + 1]) {
                    ++cx;
                } else {
                    flags |= (uint64_t)1 << i;
                    ++cy;
                }
            }
            uint64_t d = (flags << sh_flag) | (dy << sh_dy) | dx;
            if (!wide) d &= 0xFFFFFFFFull; /* 32-bit word in the reference */
            lane_desc[gid] = d;
            if (y_start != cy) all_same = 0;
        }
        tile_x[tile] = (uint32_t)wx0;
        tile_y[tile] = (uint32_t)wy0 | (all_same ? 0x80000000u : 0u);
    }
    /* sentinel, include/merbit.cuh:127-131 */
    tile_x[tile_num] = (uint32_t)nnz;
    tile_y[tile_num] = (uint32_t)nrow;
    return 0;
}

/* ---------------------------------------------------------- permutation -- */

typedef struct { int32_t col; int32_t pos; } colpos;

static int colpos_cmp(const void* a, const void* b)
{
    const colpos* p = (const colpos*)a;
    const colpos* q = (const colpos*)b;
    if (p->col != q->col) return p->col < q->col ? -1 : 1;
    return p->pos < q->pos ? -1 : (p->pos > q->pos);
}

void orc_permute_csr(int n, const int32_t* rowptr, const int32_t* colidx,
                     const float* vals, const int32_t* perm,
                     int32_t* out_rowptr, int32_t* out_colidx, float* out_vals)
{
    /* perm[old] = new; inverse gives the source row of each new row
     * (scatter at src/class.cu:2688-2689). */
    int32_t* inv = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    out_rowptr[0] = 0;
    for (int i = 0; i < n; ++i) {
        int o = inv[i];
        out_rowptr[i + 1] = out_rowptr[i] + (rowptr[o + 1] - rowptr[o]);
    }
    int32_t maxlen = 0;
    for (int i = 0; i < n; ++i)
        if (rowptr[i + 1] - rowptr[i] > maxlen) maxlen = rowptr[i + 1] - rowptr[i];
    colpos* buf = (colpos*)malloc(sizeof(colpos) * (size_t)(maxlen > 0 ? maxlen : 1));
    for (int i = 0; i < n; ++i) {
        int o = inv[i];
        int32_t b = rowptr[o], len = rowptr[o + 1] - rowptr[o];
        for (int32_t k = 0; k < len; ++k) {
            buf[k].col = perm[colidx[b + k]]; /* gather relabel, :2701-2704 */
            buf[k].pos = k;
        }
        /* sort by (new row, new col), src/class.cu:445-454; ties keep order */
        qsort(buf, (size_t)len, sizeof(colpos), colpos_cmp);
        int32_t ob = out_rowptr[i];
        for (int32_t k = 0; k < len; ++k) {
            out_colidx[ob + k] = buf[k].col;
            out_vals[ob + k] = vals[b + buf[k].pos];
        }
    }
    free(buf);
    free(inv);
}

/* -------------------------------------------------------- exact RD hist -- */

/* Fenwick tree + last-position table, src/class.cu:864-936. */
void orc_rd_hist_exact(const int32_t* stream, int64_t nnz, int ncols, int sector_size,
                       const int32_t* edges, int nedges, int64_t* counts, int64_t* valid)
{
    const int64_t num_sectors = ((int64_t)ncols + sector_size - 1) / sector_size;
    int64_t* last = (int64_t*)malloc(sizeof(int64_t) * (size_t)(num_sectors > 0 ? num_sectors : 1));
    for (int64_t s = 0; s < num_sectors; ++s) last[s] = -1;
    int32_t* bit = (int32_t*)calloc((size_t)nnz + 1, sizeof(int32_t));
    for (int b = 0; b <= nedges; ++b) counts[b] = 0;
    int64_t nvalid = 0;

#define BIT_ADD(idx, d) do { for (int64_t _i = (idx) + 1; _i <= nnz; _i += _i & -_i) bit[_i] += (d); } while (0)

    for (int64_t k = 0; k < nnz; ++k) {
        const int64_t sector = stream[k] / sector_size;
        const int64_t old = last[sector];
        if (old < 0) {
            BIT_ADD(k, 1);
            last[sector] = k;
            continue;
        }
        BIT_ADD(old, -1);
        /* range_sum(old+1, k-1) = sum(k-1) - sum(old) */
        int64_t s_hi = 0, s_lo = 0;
        for (int64_t i = k; i > 0; i -= i & -i) s_hi += bit[i];
        for (int64_t i = old + 1; i > 0; i -= i & -i) s_lo += bit[i];
        const int64_t rd = s_hi - s_lo;
        /* bin_id: upper_bound over the edges, src/class.cu:887-890 */
        int b = 0;
        while (b < nedges && (double)edges[b] <= (double)rd) ++b;
        ++counts[b];
        ++nvalid;
        BIT_ADD(k, 1);
        last[sector] = k;
    }
#undef BIT_ADD
    *valid = nvalid;
    free(bit);
    free(last);
}

/* ------------------------------------------------------ sampled HLL RD -- */

/* hash, rank, update and estimate: src/class.cu:954-1012 */
static uint32_t hll_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

static int hll_rank(uint32_t h, int p)
{
    uint32_t w = h >> p;
    const int max_rank = 32 - p + 1;
    if (w == 0U) return max_rank;
    int r = __builtin_clz(w) - p + 1;
    if (r < 1) r = 1;
    if (r > max_rank) r = max_rank;
    return r;
}

static float hll_estimate(const int* regs, int m)
{
    float sum = 0.0f;
    int zeros = 0;
    for (int i = 0; i < m; ++i) {
        int r = regs[i];
        if (r == 0) ++zeros;
        sum += exp2f(-(float)r);
    }
    const float mf = (float)m;
    float alpha;
    if (m == 16) alpha = 0.673f;
    else if (m == 32) alpha = 0.697f;
    else if (m == 64) alpha = 0.709f;
    else alpha = 0.7213f / (1.0f + 1.079f / mf);
    float e = alpha * mf * mf / sum;
    if (e <= 2.5f * mf && zeros > 0) e = mf * logf(mf / (float)zeros);
    return e;
}

/* Sequential simulation of sampled_hll_rd_block_kernel (src/class.cu:1014-1131)
 * with its 256-position chunks and its 16-chunk cap-check cadence. */
void orc_hll_sampled(const int32_t* stream, int nnz, int samples, int sector_size,
                     uint32_t seed, int rd_cap, int max_scan, int hll_p,
                     float* est, int32_t* status, int32_t* pos)
{
    const int chunk = 256;
    const int m = 1 << hll_p;
    int* regs = (int*)malloc(sizeof(int) * (size_t)m);
    for (int sid = 0; sid < samples; ++sid) {
        if (nnz <= 1) return;
        memset(regs, 0, sizeof(int) * (size_t)m);
        uint32_t r = hll_hash(seed ^ (uint32_t)((uint32_t)sid * 0x9e3779b9U + 17U));
        int sp = 1 + (int)(r % (uint32_t)(nnz - 1));
        int lo = (max_scan > 0) ? (sp - max_scan > 0 ? sp - max_scan : 0) : 0;
        int st = -99;
        float e = 0.0f;
        int chunks_done = 0;
        pos[sid] = sp;
        const int target = stream[sp] / sector_size;
        for (int hi = sp - 1; hi >= lo && st == -99; hi -= chunk) {
            int found = -1;
            for (int t = 0; t < chunk; ++t) {
                int idx = hi - t;
                if (idx >= lo && stream[idx] / sector_size == target && idx > found) found = idx;
            }
            for (int t = 0; t < chunk; ++t) {
                int idx = hi - t;
                if (idx < lo) break;
                int sec = stream[idx] / sector_size;
                if (sec != target && (found < 0 || idx > found)) {
                    uint32_t h = hll_hash((uint32_t)sec);
                    int rid = (int)(h & (uint32_t)(m - 1));
                    int rk = hll_rank(h, hll_p);
                    if (rk > regs[rid]) regs[rid] = rk;
                }
            }
            ++chunks_done;
            if (found >= 0) {
                e = hll_estimate(regs, m);
                st = 0;
            } else if (rd_cap > 0 && (chunks_done % 16 == 0)) {
                float tmp = hll_estimate(regs, m);
                if (tmp > (float)rd_cap * 1.03f) {
                    e = tmp;
                    st = 2;
                }
            }
        }
        if (st == -99) {
            e = hll_estimate(regs, m);
            st = (lo == 0) ? 1 : 3;
        }
        est[sid] = e;
        status[sid] = st;
    }
    free(regs);
}

void orc_hll_bin(int samples, const float* est, const int32_t* status,
                 const int32_t* edges, int nedges, int64_t* counts,
                 int64_t* found, int64_t* cold, int64_t* large, int64_t* unresolved)
{
    for (int b = 0; b <= nedges; ++b) counts[b] = 0;
    *found = *cold = *large = *unresolved = 0;
    for (int i = 0; i < samples; ++i) {
        switch (status[i]) {
        case 0: {
            ++*found;
            double v = (double)est[i];
            int b = 0;
            while (b < nedges && (double)edges[b] <= v) ++b;
            ++counts[b];
            break;
        }
        case 1: ++*cold; break;
        case 2: ++*large; ++counts[nedges]; break;
        default: ++*unresolved; break;
        }
    }
}

/* -------------------------------------------------------------- pGOrder -- */

/* Bucket priority queue with the exact link order of Integer_Heap
 * (include/integer_heap.cuh:34-151): buckets are circular doubly linked lists
 * indexed by key1; insertion goes right after the bucket head. Node ids are
 * local to one batch. */
typedef struct {
    int* left; int* right; int* key1; int* key2;
    int* htab; int cap; int pmax; int cnt;
} iheap;

static void ih_grow(iheap* h, int key)
{
    if (key < h->cap) return;
    int nc = h->cap;
    while (nc <= key) nc *= 2;
    h->htab = (int*)realloc(h->htab, sizeof(int) * (size_t)nc);
    for (int i = h->cap; i < nc; ++i) h->htab[i] = -1;
    h->cap = nc;
}

static void ih_remove(iheap* h, int v)
{
    int* head = &h->htab[h->key1[v]];
    if (*head == v) {
        if (h->right[v] == v) {
            *head = -1;
        } else {
            *head = h->right[v];
            h->right[h->left[v]] = h->right[v];
            h->left[h->right[v]] = h->left[v];
            h->left[v] = v;
            h->right[v] = v;
        }
    } else {
        h->right[h->left[v]] = h->right[v];
        h->left[h->right[v]] = h->left[v];
        h->left[v] = v;
        h->right[v] = v;
    }
}

static void ih_insert(iheap* h, int v)
{
    h->key1[v] += h->key2[v];
    h->key2[v] = 0;
    ih_grow(h, h->key1[v]);
    int t = h->htab[h->key1[v]];
    if (t < 0) {
        h->htab[h->key1[v]] = v;
    } else {
        h->left[v] = t;
        h->right[v] = h->right[t];
        h->left[h->right[t]] = v;
        h->right[t] = v;
    }
}

static void ih_push(iheap* h, int v)
{
    ih_insert(h, v);
    ++h->cnt;
    if (h->key1[v] > h->pmax) h->pmax = h->key1[v];
}

static void ih_modify(iheap* h, int v, int val)
{
    h->key2[v] += val;
    if (h->key2[v] > 0) {
        ih_remove(h, v);
        ih_insert(h, v);
        if (h->key1[v] > h->pmax) h->pmax = h->key1[v];
    }
}

static int ih_pop(iheap* h)
{
    while (h->cnt > 0) {
        while (h->pmax > 0 && h->htab[h->pmax] < 0) --h->pmax;
        int t = h->htab[h->pmax];
        while (t >= 0) {
            if (h->key2[t] == 0) {
                ih_remove(h, t);
                --h->cnt;
                return t;
            }
            ih_remove(h, t);
            ih_insert(h, t);
            t = h->htab[h->pmax];
        }
    }
    return -1;
}

int orc_get_width(int nrow, int nnz)
{
    /* GRAPH::get_width, src/class.cu:733-750 (float arithmetic, integer nnz/nrow) */
    float bound = roundf(log2f(sqrtf((float)nrow / (float)(nnz / nrow))));
    if (bound < 10) return 1024;
    if (bound >= 10 && bound < 12) return 16384;
    return 262144;
}

/* order_on_cpu, src/class.cu:2220-2314, for the batch [start, start+len). */
static void order_batch(const int32_t* off1, const int32_t* ind1,
                        const int32_t* off2, const int32_t* ind2,
                        uint32_t* perm, int start, int len, int width, int degree)
{
    iheap h;
    h.left = (int*)malloc(sizeof(int) * (size_t)len);
    h.right = (int*)malloc(sizeof(int) * (size_t)len);
    h.key1 = (int*)calloc((size_t)len, sizeof(int));
    h.key2 = (int*)calloc((size_t)len, sizeof(int));
    h.cap = 64;
    h.htab = (int*)malloc(sizeof(int) * 64);
    for (int i = 0; i < 64; ++i) h.htab[i] = -1;
    h.pmax = 0;
    h.cnt = 0;
    char* sts = (char*)malloc((size_t)len);
    for (int i = 0; i < len; ++i) { h.left[i] = h.right[i] = i; sts[i] = 1; }

    /* seed: largest off1 degree, first one wins ties (:2234-2243) */
    int id = (int)perm[0];
    int deg = off1[id + 1] - off1[id];
    for (int i = 0; i < len; ++i) {
        int v = (int)perm[i];
        if (off1[v + 1] - off1[v] > deg) { deg = off1[v + 1] - off1[v]; id = v; }
    }
    for (int i = 0; i < len; ++i) ih_push(&h, (int)perm[i] - start);
    ih_modify(&h, id - start, 1);

    for (int pos = 0; h.cnt > 0; ++pos) {
        int u = ih_pop(&h);
        sts[u] = 0;
        int ug = u + start;
        perm[pos] = (uint32_t)ug;
        /* raise siblings of the node entering the window (:2262-2280) */
        if (off2[ug + 1] - off2[ug] < degree) {
            for (int32_t j = off2[ug]; j < off2[ug + 1]; ++j) {
                int c = ind2[j];
                if (off1[c + 1] - off1[c] < degree) {
                    for (int32_t j2 = off1[c]; j2 < off1[c + 1]; ++j2) {
                        int w = ind1[j2];
                        if (w >= start && w < start + len && sts[w - start]) ih_modify(&h, w - start, 1);
                    }
                }
            }
        }
        /* lower siblings of the node leaving the window (:2283-2309) */
        if (pos >= width) {
            int vg = (int)perm[pos - width];
            if (off2[vg + 1] - off2[vg] < degree) {
                for (int32_t j = off2[vg]; j < off2[vg + 1]; ++j) {
                    int c = ind2[j];
                    if (off1[c + 1] - off1[c] < degree) {
                        for (int32_t j2 = off1[c]; j2 < off1[c + 1]; ++j2) {
                            int w = ind1[j2];
                            if (w >= start && w < start + len && sts[w - start]) ih_modify(&h, w - start, -1);
                        }
                    }
                }
            }
        }
    }
    free(sts); free(h.htab); free(h.key2); free(h.key1); free(h.right); free(h.left);
}

/* gorder4, src/class.cu:2608-2690. off1/ind1 are the column lists (CSC) of
 * our matrix and off2/ind2 its rows (CSR), see the header comment. */
void orc_pgorder(int n, const int32_t* rowptr, const int32_t* colidx,
                 int vsize, int width, uint32_t* perm)
{
    const int32_t nnz = rowptr[n];
    int32_t* off1 = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t* ind1 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz > 0 ? nnz : 1));
    for (int32_t k = 0; k < nnz; ++k) off1[colidx[k] + 1]++;
    for (int i = 0; i < n; ++i) off1[i + 1] += off1[i];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) fill[i] = off1[i];
    for (int i = 0; i < n; ++i)
        for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) ind1[fill[colidx[k]]++] = i;
    free(fill);

    for (int i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    const int degree = (int)(sqrt((double)n) / 4); /* L, :2659 */
    const int nb = (n + vsize - 1) / vsize;
    for (int b = 0; b < nb; ++b) {
        int start = b * vsize;
        int len = (start + vsize < n) ? vsize : n - start;
        order_batch(off1, ind1, rowptr, colidx, perm + start, start, len, width, degree);
    }
    free(ind1);
    free(off1);
}

/* ------------------------------------------------------------ predictor -- */

double orc_predict(const double* coef, double intercept, const double* r)
{
    /* PredictLogSpeedup + PredictSpeedup, include/model.cuh:84-95 */
    double v = intercept;
    for (int i = 0; i < 10; ++i) v += coef[i] * r[i];
    return exp(v);
}

/* ------------------------------------------------------- random order -- */

/* minstd_rand (x <- 48271 x mod 2^31 - 1), Thrust's default_random_engine;
 * seed(s) takes s mod m and replaces 0 by 1. */
static uint32_t minstd_next(uint64_t* x)
{
    *x = (*x * 48271u) % 2147483647u;
    return (uint32_t)*x;
}

void orc_order_random(int n, uint32_t seed, int32_t* perm)
{
    /* relabel_random seeds the engine with graph_id and shuffles the
     * identity perm (src/class.cu:1467-1473); thrust::shuffle copies the
     * input and writes out[j] = in[key_j], key_j the j-th value of the
     * Feistel bijection below that is < n, taken in index order. */
    uint64_t x = seed % 2147483647u;
    if (x == 0) x = 1;
    uint32_t key[24];
    for (int i = 0; i < 24; ++i) key[i] = minstd_next(&x);
    /* cipher width: 4 bits up to n = 16, else ceil(log2 n) */
    uint32_t bits = 4;
    if (n > 16) {
        bits = 0;
        for (uint64_t m = (uint64_t)n - 1; m; m >>= 1) ++bits;
    }
    const uint32_t lb = bits / 2, rb = bits - lb;
    const uint64_t lmask = (1ull << lb) - 1, rmask = (1ull << rb) - 1;
    const uint64_t span = 1ull << bits;
    int64_t j = 0;
    for (uint64_t v = 0; v < span; ++v) {
        uint32_t a = (uint32_t)(v >> rb), b = (uint32_t)(v & rmask);
        for (int r = 0; r < 24; ++r) {
            const uint64_t p = 0xD2B74407B1CE6E93ull * (uint64_t)a;
            const uint32_t hi = (uint32_t)(p >> 32);
            const uint32_t lo = ((uint32_t)p << (rb - lb)) | (b >> lb);
            a = (uint32_t)(((hi ^ key[r]) ^ b) & lmask);
            b = (uint32_t)(lo & rmask);
        }
        const uint64_t k = ((uint64_t)a << rb) | b;
        if (k < (uint64_t)n) perm[j++] = (int32_t)k;
    }
}
