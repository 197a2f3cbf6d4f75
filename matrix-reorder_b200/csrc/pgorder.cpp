// pGOrder ("gorder4"): GOrder-style greedy ordering run independently inside
// consecutive blocks of vsize vertex ids, on host threads.
//
// Semantics follow GRAPH::gorder4 / order_on_cpu (src/class.cu:2608-2690,
// :2220-2314) exactly, so the permutation is bit-identical:
//  * inside block [start, start+len): seed = the vertex with the largest
//    column count (first one on ties); all block vertices enter a bucket
//    queue at key 0 and the seed is raised by one;
//  * repeatedly pop the maximum key; the popped vertex u takes the next
//    position; every still-queued vertex w of the block that shares a column
//    with u (via u's row if it has fewer than L entries, and the column's
//    entries if the column has fewer than L) gains one; when a vertex leaves
//    the window of the last `width` placed vertices, the same vertices lose
//    one (lazily, as a pending negative key);
//  * L = (int)(sqrt(n) / 4).
// The bucket queue keeps the link order of Integer_Heap
// (include/integer_heap.cuh:34-151): circular lists per key, insertion right
// after the bucket head, pending decreases applied when the head is popped.
// Here it is an index-based structure private to one block, and blocks run
// on a pool of std::threads instead of a 128-thread ThreadPool with shared
// Node objects.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "internal.hpp"

namespace mr {
namespace {

class BucketQueue {
public:
    void reset(int len)
    {
        left.resize((size_t)len);
        right.resize((size_t)len);
        key1.assign((size_t)len, 0);
        key2.assign((size_t)len, 0);
        for (int i = 0; i < len; ++i) left[(size_t)i] = right[(size_t)i] = i;
        std::fill(htab.begin(), htab.end(), -1);
        if (htab.size() < 64) htab.assign(64, -1);
        pmax = 0;
        cnt = 0;
    }
    void push(int v)
    {
        insert(v);
        ++cnt;
        if (key1[(size_t)v] > pmax) pmax = key1[(size_t)v];
    }
    void modify(int v, int d)
    {
        key2[(size_t)v] += d;
        if (key2[(size_t)v] > 0) {
            remove(v);
            insert(v);
            if (key1[(size_t)v] > pmax) pmax = key1[(size_t)v];
        }
    }
    int pop()
    {
        while (cnt > 0) {
            while (pmax > 0 && htab[(size_t)pmax] < 0) --pmax;
            int t = htab[(size_t)pmax];
            while (t >= 0) {
                if (key2[(size_t)t] == 0) {
                    remove(t);
                    --cnt;
                    return t;
                }
                remove(t);
                insert(t);
                t = htab[(size_t)pmax];
            }
        }
        return -1;
    }
    int size() const { return cnt; }

private:
    void remove(int v)
    {
        int& head = htab[(size_t)key1[(size_t)v]];
        const int l = left[(size_t)v], r = right[(size_t)v];
        if (head == v) {
            if (r == v) {
                head = -1;
                return;
            }
            head = r;
        }
        right[(size_t)l] = r;
        left[(size_t)r] = l;
        left[(size_t)v] = v;
        right[(size_t)v] = v;
    }
    void insert(int v)
    {
        int k = key1[(size_t)v] + key2[(size_t)v];
        key1[(size_t)v] = k;
        key2[(size_t)v] = 0;
        if ((size_t)k >= htab.size()) htab.resize(std::max(htab.size() * 2, (size_t)k + 1), -1);
        int& head = htab[(size_t)k];
        if (head < 0) {
            head = v;
        } else {
            left[(size_t)v] = head;
            right[(size_t)v] = right[(size_t)head];
            left[(size_t)right[(size_t)head]] = v;
            right[(size_t)head] = v;
        }
    }
    std::vector<int> left, right, key1, key2, htab;
    int pmax = 0, cnt = 0;
};

struct Csr {
    const int32_t* off;
    const int32_t* ind;
    int deg(int v) const { return off[v + 1] - off[v]; }
};

void order_block(const Csr& cols, const Csr& rows, uint32_t* perm, int start, int len, int width, int degree,
                 BucketQueue& q, std::vector<char>& sts)
{
    int id = (int)perm[0];
    int best = cols.deg(id);
    for (int i = 0; i < len; ++i) {
        const int v = (int)perm[i];
        if (cols.deg(v) > best) {
            best = cols.deg(v);
            id = v;
        }
    }
    q.reset(len);
    sts.assign((size_t)len, 1);
    for (int i = 0; i < len; ++i) q.push((int)perm[i] - start);
    q.modify(id - start, 1);

    auto bump = [&](int u, int d) {
        if (rows.deg(u) >= degree) return;
        for (int32_t j = rows.off[u]; j < rows.off[u + 1]; ++j) {
            const int c = rows.ind[j];
            if (cols.deg(c) >= degree) continue;
            for (int32_t j2 = cols.off[c]; j2 < cols.off[c + 1]; ++j2) {
                const unsigned w = (unsigned)(cols.ind[j2] - start);
                if (w < (unsigned)len && sts[w]) q.modify((int)w, d);
            }
        }
    };
    for (int pos = 0; q.size() > 0; ++pos) {
        const int u = q.pop();
        sts[(size_t)u] = 0;
        perm[pos] = (uint32_t)(u + start);
        bump(u + start, 1);
        if (pos >= width) bump((int)perm[pos - width], -1);
    }
}

}  // namespace

int32_t pgorder_width(int32_t n, int64_t nnz)
{
    // GRAPH::get_width (src/class.cu:733-750): float arithmetic, integer nnz/n
    const int32_t q = (int32_t)(nnz / n);
    const float bound = std::round(std::log2(std::sqrt((float)n / (float)q)));
    if (bound < 10) return 1024;
    if (bound >= 10 && bound < 12) return 16384;
    return 262144;
}

int pgorder_host(int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t vsize, int32_t width,
                 int32_t threads, uint32_t* perm)
{
    if (n < 0 || !rowptr || !perm || (n > 0 && rowptr[n] > 0 && !colidx)) return MR_ERR_INVALID_ARG;
    if (n == 0) return MR_OK;
    const int32_t nnz = rowptr[n];
    if (vsize <= 0) vsize = pgorder_width(n, nnz);
    if (width < 1) return MR_ERR_INVALID_ARG;
    // column lists (rows ascending within each column): the reference's
    // sort(true) + coo2csr (src/class.cu:2629-2631)
    std::vector<int32_t> coff((size_t)n + 1, 0), cind((size_t)std::max(nnz, 1));
    for (int32_t k = 0; k < nnz; ++k) {
        const int32_t c = colidx[k];
        if (c < 0 || c >= n) return MR_ERR_INVALID_ARG;
        ++coff[(size_t)c + 1];
    }
    for (int32_t i = 0; i < n; ++i) coff[(size_t)i + 1] += coff[(size_t)i];
    {
        std::vector<int32_t> fill(coff.begin(), coff.end() - 1);
        for (int32_t i = 0; i < n; ++i)
            for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) cind[(size_t)fill[(size_t)colidx[k]]++] = i;
    }
    const Csr cols{coff.data(), cind.data()};
    const Csr rows{rowptr, colidx};
    for (int32_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    const int degree = (int)(std::sqrt((double)n) / 4);
    const int nb = (int)(((int64_t)n + vsize - 1) / vsize);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    threads = std::min(threads, nb);
    std::atomic<int> next{0};
    auto worker = [&]() {
        BucketQueue q;
        std::vector<char> sts;
        for (int b = next++; b < nb; b = next++) {
            const int start = b * vsize;
            const int len = (int)std::min<int64_t>(vsize, (int64_t)n - start);
            order_block(cols, rows, perm + start, start, len, width, degree, q, sts);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return MR_OK;
}

}  // namespace mr

extern "C" int32_t mr_pgorder_width(int32_t n, int64_t nnz)
{
    if (n <= 0) return 1024;
    return mr::pgorder_width(n, nnz);
}

extern "C" int mr_pgorder(int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t vsize, int32_t width,
                          int32_t threads, uint32_t* perm)
{
    return mr::pgorder_host(n, rowptr, colidx, vsize, width, threads, perm);
}
