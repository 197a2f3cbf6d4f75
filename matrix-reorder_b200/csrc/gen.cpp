// Seeded synthetic workload generators (host C++, OpenMP).
//
// The reference measures on SuiteSparse / Graph500 .mtx files that are not
// available here; these generators produce matrices with the shapes the
// workloads name: Graph500-style R-MAT (the bit-descent scheme of GAP's
// generator, parsb/include/generator.h:80-108, with its id shuffle :52-63),
// a 2-D 5-point Laplacian, a Chung-Lu power-law matrix and banded matrices.
// Every output is textbook CSR with columns sorted and duplicates merged.
// Values are uniform in [-1, 1] from a counter-based hash of (seed, position),
// so they do not depend on the thread count.
#include "gen.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <cstdio>
#include <string>
#include <vector>
#include <omp.h>

struct mrg_csr {
    int32_t n = 0;
    std::vector<int32_t> rowptr;
    std::vector<int32_t> colidx;
    std::vector<float> vals;
};

namespace {

inline uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// uniform in [-1, 1): 24 random bits, exactly representable in FP32
inline float unit_pm1(uint64_t seed, uint64_t i)
{
    uint64_t h = splitmix64(seed * 0x632be59bd9b4e019ull + i);
    return (float)((int64_t)(h >> 40) - (1ll << 23)) * (1.0f / (float)(1 << 23));
}

void fill_values(mrg_csr* m, uint64_t seed)
{
    const int64_t nnz = (int64_t)m->colidx.size();
    m->vals.resize((size_t)nnz);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nnz; ++k) m->vals[(size_t)k] = unit_pm1(seed ^ 0x5eedull, (uint64_t)k);
}

// Build CSR from an edge list: counting sort by source, then sort and merge
// duplicate columns inside each row. Deterministic for any thread count.
mrg_csr* csr_from_edges(int32_t n, const std::vector<int32_t>& src, const std::vector<int32_t>& dst)
{
    const int64_t m = (int64_t)src.size();
    std::vector<int64_t> cnt((size_t)n + 1, 0);
    {
        std::vector<std::atomic<int64_t>> c((size_t)n);
        for (auto& a : c) a.store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < m; ++e) c[(size_t)src[(size_t)e]].fetch_add(1, std::memory_order_relaxed);
        for (int32_t i = 0; i < n; ++i) cnt[(size_t)i + 1] = cnt[(size_t)i] + c[(size_t)i].load();
    }
    std::vector<int32_t> tmp((size_t)m);
    {
        std::vector<std::atomic<int64_t>> fill((size_t)n);
        for (int32_t i = 0; i < n; ++i) fill[(size_t)i].store(cnt[(size_t)i], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < m; ++e)
            tmp[(size_t)fill[(size_t)src[(size_t)e]].fetch_add(1, std::memory_order_relaxed)] = dst[(size_t)e];
    }
    std::vector<int32_t> uniq((size_t)n + 1, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t i = 0; i < n; ++i) {
        auto b = tmp.begin() + cnt[(size_t)i], e = tmp.begin() + cnt[(size_t)i + 1];
        std::sort(b, e);
        uniq[(size_t)i + 1] = (int32_t)(std::unique(b, e) - b);
    }
    auto* out = new mrg_csr;
    out->n = n;
    out->rowptr.assign((size_t)n + 1, 0);
    for (int32_t i = 0; i < n; ++i) out->rowptr[(size_t)i + 1] = out->rowptr[(size_t)i] + uniq[(size_t)i + 1];
    out->colidx.resize((size_t)out->rowptr[(size_t)n]);
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t i = 0; i < n; ++i)
        std::copy(tmp.begin() + cnt[(size_t)i], tmp.begin() + cnt[(size_t)i] + uniq[(size_t)i + 1],
                  out->colidx.begin() + out->rowptr[(size_t)i]);
    return out;
}

// Symmetric relabel B[p[r], p[c]] = A[r, c] (keeps values with their entries).
void relabel(mrg_csr* a, const std::vector<int32_t>& p)
{
    const int32_t n = a->n;
    std::vector<int32_t> inv((size_t)n);
    for (int32_t i = 0; i < n; ++i) inv[(size_t)p[(size_t)i]] = i;
    std::vector<int32_t> rp((size_t)n + 1, 0);
    for (int32_t i = 0; i < n; ++i) {
        int32_t o = inv[(size_t)i];
        rp[(size_t)i + 1] = rp[(size_t)i] + (a->rowptr[(size_t)o + 1] - a->rowptr[(size_t)o]);
    }
    std::vector<int32_t> ci(a->colidx.size());
    std::vector<float> cv(a->vals.size());
    const bool hasv = !a->vals.empty();
#pragma omp parallel
    {
        std::vector<std::pair<int32_t, int32_t>> buf;
#pragma omp for schedule(dynamic, 256)
        for (int32_t i = 0; i < n; ++i) {
            int32_t o = inv[(size_t)i], b = a->rowptr[(size_t)o], len = a->rowptr[(size_t)o + 1] - b;
            buf.resize((size_t)len);
            for (int32_t k = 0; k < len; ++k) buf[(size_t)k] = {p[(size_t)a->colidx[(size_t)(b + k)]], b + k};
            std::sort(buf.begin(), buf.end());
            for (int32_t k = 0; k < len; ++k) {
                ci[(size_t)(rp[(size_t)i] + k)] = buf[(size_t)k].first;
                if (hasv) cv[(size_t)(rp[(size_t)i] + k)] = a->vals[(size_t)buf[(size_t)k].second];
            }
        }
    }
    a->rowptr.swap(rp);
    a->colidx.swap(ci);
    a->vals.swap(cv);
}

std::vector<int32_t> random_perm(int32_t n, uint64_t seed)
{
    std::vector<int32_t> p((size_t)n);
    std::iota(p.begin(), p.end(), 0);
    std::mt19937_64 rng(seed);
    std::shuffle(p.begin(), p.end(), rng);
    return p;
}

// R-MAT bit descent (parsb/include/generator.h:80-108). Endpoints >= n are
// redrawn so that any row count works (n = 2^scale needs no redraw).
void rmat_edges(int32_t n, int scale, int64_t m, double a, double b, double c, uint64_t seed,
                std::vector<int32_t>& src, std::vector<int32_t>& dst)
{
    const float A = (float)a, B = (float)b, C = (float)c;
    const int64_t block = 1 << 18;
    src.resize((size_t)m);
    dst.resize((size_t)m);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t blk = 0; blk < (m + block - 1) / block; ++blk) {
        std::mt19937 rng((uint32_t)(seed + (uint64_t)blk));
        std::uniform_real_distribution<float> u(0.0f, 1.0f);
        for (int64_t e = blk * block; e < std::min(m, (blk + 1) * block); ++e) {
            int64_t s, d;
            do {
                s = 0;
                d = 0;
                for (int depth = 0; depth < scale; ++depth) {
                    float r = u(rng);
                    s <<= 1;
                    d <<= 1;
                    if (r < A + B) {
                        if (r > A) d++;
                    } else {
                        s++;
                        if (r > A + B + C) d++;
                    }
                }
            } while (s >= n || d >= n);
            src[(size_t)e] = (int32_t)s;
            dst[(size_t)e] = (int32_t)d;
        }
    }
}

}  // namespace

extern "C" {

mrg_csr* mrg_rmat(int32_t n, int32_t edge_factor, double a, double b, double c, uint64_t seed, int permute_ids)
{
    if (n <= 0 || edge_factor <= 0) return nullptr;
    int scale = 0;
    while ((1ll << scale) < n) ++scale;
    std::vector<int32_t> src, dst;
    rmat_edges(n, scale, (int64_t)n * edge_factor, a, b, c, seed, src, dst);
    if (permute_ids) {
        // GAP's PermuteIDs (parsb/include/generator.h:52-63): one shuffled
        // id map applied to both endpoints.
        std::vector<int32_t> p((size_t)n);
        std::iota(p.begin(), p.end(), 0);
        std::mt19937 rng((uint32_t)seed);
        std::shuffle(p.begin(), p.end(), rng);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < (int64_t)src.size(); ++e) {
            src[(size_t)e] = p[(size_t)src[(size_t)e]];
            dst[(size_t)e] = p[(size_t)dst[(size_t)e]];
        }
    }
    mrg_csr* m = csr_from_edges(n, src, dst);
    fill_values(m, seed);
    return m;
}

mrg_csr* mrg_laplace2d(int32_t g, int shuffle, uint64_t seed)
{
    if (g <= 0 || (int64_t)g * g > INT32_MAX) return nullptr;
    auto* m = new mrg_csr;
    const int32_t n = g * g;
    m->n = n;
    m->rowptr.resize((size_t)n + 1);
    m->rowptr[0] = 0;
    for (int32_t r = 0; r < n; ++r) {
        int32_t i = r / g, j = r % g;
        m->rowptr[(size_t)r + 1] = m->rowptr[(size_t)r] + 1 + (i > 0) + (j > 0) + (j + 1 < g) + (i + 1 < g);
    }
    m->colidx.resize((size_t)m->rowptr[(size_t)n]);
    m->vals.resize(m->colidx.size());
#pragma omp parallel for schedule(static)
    for (int32_t r = 0; r < n; ++r) {
        int32_t i = r / g, j = r % g, k = m->rowptr[(size_t)r];
        auto put = [&](int32_t c, float v) { m->colidx[(size_t)k] = c; m->vals[(size_t)k] = v; ++k; };
        if (i > 0) put(r - g, -1.0f);
        if (j > 0) put(r - 1, -1.0f);
        put(r, 4.0f);
        if (j + 1 < g) put(r + 1, -1.0f);
        if (i + 1 < g) put(r + g, -1.0f);
    }
    if (shuffle) relabel(m, random_perm(n, seed));
    return m;
}

mrg_csr* mrg_chung_lu(int32_t n, double gamma, double mean_deg, int32_t dmin, int32_t dmax, uint64_t seed)
{
    if (n <= 0 || gamma <= 1.0 || mean_deg <= 0) return nullptr;
    // expected degree of rank i: w_i = s (i+1)^(-1/(gamma-1)), clamped to
    // [dmin, dmax]; s is found by bisection so the clamped mean is mean_deg.
    const double ex = -1.0 / (gamma - 1.0);
    auto mean_for = [&](double s) {
        double t = 0;
#pragma omp parallel for reduction(+ : t)
        for (int32_t i = 0; i < n; ++i) t += std::min((double)dmax, std::max((double)dmin, s * std::pow(i + 1.0, ex)));
        return t / n;
    };
    double lo = 1e-3, hi = (double)dmax * (double)n;  // mean_for(hi) = dmax: every mean up to dmax is reachable
    for (int it = 0; it < 80; ++it) {
        double mid = std::sqrt(lo * hi);
        (mean_for(mid) < mean_deg ? lo : hi) = mid;
    }
    const double s = std::sqrt(lo * hi);
    std::vector<double> w((size_t)n);
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) w[(size_t)i] = std::min((double)dmax, std::max((double)dmin, s * std::pow(i + 1.0, ex)));
    // ranks are spread over ids by a seeded shuffle
    std::vector<int32_t> id = random_perm(n, seed ^ 0xc1u);
    // Walker alias table over the column weights
    std::vector<double> prob((size_t)n);
    std::vector<int32_t> alias((size_t)n);
    {
        double tot = 0;
        for (double v : w) tot += v;
        std::vector<int32_t> small, large;
        std::vector<double> q((size_t)n);
        for (int32_t i = 0; i < n; ++i) {
            q[(size_t)i] = w[(size_t)i] * n / tot;
            (q[(size_t)i] < 1.0 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            int32_t l = small.back(), g2 = large.back();
            small.pop_back();
            prob[(size_t)l] = q[(size_t)l];
            alias[(size_t)l] = g2;
            q[(size_t)g2] = (q[(size_t)g2] + q[(size_t)l]) - 1.0;
            if (q[(size_t)g2] < 1.0) {
                large.pop_back();
                small.push_back(g2);
            }
        }
        for (int32_t i : large) { prob[(size_t)i] = 1.0; alias[(size_t)i] = i; }
        for (int32_t i : small) { prob[(size_t)i] = 1.0; alias[(size_t)i] = i; }
    }
    // row degrees: round(w) with a random fractional part
    std::vector<int64_t> start((size_t)n + 1, 0);
    std::vector<int32_t> deg((size_t)n);
    for (int32_t r = 0; r < n; ++r) {
        double f = w[(size_t)r];
        double u = (double)(splitmix64(seed * 31 + (uint64_t)r) >> 11) * (1.0 / 9007199254740992.0);
        deg[(size_t)r] = (int32_t)std::floor(f + u);
        start[(size_t)r + 1] = start[(size_t)r] + deg[(size_t)r];
    }
    std::vector<int32_t> src((size_t)start[(size_t)n]), dst((size_t)start[(size_t)n]);
    // each row draws its deg distinct columns in proportion to the weights
    // (without replacement: a heavy row would otherwise collapse onto the
    // few heaviest columns when duplicates are merged); if rejections stall
    // (the row needs most of the remaining weight), the rest is drawn
    // uniformly
#pragma omp parallel
    {
        std::vector<int32_t> table;
        std::vector<uint32_t> used;
#pragma omp for schedule(dynamic, 64)
        for (int32_t r = 0; r < n; ++r) {
            const int64_t d = std::min<int64_t>(deg[(size_t)r], n);
            const int64_t e0 = start[(size_t)r];
            if (d <= 0) continue;
            size_t cap = 16;
            while (cap < (size_t)(2 * d)) cap <<= 1;
            if (table.size() < cap) table.assign(cap, -1);
            const int shift = 64 - __builtin_ctzll((unsigned long long)cap);
            used.clear();
            auto insert = [&](int32_t c) {
                size_t h = (size_t)(((uint64_t)(uint32_t)c * 0x9E3779B97F4A7C15ull) >> shift);
                while (table[h] != -1) {
                    if (table[h] == c) return false;
                    h = (h + 1) & (cap - 1);
                }
                table[h] = c;
                used.push_back((uint32_t)h);
                return true;
            };
            uint64_t st = splitmix64(seed ^ ((uint64_t)r << 20) ^ 0xabcdefull);
            int64_t got = 0, tries = 0;
            const int64_t max_tries = 64 * d + 1024;
            while (got < d) {
                st = splitmix64(st);
                int32_t col = (int32_t)((st >> 32) % (uint64_t)n);
                if (tries++ < max_tries) {
                    const double u = (double)(st & 0xffffffffull) * (1.0 / 4294967296.0);
                    if (u >= prob[(size_t)col]) col = alias[(size_t)col];
                }
                if (!insert(col)) continue;
                src[(size_t)(e0 + got)] = id[(size_t)r];
                dst[(size_t)(e0 + got)] = id[(size_t)col];
                ++got;
            }
            for (uint32_t h : used) table[h] = -1;
        }
    }
    mrg_csr* m = csr_from_edges(n, src, dst);
    fill_values(m, seed);
    return m;
}

mrg_csr* mrg_banded(int32_t n, int32_t bandwidth, uint64_t seed)
{
    if (n <= 0 || bandwidth <= 0) return nullptr;
    const int32_t h = bandwidth / 2;
    auto* m = new mrg_csr;
    m->n = n;
    m->rowptr.resize((size_t)n + 1);
    m->rowptr[0] = 0;
    for (int32_t r = 0; r < n; ++r)
        m->rowptr[(size_t)r + 1] = m->rowptr[(size_t)r] + (std::min(n - 1, r + h) - std::max(0, r - h) + 1);
    m->colidx.resize((size_t)m->rowptr[(size_t)n]);
#pragma omp parallel for schedule(static)
    for (int32_t r = 0; r < n; ++r) {
        int32_t k = m->rowptr[(size_t)r];
        for (int32_t c = std::max(0, r - h); c <= std::min(n - 1, r + h); ++c) m->colidx[(size_t)k++] = c;
    }
    fill_values(m, seed);
    return m;
}

mrg_csr* mrg_from_csr(int32_t n, const int32_t* rowptr, const int32_t* colidx, const float* vals)
{
    auto* m = new mrg_csr;
    m->n = n;
    m->rowptr.assign(rowptr, rowptr + n + 1);
    m->colidx.assign(colidx, colidx + rowptr[n]);
    if (vals) m->vals.assign(vals, vals + rowptr[n]);
    return m;
}

int mrg_relabel(mrg_csr* m, const int32_t* perm_old2new)
{
    if (!m) return 1;
    relabel(m, std::vector<int32_t>(perm_old2new, perm_old2new + m->n));
    return 0;
}

// Matrix Market reader with the reference's semantics (BASEGRAPH ctor,
// src/class.cu:5-73): "symmetric" in the banner line doubles every entry
// (the mirrored copies are appended after the Nnz listed ones, diagonal
// entries included); "basezero" in the banner means 0-based indices; values
// are forced to 1.0 unless keep_values. The reference multiplies the
// transpose of the file's matrix (its col_ind is the SpMV row, :1342), so the
// CSR returned here has row = file column and column = file row, sorted by
// (row, column) with duplicates kept in file order. Blank lines are skipped.
// *err: 0 ok, 1 cannot open, 2 bad header, 3 bad entry / index out of range.
mrg_csr* mrg_read_mtx(const char* path, int keep_values, int* err)
{
    auto fail = [&](int e) -> mrg_csr* { if (err) *err = e; return nullptr; };
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(1);
    std::vector<char> line(1 << 16);
    bool first = true, symmetric = false, zero_base = false;
    long long R = -1, Cc = -1, N = -1;
    while (std::fgets(line.data(), (int)line.size(), f)) {
        std::string l(line.data());
        if (first) {
            symmetric = l.find("symmetric") != std::string::npos;
            zero_base = l.find("basezero") != std::string::npos;
            first = false;
        }
        if (!l.empty() && l[0] == '%') continue;
        if (std::sscanf(l.c_str(), "%lld %lld %lld", &R, &Cc, &N) == 3) break;
        if (l.find_first_not_of(" \t\r\n") == std::string::npos) continue;
        std::fclose(f);
        return fail(2);
    }
    if (R < 0 || Cc < 0 || N < 0 || R > INT32_MAX || Cc > INT32_MAX || (symmetric ? 2 * N : N) > INT32_MAX) {
        std::fclose(f);
        return fail(2);
    }
    const int64_t total = symmetric ? 2 * N : N;
    std::vector<int32_t> rows((size_t)total), cols((size_t)total);
    std::vector<float> vals(keep_values ? (size_t)total : 0);
    int64_t i = 0;
    const int32_t n = (int32_t)std::max(R, Cc);
    while (i < N && std::fgets(line.data(), (int)line.size(), f)) {
        long long r, c;
        double v = 1.0;
        const int k = std::sscanf(line.data(), "%lld %lld %lf", &r, &c, &v);
        if (k < 2) continue;  // blank or comment line
        if (!zero_base) { --r; --c; }
        if (r < 0 || c < 0 || r >= n || c >= n) { std::fclose(f); return fail(3); }
        // SpMV row = file column, SpMV column = file row
        rows[(size_t)i] = (int32_t)c;
        cols[(size_t)i] = (int32_t)r;
        if (keep_values) vals[(size_t)i] = (float)v;
        if (symmetric) {
            rows[(size_t)(N + i)] = (int32_t)r;
            cols[(size_t)(N + i)] = (int32_t)c;
            if (keep_values) vals[(size_t)(N + i)] = (float)v;
        }
        ++i;
    }
    std::fclose(f);
    if (i != N) return fail(3);
    // counting sort by row (stable in file order), then stable sort by column
    auto* m = new mrg_csr;
    m->n = n;
    m->rowptr.assign((size_t)n + 1, 0);
    for (int64_t e = 0; e < total; ++e) ++m->rowptr[(size_t)rows[(size_t)e] + 1];
    for (int32_t r = 0; r < n; ++r) m->rowptr[(size_t)r + 1] += m->rowptr[(size_t)r];
    std::vector<int32_t> fill(m->rowptr.begin(), m->rowptr.end() - 1);
    std::vector<int64_t> src((size_t)total);
    for (int64_t e = 0; e < total; ++e) src[(size_t)fill[(size_t)rows[(size_t)e]]++] = e;
    m->colidx.resize((size_t)total);
    m->vals.resize((size_t)total);
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t r = 0; r < n; ++r) {
        auto b = src.begin() + m->rowptr[(size_t)r], e = src.begin() + m->rowptr[(size_t)r + 1];
        std::stable_sort(b, e, [&](int64_t a, int64_t q) { return cols[(size_t)a] < cols[(size_t)q]; });
        for (auto it = b; it != e; ++it) {
            const size_t k = (size_t)(it - src.begin());
            m->colidx[k] = cols[(size_t)*it];
            m->vals[k] = keep_values ? vals[(size_t)*it] : 1.0f;
        }
    }
    if (err) *err = 0;
    return m;
}

// The reference's controlled perturbation local_swap (src/class.cu:236-301):
// rho*n seeded swaps of i with a j drawn from [i-window, i-near] or
// [i+near, i+window] (side chosen in proportion to the lengths). Uses the
// same standard-library engine and distributions, so a given seed gives the
// reference's permutation on the same C++ standard library.
void mrg_local_swap(int32_t n, float rho, int32_t near_, int32_t window, uint64_t seed, int32_t* permutation)
{
    std::mt19937_64 rng(seed);
    const int n_swaps = (int)std::llround(rho * (double)n);
    std::vector<int> list((size_t)n);
    std::iota(list.begin(), list.end(), 0);
    std::shuffle(list.begin(), list.end(), rng);
    list.resize((size_t)n_swaps);
    for (int i : list) {
        const int l1 = std::max(0, i - window), r1 = std::min(n - 1, i - near_);
        const int l2 = std::max(0, i + near_), r2 = std::min(n - 1, i + window);
        const int len1 = (l1 <= r1) ? (r1 - l1 + 1) : 0;
        const int len2 = (l2 <= r2) ? (r2 - l2 + 1) : 0;
        if (len1 + len2 == 0) continue;
        bool left;
        if (len1 > 0 && len2 > 0) {
            std::bernoulli_distribution pick(double(len1) / double(len1 + len2));
            left = pick(rng);
        } else {
            left = len1 > 0;
        }
        int j;
        if (left) {
            std::uniform_int_distribution<int> u(l1, r1);
            j = u(rng);
        } else {
            std::uniform_int_distribution<int> u(l2, r2);
            j = u(rng);
        }
        if (j != i) std::swap(permutation[i], permutation[j]);
    }
}

int32_t mrg_n(const mrg_csr* m) { return m ? m->n : 0; }
int64_t mrg_nnz(const mrg_csr* m) { return m ? (int64_t)m->colidx.size() : 0; }
const int32_t* mrg_rowptr(const mrg_csr* m) { return m->rowptr.data(); }
const int32_t* mrg_colidx(const mrg_csr* m) { return m->colidx.data(); }
const float* mrg_vals(const mrg_csr* m) { return m->vals.data(); }

void mrg_copy(const mrg_csr* m, int32_t* rowptr, int32_t* colidx, float* vals)
{
    std::memcpy(rowptr, m->rowptr.data(), sizeof(int32_t) * m->rowptr.size());
    std::memcpy(colidx, m->colidx.data(), sizeof(int32_t) * m->colidx.size());
    if (vals) std::memcpy(vals, m->vals.data(), sizeof(float) * m->vals.size());
}

void mrg_free(mrg_csr* m) { delete m; }

void mrg_uniform(uint64_t seed, int64_t count, float* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) out[i] = unit_pm1(seed, (uint64_t)i);
}

void mrg_random_perm(int32_t n, uint64_t seed, int32_t* out)
{
    std::vector<int32_t> p = random_perm(n, seed);
    std::memcpy(out, p.data(), sizeof(int32_t) * (size_t)n);
}

int mrg_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
