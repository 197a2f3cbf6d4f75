// Seeded synthetic workload generators (host C++). See gen.cpp.
#ifndef MR_GEN_H
#define MR_GEN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct mrg_csr mrg_csr;

/* Graph500 R-MAT, n rows (2^scale when n is a power of two), n*edge_factor
 * draws, quadrant probabilities a, b, c (d = 1-a-b-c); permute_ids applies
 * GAP's shuffled id map. Duplicates merged, self loops kept. */
mrg_csr* mrg_rmat(int32_t n, int32_t edge_factor, double a, double b, double c, uint64_t seed, int permute_ids);
/* 5-point Laplacian on a g x g grid (4 on the diagonal, -1 off it);
 * shuffle applies a seeded symmetric relabel. */
mrg_csr* mrg_laplace2d(int32_t g, int shuffle, uint64_t seed);
/* Chung-Lu power law: degree exponent gamma, mean degree, degrees clamped. */
mrg_csr* mrg_chung_lu(int32_t n, double gamma, double mean_deg, int32_t dmin, int32_t dmax, uint64_t seed);
/* Banded matrix: |r - c| <= bandwidth/2. */
mrg_csr* mrg_banded(int32_t n, int32_t bandwidth, uint64_t seed);
mrg_csr* mrg_from_csr(int32_t n, const int32_t* rowptr, const int32_t* colidx, const float* vals);
int mrg_relabel(mrg_csr* m, const int32_t* perm_old2new);

/* Matrix Market file with the reference's reader semantics (see gen.cpp);
 * returns the CSR the reference multiplies. *err: 0 ok, 1 open, 2 header,
 * 3 entries. */
mrg_csr* mrg_read_mtx(const char* path, int keep_values, int* err);
/* The reference's local_swap perturbation of `permutation` (in place). */
void mrg_local_swap(int32_t n, float rho, int32_t near_, int32_t window, uint64_t seed, int32_t* permutation);
int32_t mrg_n(const mrg_csr* m);
int64_t mrg_nnz(const mrg_csr* m);
const int32_t* mrg_rowptr(const mrg_csr* m);
const int32_t* mrg_colidx(const mrg_csr* m);
const float* mrg_vals(const mrg_csr* m);
void mrg_copy(const mrg_csr* m, int32_t* rowptr, int32_t* colidx, float* vals);
void mrg_free(mrg_csr* m);
/* count values uniform in [-1, 1) from a counter-based hash of (seed, i) */
void mrg_uniform(uint64_t seed, int64_t count, float* out);
void mrg_random_perm(int32_t n, uint64_t seed, int32_t* out);
int mrg_threads(void);
#ifdef __cplusplus
}
#endif
#endif
