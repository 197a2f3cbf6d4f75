"""ctypes wrappers of the CPU oracle (liboracle.so) and of the reference's own
code built from its sources (oracle/_ref/libmr_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's CPU-baseline
leg, never by the product. See oracle.h for what each function restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBORACLE = os.path.join(HERE, "liboracle.so")
LIBREF = os.path.join(HERE, "_ref", "libmr_ref.so")

_orc = None
_ref = None


def _sig(f, res, *args):
    f.restype = res
    f.argtypes = list(args)


def build() -> None:
    """Builds liboracle.so (always possible: plain C)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(LIBORACLE):
            build()
        L = C.CDLL(LIBORACLE)
        vp, i32, i64, u32 = C.c_void_p, C.c_int, C.c_int64, C.c_uint32
        _sig(L.orc_spmv_csr_f64, None, i32, vp, vp, vp, vp, vp)
        _sig(L.orc_spmv_csr_f32_omp, C.c_int, i32, vp, vp, vp, vp, vp, i32)
        _sig(L.orc_merbit_plan, C.c_int, vp, i32, i32, i32, vp, vp, vp)
        _sig(L.orc_merbit_sizes, None, i32, i32, i32, C.POINTER(C.c_int), C.POINTER(C.c_int))
        _sig(L.orc_permute_csr, None, i32, vp, vp, vp, vp, vp, vp, vp)
        _sig(L.orc_rd_hist_exact, None, vp, i64, i32, i32, vp, i32, vp, vp)
        _sig(L.orc_hll_sampled, None, vp, i32, i32, i32, u32, i32, i32, i32, vp, vp, vp)
        _sig(L.orc_hll_bin, None, i32, vp, vp, vp, i32, vp, vp, vp, vp, vp)
        _sig(L.orc_pgorder, None, i32, vp, vp, i32, i32, vp)
        _sig(L.orc_get_width, C.c_int, i32, i32)
        _sig(L.orc_predict, C.c_double, vp, C.c_double, vp)
        _sig(L.orc_order_random, None, i32, u32, vp)
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(LIBREF)


def ref():
    """The reference's own code (None if it was not built here)."""
    global _ref
    if _ref is None:
        if not ref_available():
            return None
        L = C.CDLL(LIBREF)
        vp, i32, u32 = C.c_void_p, C.c_int, C.c_uint32
        _sig(L.ref_get_width, C.c_int, i32, i32)
        _sig(L.ref_rd_hist_exact, None, vp, i32, i32, i32, vp, i32, vp)
        _sig(L.ref_pgorder_host, None, i32, vp, vp, vp, vp, i32, i32, vp)
        _sig(L.ref_predict, C.c_double, vp)
        _sig(L.ref_local_swap, None, i32, C.c_float, i32, i32, C.c_ulonglong, vp)
        _sig(L.ref_tile_build, C.c_int, vp, i32, i32, vp, vp, vp)
        _sig(L.ref_merbit_spmv, C.c_int, vp, vp, vp, i32, i32, vp, vp, vp, vp, vp, vp, i32, C.POINTER(C.c_float))
        _sig(L.ref_hll_sampled, C.c_int, vp, i32, i32, i32, u32, i32, i32, i32, vp, vp, vp)
        _sig(L.ref_relabel_sort, C.c_int, i32, i32, vp, vp, vp, vp)
        _sig(L.ref_gorder4_full, C.c_int, i32, i32, vp, vp, vp, i32, i32, vp)
        _sig(L.ref_relabel_order, C.c_int, i32, i32, i32, vp, vp, vp, i32, vp)
        _sig(L.ref_shuffle_host, C.c_int, i32, u32, vp)
        _sig(L.ref_cusparse_spmv, C.c_int, vp, vp, vp, i32, i32, vp, vp, i32, C.POINTER(C.c_float))
        _ref = L
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.int32)


# ---------------------------------------------------------------- oracle ----

def spmv_f64(rowptr, colidx, vals, x) -> np.ndarray:
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    vals = np.ascontiguousarray(vals, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty(rowptr.size - 1, np.float64)
    orc().orc_spmv_csr_f64(rowptr.size - 1, _p(rowptr), _p(colidx), _p(vals), _p(x), _p(y))
    return y


def spmv_f32_omp(rowptr, colidx, vals, x, y, threads: int = 0) -> int:
    return orc().orc_spmv_csr_f32_omp(rowptr.size - 1, _p(rowptr), _p(colidx), _p(vals), _p(x), _p(y), threads)


def merbit_plan(rowptr, nnz: int, sigma: int = 14):
    rowptr = _i32(rowptr)
    n = rowptr.size - 1
    ln, tn = C.c_int(), C.c_int()
    orc().orc_merbit_sizes(n, nnz, sigma, C.byref(ln), C.byref(tn))
    tx = np.zeros(tn.value + 1, np.uint32)
    ty = np.zeros(tn.value + 1, np.uint32)
    ld = np.zeros(ln.value, np.uint64)
    rc = orc().orc_merbit_plan(_p(rowptr), n, nnz, sigma, _p(tx), _p(ty), _p(ld))
    assert rc == 0
    return tx, ty, (ld.astype(np.uint32) if sigma < 15 else ld)


def permute_csr(rowptr, colidx, vals, perm):
    rowptr, colidx, perm = _i32(rowptr), _i32(colidx), _i32(perm)
    vals = np.ascontiguousarray(vals, np.float32)
    n = rowptr.size - 1
    orp = np.empty(n + 1, np.int32)
    oci = np.empty(colidx.size, np.int32)
    ov = np.empty(colidx.size, np.float32)
    orc().orc_permute_csr(n, _p(rowptr), _p(colidx), _p(vals), _p(perm), _p(orp), _p(oci), _p(ov))
    return orp, oci, ov


def rd_hist_exact(stream, ncols: int, sector: int = 32, edges=None):
    from_edges = [1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824] if edges is None else edges
    e = _i32(from_edges)
    s = _i32(stream)
    counts = np.zeros(e.size + 1, np.int64)
    valid = np.zeros(1, np.int64)
    orc().orc_rd_hist_exact(_p(s), s.size, ncols, sector, _p(e), e.size, _p(counts), _p(valid))
    return counts, int(valid[0])


def hll_sampled(stream, samples: int, sector: int = 32, seed: int = 246813579, rd_cap: int = 589824,
                max_scan: int = 0, hll_p: int = 12):
    s = _i32(stream)
    est = np.zeros(samples, np.float32)
    st = np.zeros(samples, np.int32)
    pos = np.zeros(samples, np.int32)
    orc().orc_hll_sampled(_p(s), s.size, samples, sector, seed, rd_cap, max_scan, hll_p, _p(est), _p(st), _p(pos))
    return est, st, pos


def hll_bin(est, status, edges=None):
    e = _i32([1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824] if edges is None else edges)
    est = np.ascontiguousarray(est, np.float32)
    status = _i32(status)
    counts = np.zeros(e.size + 1, np.int64)
    f, c, l, u = (C.c_int64() for _ in range(4))
    orc().orc_hll_bin(est.size, _p(est), _p(status), _p(e), e.size, _p(counts), C.byref(f), C.byref(c), C.byref(l),
                      C.byref(u))
    return counts, np.array([f.value, c.value, l.value, u.value], np.int64)


def pgorder(rowptr, colidx, vsize: int, width: int = 5) -> np.ndarray:
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    n = rowptr.size - 1
    out = np.empty(n, np.uint32)
    orc().orc_pgorder(n, _p(rowptr), _p(colidx), vsize, width, _p(out))
    return out


def get_width(nrow: int, nnz: int) -> int:
    return orc().orc_get_width(nrow, nnz)


def predict(coef, intercept: float, r) -> float:
    c = np.ascontiguousarray(coef, np.float64)
    rr = np.ascontiguousarray(r, np.float64)
    return orc().orc_predict(_p(c), intercept, _p(rr))


# ------------------------------------------------------------- reference ----

def csc_of(rowptr, colidx):
    """Column lists of a CSR matrix, rows ascending in each column (the
    reference's sort(true) + coo2csr, src/class.cu:2629-2631)."""
    n = rowptr.size - 1
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
    order = np.lexsort((rows, colidx))
    ind = rows[order].astype(np.int32)
    off = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(colidx, minlength=n), out=off[1:])
    return off, ind


def ref_pgorder(rowptr, colidx, vsize: int, width: int = 5) -> np.ndarray:
    rowptr, colidx = _i32(rowptr), _i32(colidx)
    off1, ind1 = csc_of(rowptr, colidx)
    n = rowptr.size - 1
    out = np.empty(n, np.uint32)
    ref().ref_pgorder_host(n, _p(off1), _p(ind1), _p(rowptr), _p(colidx), vsize, width, _p(out))
    return out


def ref_rd_probs(stream, ncols: int, sector: int = 32, edges=None) -> np.ndarray:
    e = _i32([1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824] if edges is None else edges)
    s = _i32(stream)
    probs = np.zeros(e.size + 1, np.float64)
    ref().ref_rd_hist_exact(_p(s), ncols, s.size, sector, _p(e), e.size, _p(probs))
    return probs


def ref_get_width(nrow: int, nnz: int) -> int:
    return ref().ref_get_width(nrow, nnz)


def ref_predict(r) -> float:
    rr = np.ascontiguousarray(r, np.float64)
    return ref().ref_predict(_p(rr))


def ref_local_swap(n: int, rho: float, near: int, window: int, seed: int) -> np.ndarray:
    p = np.arange(n, dtype=np.int32)
    ref().ref_local_swap(n, rho, near, window, seed, _p(p))
    return p


# ------------------------------------------------ comparator producers ----

def order_degree(rowptr, colidx):
    """GRAPH::relabel_degree (src/class.cu:1493-1549): degree of v = count
    of v in the column indices (desc_kernel1 over row_ind, :473-481);
    decreasing degree, ties by increasing id (stable radix sort_by_key);
    perm[seq[k]] = k."""
    n = len(rowptr) - 1
    deg = np.bincount(np.asarray(colidx, np.int64), minlength=n)[:n]
    order = np.lexsort((np.arange(n), -deg))
    perm = np.empty(n, np.int32)
    perm[order] = np.arange(n, dtype=np.int32)
    return perm


def order_random(n: int, seed: int) -> np.ndarray:
    """GRAPH::relabel_random (src/class.cu:1460-1491): thrust::shuffle of the
    identity with default_random_engine(graph_id) (oracle.c restatement of
    Thrust's Feistel-bijection shuffle); perm[old] = new."""
    perm = np.empty(n, np.int32)
    orc().orc_order_random(n, seed, _p(perm))
    return perm


def ref_shuffle(n: int, seed: int) -> np.ndarray:
    """Thrust's own shuffle (host backend) of the identity, seeded as
    relabel_random seeds it (oracle/_ref)."""
    out = np.empty(n, np.int32)
    ref().ref_shuffle_host(n, seed, _p(out))
    return out


def order_dbg(rowptr, colidx):
    """GRAPH::dbg (src/class.cu:1660-1760): class ceilf(log2(deg + 1.0))
    computed in double then rounded to float (dbg_kernel, :1682-1690),
    decreasing class, increasing id (DegIdCompare, :1673-1679)."""
    n = len(rowptr) - 1
    deg = np.bincount(np.asarray(colidx, np.int64), minlength=n)[:n]
    cls = np.ceil(np.log2(deg.astype(np.float64) + 1.0).astype(np.float32)).astype(np.int64)
    order = np.lexsort((np.arange(n), -cls))
    perm = np.empty(n, np.int32)
    perm[order] = np.arange(n, dtype=np.int32)
    return perm
