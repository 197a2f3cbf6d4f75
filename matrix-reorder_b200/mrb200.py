"""ctypes binding of libmr.so (include/mr.h) and libmr_gen.so.

Python mirror of the library's C-ABI for tests and the benchmark. Device
buffers are torch CUDA tensors (torch is only the allocator and stream
provider here); every compute call goes through libmr.so. If the library is
missing the import of its entry points fails loudly: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBMR_PATH = os.path.join(HERE, "libmr.so")
LIBGEN_PATH = os.path.join(HERE, "libmr_gen.so")

MR_OK = 0
MR_ERR_INVALID_ARG = 1
MR_ERR_CUDA = 2
MR_ERR_NOMEM = 3
MR_ERR_INVALID_PERM = 4
MR_ERR_UNSUPPORTED = 5
MR_ERR_TIMEOUT = 6
MR_ERR_BUSY = 7
MR_ERR_NOT_FOUND = 8
MR_ERR_INTERNAL = 9
MR_ERR_PREDICT = 10

MR_F32, MR_F16, MR_BF16 = 0, 1, 2
MODEL_MERBIT_SAMPLED, MODEL_MERBIT_EXACT, MODEL_CSR_SAMPLED, MODEL_CSR_EXACT = 0, 1, 2, 3
# plan flags (include/mr.h MR_PLAN_*)
PLAN_NO_HUB_CACHE, PLAN_GATHER_NO_L1, PLAN_GATHER_L2_ONLY, PLAN_SMALL_HUB_CACHE = 1, 2, 4, 8


def PLAN_HUB_LIMIT(kcols: int) -> int:
    return int(kcols) << 8

# reference RD bins (src/class.cu:1267)
REF_EDGES = [1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824]


class MRError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = lib().mr_status_string(code).decode()
        last = lib().mr_last_error().decode()
        super().__init__(f"{where}: {msg} ({code})" + (f" [{last}]" if last else ""))


class CsrView(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("nnz", C.c_int64), ("rowptr", C.c_void_p),
                ("colidx", C.c_void_p), ("vals", C.c_void_p), ("dtype", C.c_int32)]


class PlanInfo(C.Structure):
    _fields_ = [("sigma", C.c_int32), ("block", C.c_int32), ("n_rows", C.c_int32), ("nnz", C.c_int64),
                ("lane_num", C.c_int32), ("tile_num", C.c_int32), ("desc_bytes", C.c_int32),
                ("tile_x_dev", C.c_void_p), ("tile_y_dev", C.c_void_p), ("lane_desc_dev", C.c_void_p),
                ("hub_columns", C.c_int32), ("hub_coverage", C.c_double)]


_lib = None
_gen = None


def _sig(f, res, *args):
    f.restype = res
    f.argtypes = list(args)


def lib():
    """Loads libmr.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBMR_PATH):
        raise RuntimeError(f"{LIBMR_PATH} is missing: run build.py (or __graft_entry__.build())")
    L = C.CDLL(LIBMR_PATH)
    vp, i32, i64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
    P = C.POINTER
    _sig(L.mr_status_string, C.c_char_p, C.c_int)
    _sig(L.mr_last_error, C.c_char_p)
    _sig(L.mr_version, C.c_int)
    _sig(L.mr_spmv_csr, C.c_int, P(CsrView), vp, vp, vp)
    _sig(L.mr_merbit_plan_create, C.c_int, P(CsrView), C.c_int, C.c_int, vp, P(vp))
    _sig(L.mr_merbit_plan_create_ex, C.c_int, P(CsrView), C.c_int, C.c_int, C.c_int, vp, P(vp))
    _sig(L.mr_merbit_plan_destroy, C.c_int, vp)
    _sig(L.mr_merbit_plan_get_info, C.c_int, vp, P(PlanInfo))
    _sig(L.mr_spmv_merbit, C.c_int, vp, P(CsrView), vp, vp, vp)
    _sig(L.mr_permute_csr, C.c_int, P(CsrView), vp, vp, vp, vp, vp)
    _sig(L.mr_permute_vector, C.c_int, i32, vp, vp, vp, C.c_int, vp)
    _sig(L.mr_perm_invert, C.c_int, i32, vp, vp, vp)
    _sig(L.mr_check_perm, C.c_int, vp, i32, P(C.c_int), vp)
    _sig(L.mr_predict_speedup, C.c_int, C.c_int, P(C.c_double), P(C.c_double))
    _sig(L.mr_pgorder_width, i32, i32, i64)
    _sig(L.mr_pgorder, C.c_int, i32, vp, vp, i32, i32, i32, vp)
    if hasattr(L, "mr_rd_hist_exact"):
        _sig(L.mr_rd_hist_exact, C.c_int, vp, i64, i32, i32, vp, i32, vp, vp, vp)
        _sig(L.mr_rd_hist_sampled, C.c_int, vp, i32, i32, i32, i32, i32, i32, u32, vp, i32, vp, vp, vp, vp, vp, vp)
        _sig(L.mr_hll_seed, u32, i32, i32)
        _sig(L.mr_locality_predict, C.c_int, vp, i32, i32, i32, vp, P(C.c_float), vp)
    if hasattr(L, "mr_graph_create"):
        _sig(L.mr_graph_create, C.c_int, i32, i64, vp, vp, vp, i32, i32, P(vp))
        _sig(L.mr_graph_destroy, C.c_int, vp)
        _sig(L.mr_graph_gorder4, C.c_int, vp, i32, i32, P(C.c_double), P(C.c_double))
        _sig(L.mr_graph_locality_predict, C.c_int, vp, vp, P(C.c_float))
        _sig(L.mr_graph_spmv, C.c_int, vp, C.c_char_p, i32, vp, vp, P(C.c_double), P(C.c_double))
        _sig(L.mr_graph_get_perm, C.c_int, vp, vp)
        _sig(L.mr_graph_view, C.c_int, vp, P(CsrView))
    _lib = L
    return L


def check(code: int, where: str) -> None:
    if code != MR_OK:
        raise MRError(code, where)


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def torch_dtype_code(t) -> int:
    import torch
    return {torch.float32: MR_F32, torch.float16: MR_F16, torch.bfloat16: MR_BF16}[t.dtype]


def view(rowptr, colidx, vals, n_cols: Optional[int] = None) -> CsrView:
    """CsrView over device tensors (int32 rowptr/colidx, f32/f16/bf16 vals)."""
    n = rowptr.numel() - 1
    v = CsrView(n, n if n_cols is None else n_cols, colidx.numel(), _ptr(rowptr), _ptr(colidx), _ptr(vals),
                torch_dtype_code(vals))
    v._keep = (rowptr, colidx, vals)  # the view owns references to its buffers
    return v


# ---------------------------------------------------------------- SpMV ----

def spmv_csr(A: CsrView, x, y, stream=None) -> None:
    check(lib().mr_spmv_csr(C.byref(A), _ptr(x), _ptr(y), _stream(stream)), "mr_spmv_csr")


class MerbitPlan:
    """Owner of an mr_merbit_plan (the reference's TILE<BLOCK,SIGMA>)."""

    def __init__(self, A: CsrView, sigma: int = 14, block: int = 0, stream=None, hub_cache: bool = True,
                 flags: Optional[int] = None):
        """flags: MR_PLAN_* bits (as returned by autotune); default from hub_cache."""
        h = C.c_void_p()
        if flags is None:
            flags = 0 if hub_cache else PLAN_NO_HUB_CACHE
        check(lib().mr_merbit_plan_create_ex(C.byref(A), sigma, block, flags, _stream(stream), C.byref(h)),
              "mr_merbit_plan_create_ex")
        self.h = h
        self.A = A

    def info(self) -> PlanInfo:
        inf = PlanInfo()
        check(lib().mr_merbit_plan_get_info(self.h, C.byref(inf)), "mr_merbit_plan_get_info")
        return inf

    def spmv(self, x, y, A: Optional[CsrView] = None, stream=None) -> None:
        check(lib().mr_spmv_merbit(self.h, C.byref(A or self.A), _ptr(x), _ptr(y), _stream(stream)),
              "mr_spmv_merbit")

    def descriptors(self):
        """Copies (tile_x, tile_y, lane_desc) to host numpy arrays."""
        import torch
        inf = self.info()
        torch.cuda.synchronize()
        tx = np.empty(inf.tile_num + 1, np.uint32)
        ty = np.empty(inf.tile_num + 1, np.uint32)
        dt = np.uint32 if inf.desc_bytes == 4 else np.uint64
        ld = np.empty(inf.lane_num, dt)
        for arr, p in ((tx, inf.tile_x_dev), (ty, inf.tile_y_dev), (ld, inf.lane_desc_dev)):
            _d2h(arr, p)
        return tx, ty, ld

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().mr_merbit_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _DevArray:
    """Minimal __cuda_array_interface__ holder so torch can view a raw device pointer."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 2, "strides": None}


def dev_view(ptr: int, nbytes: int):
    """uint8 torch tensor aliasing nbytes of device memory at ptr (no copy)."""
    import torch
    return torch.as_tensor(_DevArray(ptr, nbytes), device="cuda")


def _d2h(arr: np.ndarray, dev_ptr: int) -> None:
    """Copies arr.nbytes from a raw device pointer into arr."""
    if arr.nbytes == 0:
        return
    arr.view(np.uint8)[:] = dev_view(dev_ptr, arr.nbytes).cpu().numpy()


# ---------------------------------------------------------- permutation ----

def permute_csr(A: CsrView, perm, out_rowptr, out_colidx, out_vals, stream=None) -> None:
    check(lib().mr_permute_csr(C.byref(A), _ptr(perm), _ptr(out_rowptr), _ptr(out_colidx), _ptr(out_vals),
                               _stream(stream)), "mr_permute_csr")


def permute_vector(perm, inp, out, inverse: bool, stream=None) -> None:
    check(lib().mr_permute_vector(perm.numel(), _ptr(perm), _ptr(inp), _ptr(out), int(inverse), _stream(stream)),
          "mr_permute_vector")


def perm_invert(perm, inv, stream=None) -> None:
    check(lib().mr_perm_invert(perm.numel(), _ptr(perm), _ptr(inv), _stream(stream)), "mr_perm_invert")


def check_perm(perm, stream=None) -> bool:
    v = C.c_int(0)
    check(lib().mr_check_perm(_ptr(perm), perm.numel(), C.byref(v), _stream(stream)), "mr_check_perm")
    return bool(v.value)


# -------------------------------------------------------- RD / predictor ----

def rd_hist_exact(stream_dev, ncols: int, sector: int = 32, edges=REF_EDGES, stream=None):
    e = np.asarray(edges, np.int32)
    counts = np.zeros(len(e) + 1, np.int64)
    valid = np.zeros(1, np.int64)
    check(lib().mr_rd_hist_exact(_ptr(stream_dev), stream_dev.numel(), ncols, sector, e.ctypes.data, len(e),
                                 counts.ctypes.data, valid.ctypes.data, _stream(stream)), "mr_rd_hist_exact")
    return counts, int(valid[0])


def rd_hist_sampled(stream_dev, samples: int = 30960, sector: int = 32, rd_cap: int = 589824, hll_p: int = 12,
                    max_scan: int = 0, seed: int = 246813579, edges=REF_EDGES, est=None, status=None, pos=None,
                    stream=None):
    e = np.asarray(edges, np.int32)
    counts = np.zeros(len(e) + 1, np.int64)
    stats = np.zeros(4, np.int64)
    check(lib().mr_rd_hist_sampled(_ptr(stream_dev), stream_dev.numel(), samples, sector, rd_cap, hll_p, max_scan,
                                   seed, e.ctypes.data, len(e), counts.ctypes.data, stats.ctypes.data, _ptr(est),
                                   _ptr(status), _ptr(pos), _stream(stream)), "mr_rd_hist_sampled")
    return counts, stats


def hll_seed(graph_id: int, stream_type: int = 0) -> int:
    return int(lib().mr_hll_seed(graph_id, stream_type))


def predict_speedup(features, model: int = MODEL_MERBIT_SAMPLED) -> float:
    r = (C.c_double * 10)(*[float(v) for v in features])
    out = C.c_double(0)
    check(lib().mr_predict_speedup(model, r, C.byref(out)), "mr_predict_speedup")
    return out.value


def locality_predict(stream_dev, ncols: int, graph_id: int = 0, stream=None):
    f = np.zeros(10, np.float64)
    s = C.c_float(0)
    check(lib().mr_locality_predict(_ptr(stream_dev), stream_dev.numel(), ncols, graph_id, f.ctypes.data,
                                    C.byref(s), _stream(stream)), "mr_locality_predict")
    return s.value, f


# -------------------------------------------------------------- pGOrder ----

def order_degree(A: CsrView, perm_out, stream=None) -> None:
    """mr_order_degree: perm_out[old] = new (device int32 tensor)."""
    L = lib()
    _sig(L.mr_order_degree, C.c_int, C.POINTER(CsrView), C.c_void_p, C.c_void_p)
    check(L.mr_order_degree(C.byref(A), _ptr(perm_out), _stream(stream)), "mr_order_degree")


def order_dbg(A: CsrView, perm_out, stream=None) -> None:
    L = lib()
    _sig(L.mr_order_dbg, C.c_int, C.POINTER(CsrView), C.c_void_p, C.c_void_p)
    check(L.mr_order_dbg(C.byref(A), _ptr(perm_out), _stream(stream)), "mr_order_dbg")


def order_random(n: int, seed: int, perm_out, stream=None) -> None:
    L = lib()
    _sig(L.mr_order_random, C.c_int, C.c_int32, C.c_uint32, C.c_void_p, C.c_void_p)
    check(L.mr_order_random(n, seed, _ptr(perm_out), _stream(stream)), "mr_order_random")


GATE_SKIP, GATE_RELABEL, GATE_UNCERTAIN = 0, 1, 2
# the trainer's scanned (tau_l, tau_h) pairs, ridge/train.py:91-99
BAND_GATE_PAIRS = [(0.99, 1.01), (0.98, 1.02), (0.97, 1.03), (0.96, 1.04), (0.95, 1.05), (0.94, 1.06), (0.93, 1.07)]


def band_gate(predicted: float, tau_l: float, tau_h: float) -> int:
    L = lib()
    _sig(L.mr_band_gate, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_int32))
    d = C.c_int32(0)
    check(L.mr_band_gate(predicted, tau_l, tau_h, C.byref(d)), "mr_band_gate")
    return d.value


def predict_reorder(stream_dev, ncols: int, graph_id: int = 0, model: int = MODEL_MERBIT_SAMPLED, stream=None):
    """mr_predict_reorder: (predicted speedup, 10 features)."""
    L = lib()
    _sig(L.mr_predict_reorder, C.c_int, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
         C.POINTER(C.c_double), C.c_void_p)
    f = np.zeros(10, np.float64)
    sp = C.c_double(0)
    check(L.mr_predict_reorder(_ptr(stream_dev), stream_dev.numel(), ncols, graph_id, model, f.ctypes.data,
                               C.byref(sp), _stream(stream)), "mr_predict_reorder")
    return sp.value, f


def pgorder_gpu(A: CsrView, vsize: int = 0, width: int = 5, out=None, stream=None):
    """mr_pgorder_gpu: perm_new2old on the device (torch int32 tensor);
    raises MRError(MR_ERR_UNSUPPORTED) where the device queue does not fit."""
    import torch
    L = lib()
    _sig(L.mr_pgorder_gpu, C.c_int, C.POINTER(CsrView), C.c_int32, C.c_int32, C.c_void_p, C.c_void_p)
    if out is None:
        out = torch.empty(A.n_rows, dtype=torch.int32, device="cuda")
    check(L.mr_pgorder_gpu(C.byref(A), vsize, width, _ptr(out), _stream(stream)), "mr_pgorder_gpu")
    return out


def pgorder_width(n: int, nnz: int) -> int:
    return int(lib().mr_pgorder_width(n, nnz))


def pgorder(rowptr: np.ndarray, colidx: np.ndarray, vsize: int = 0, width: int = 5, threads: int = 0) -> np.ndarray:
    """Host pGOrder: returns perm_new2old (uint32)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    n = rowptr.size - 1
    out = np.empty(n, np.uint32)
    check(lib().mr_pgorder(n, rowptr.ctypes.data, colidx.ctypes.data, vsize, width, threads, out.ctypes.data),
          "mr_pgorder")
    return out


# ------------------------------------------------------------ GRAPH object ----

class Graph:
    """Mirror of the reference's GRAPH<float> operator API over mr_graph."""

    def __init__(self, rowptr: np.ndarray, colidx: np.ndarray, vals: np.ndarray, graph_id: int = 0):
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        colidx = np.ascontiguousarray(colidx, np.int32)
        if vals.dtype == np.float32:
            dt = MR_F32
        elif vals.dtype == np.float16:
            dt = MR_F16
        else:
            raise ValueError("vals must be float32 or float16 (bf16 via the C-ABI directly)")
        vals = np.ascontiguousarray(vals)
        h = C.c_void_p()
        check(lib().mr_graph_create(rowptr.size - 1, colidx.size, rowptr.ctypes.data, colidx.ctypes.data,
                                    vals.ctypes.data, dt, graph_id, C.byref(h)), "mr_graph_create")
        self.h = h
        self.n = rowptr.size - 1

    def gorder4(self, vsize: int = 0, width: int = 5):
        a, b = C.c_double(0), C.c_double(0)
        check(lib().mr_graph_gorder4(self.h, vsize, width, C.byref(a), C.byref(b)), "mr_graph_gorder4")
        return a.value, b.value

    def locality_predict(self):
        f = np.zeros(10, np.float64)
        s = C.c_float(0)
        check(lib().mr_graph_locality_predict(self.h, f.ctypes.data, C.byref(s)), "mr_graph_locality_predict")
        return s.value, f

    def gated_reorder(self, model: int = MODEL_MERBIT_SAMPLED, tau_l: float = 0.95, tau_h: float = 1.05,
                      relabel_uncertain: bool = False, vsize: int = 0, width: int = 5):
        """mr_graph_gated_reorder: returns (decision, predicted speedup)."""
        L = lib()
        _sig(L.mr_graph_gated_reorder, C.c_int, C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32,
             C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double))
        d, p = C.c_int32(0), C.c_double(0)
        check(L.mr_graph_gated_reorder(self.h, model, tau_l, tau_h, int(relabel_uncertain), vsize, width, C.byref(d),
                                       C.byref(p)), "mr_graph_gated_reorder")
        return d.value, p.value

    def spmv(self, method: str = "merbit", iters: int = 1, x: Optional[np.ndarray] = None):
        y = np.empty(self.n, np.float32)
        xp = None if x is None else np.ascontiguousarray(x, np.float32)
        a, b = C.c_double(0), C.c_double(0)
        check(lib().mr_graph_spmv(self.h, method.encode(), iters, None if xp is None else xp.ctypes.data,
                                  y.ctypes.data, C.byref(a), C.byref(b)), "mr_graph_spmv")
        return y, a.value, b.value

    def perm(self) -> np.ndarray:
        p = np.empty(self.n, np.int32)
        check(lib().mr_graph_get_perm(self.h, p.ctypes.data), "mr_graph_get_perm")
        return p

    def close(self):
        if getattr(self, "h", None):
            lib().mr_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------- generators ----

def gen():
    global _gen
    if _gen is not None:
        return _gen
    if not os.path.exists(LIBGEN_PATH):
        raise RuntimeError(f"{LIBGEN_PATH} is missing: run build.py")
    G = C.CDLL(LIBGEN_PATH)
    vp = C.c_void_p
    _sig(G.mrg_rmat, vp, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int)
    _sig(G.mrg_laplace2d, vp, C.c_int32, C.c_int, C.c_uint64)
    _sig(G.mrg_chung_lu, vp, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_uint64)
    _sig(G.mrg_banded, vp, C.c_int32, C.c_int32, C.c_uint64)
    _sig(G.mrg_n, C.c_int32, vp)
    _sig(G.mrg_nnz, C.c_int64, vp)
    _sig(G.mrg_copy, None, vp, vp, vp, vp)
    _sig(G.mrg_free, None, vp)
    _sig(G.mrg_uniform, None, C.c_uint64, C.c_int64, vp)
    _sig(G.mrg_random_perm, None, C.c_int32, C.c_uint64, vp)
    _sig(G.mrg_threads, C.c_int)
    _sig(G.mrg_read_mtx, vp, C.c_char_p, C.c_int, C.POINTER(C.c_int))
    _sig(G.mrg_local_swap, None, C.c_int32, C.c_float, C.c_int32, C.c_int32, C.c_uint64, vp)
    _gen = G
    return G


def _take(h):
    G = gen()
    if not h:
        raise ValueError("generator rejected its arguments")
    n, nnz = G.mrg_n(h), G.mrg_nnz(h)
    rp = np.empty(n + 1, np.int32)
    ci = np.empty(nnz, np.int32)
    v = np.empty(nnz, np.float32)
    G.mrg_copy(h, rp.ctypes.data, ci.ctypes.data, v.ctypes.data)
    G.mrg_free(h)
    return rp, ci, v


def gen_rmat(scale: int = 16, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 1, permute_ids=True,
             n: Optional[int] = None):
    """Graph500 R-MAT CSR (duplicates merged, self loops kept), values U[-1,1]."""
    n = (1 << scale) if n is None else n
    return _take(gen().mrg_rmat(n, edge_factor, a, b, c, seed, int(permute_ids)))


def gen_laplace2d(g: int = 2048, shuffle: bool = True, seed: int = 1):
    return _take(gen().mrg_laplace2d(g, int(shuffle), seed))


def gen_chung_lu(n: int, gamma=2.1, mean_deg=20.0, dmin=1, dmax=200000, seed: int = 1):
    return _take(gen().mrg_chung_lu(n, gamma, mean_deg, dmin, dmax, seed))


def gen_banded(n: int, bandwidth: int, seed: int = 1):
    return _take(gen().mrg_banded(n, bandwidth, seed))


def read_mtx(path: str, keep_values: bool = False):
    """Matrix Market file as the CSR the reference multiplies (see gen.cpp)."""
    err = C.c_int(0)
    h = gen().mrg_read_mtx(path.encode(), int(keep_values), C.byref(err))
    if not h:
        raise ValueError(f"cannot read {path}: error {err.value}")
    return _take(h)


def local_swap(n: int, rho: float, near: int, window: int, seed: int) -> np.ndarray:
    """The reference's local_swap perturbation of the identity permutation."""
    p = np.arange(n, dtype=np.int32)
    gen().mrg_local_swap(n, rho, near, window, seed, p.ctypes.data)
    return p


def uniform(count: int, seed: int) -> np.ndarray:
    out = np.empty(count, np.float32)
    gen().mrg_uniform(seed, count, out.ctypes.data)
    return out


def random_perm(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.int32)
    gen().mrg_random_perm(n, seed, out.ctypes.data)
    return out


# --------------------------------------------------------------- batching ----

class BatchItem(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("A", CsrView), ("x", C.c_void_p), ("y", C.c_void_p)]


def _batch_sigs(L):
    if getattr(L, "_batch_sigs", False):
        return
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    P = C.POINTER
    _sig(L.mr_batch_create, C.c_int, P(BatchItem), i32, vp, P(vp))
    _sig(L.mr_batch_run, C.c_int, vp, vp)
    _sig(L.mr_batch_capture, C.c_int, vp, vp)
    _sig(L.mr_batch_launch, C.c_int, vp, vp)
    _sig(L.mr_batch_set_vectors, C.c_int, vp, i32, vp, vp, vp)
    _sig(L.mr_batch_info, C.c_int, vp, P(i32), P(i64))
    _sig(L.mr_batch_destroy, C.c_int, vp)
    _sig(L.mr_autotune_merbit, C.c_int, P(CsrView), vp, vp, i32, P(i32), P(i32), P(i32), P(C.c_float), vp)
    _sig(L.mr_tuner_create, C.c_int, P(vp))
    _sig(L.mr_tuner_destroy, C.c_int, vp)
    _sig(L.mr_tuner_pick, C.c_int, vp, P(CsrView), vp, vp, P(i32), P(i32), P(i32), vp)
    _sig(L.mr_tuner_stats, C.c_int, vp, P(i32), P(i32))
    L._batch_sigs = True


class Batch:
    """mr_batch over (MerbitPlan, x, y) triples; keeps its operands alive."""

    def __init__(self, entries, stream=None):
        L = lib()
        _batch_sigs(L)
        self.entries = list(entries)
        arr = (BatchItem * len(self.entries))()
        for i, (plan, x, y) in enumerate(self.entries):
            arr[i] = BatchItem(plan.h.value, plan.A, _ptr(x), _ptr(y))
        h = C.c_void_p()
        check(L.mr_batch_create(arr, len(self.entries), _stream(stream), C.byref(h)), "mr_batch_create")
        self.h = h

    def run(self, stream=None):
        check(lib().mr_batch_run(self.h, _stream(stream)), "mr_batch_run")

    def capture(self, stream):
        check(lib().mr_batch_capture(self.h, _stream(stream)), "mr_batch_capture")

    def launch(self, stream=None):
        check(lib().mr_batch_launch(self.h, _stream(stream)), "mr_batch_launch")

    def set_vectors(self, i, x, y, stream=None):
        plan = self.entries[i][0]
        self.entries[i] = (plan, x, y)
        check(lib().mr_batch_set_vectors(self.h, i, _ptr(x), _ptr(y), _stream(stream)), "mr_batch_set_vectors")

    def info(self):
        g, t = C.c_int32(0), C.c_int64(0)
        check(lib().mr_batch_info(self.h, C.byref(g), C.byref(t)), "mr_batch_info")
        return g.value, t.value

    def close(self):
        if getattr(self, "h", None):
            lib().mr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(A: CsrView, x, y, reps: int = 5, stream=None):
    L = lib()
    _batch_sigs(L)
    s, b, f, ms = C.c_int32(0), C.c_int32(0), C.c_int32(0), C.c_float(0)
    check(L.mr_autotune_merbit(C.byref(A), _ptr(x), _ptr(y), reps, C.byref(s), C.byref(b), C.byref(f), C.byref(ms),
                               _stream(stream)), "mr_autotune_merbit")
    return s.value, b.value, f.value, ms.value


class Tuner:
    def __init__(self):
        L = lib()
        _batch_sigs(L)
        h = C.c_void_p()
        check(L.mr_tuner_create(C.byref(h)), "mr_tuner_create")
        self.h = h

    def pick(self, A: CsrView, x, y, stream=None):
        s, b, f = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        check(lib().mr_tuner_pick(self.h, C.byref(A), _ptr(x), _ptr(y), C.byref(s), C.byref(b), C.byref(f),
                                  _stream(stream)), "mr_tuner_pick")
        return s.value, b.value, f.value

    def stats(self):
        a, b = C.c_int32(0), C.c_int32(0)
        check(lib().mr_tuner_stats(self.h, C.byref(a), C.byref(b)), "mr_tuner_stats")
        return a.value, b.value

    def close(self):
        if getattr(self, "h", None):
            lib().mr_tuner_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- serving ----

class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("window_us", C.c_int32), ("max_batch", C.c_int32),
                ("lanes", C.c_int32), ("sigma", C.c_int32), ("hub_cache", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("rejected", C.c_int64),
                ("batches", C.c_int64), ("admissions", C.c_int64), ("evictions", C.c_int64),
                ("resident_bytes", C.c_int64), ("resident_matrices", C.c_int64), ("mean_batch", C.c_double),
                ("p50_us", C.c_double), ("p99_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double),
                ("req_per_s", C.c_double), ("h2d_ms", C.c_double), ("compute_ms", C.c_double), ("d2h_ms", C.c_double),
                ("launch_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _server_sigs(L):
    if getattr(L, "_server_sigs", False):
        return
    vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
    P = C.POINTER
    _sig(L.mr_server_create, C.c_int, P(ServerConfig), P(vp))
    _sig(L.mr_server_add_matrix, C.c_int, vp, i32, i64, vp, vp, vp, i32, vp, P(i32))
    _sig(L.mr_server_submit, C.c_int, vp, i32, vp, vp, P(u64))
    _sig(L.mr_server_wait, C.c_int, vp, u64, i32, P(C.c_double))
    _sig(L.mr_server_drain, C.c_int, vp, i32)
    _sig(L.mr_server_get_stats, C.c_int, vp, P(ServerStats))
    _sig(L.mr_server_reset_stats, C.c_int, vp)
    _sig(L.mr_server_destroy, C.c_int, vp)
    _sig(L.mr_server_loadgen, C.c_int, vp, vp, i32, i64, C.c_double, u64, vp, vp, i32)
    _sig(L.mr_plain_requests, C.c_int, i32, vp, vp, vp, i64, vp, vp, vp, vp, P(C.c_double), vp)
    L._server_sigs = True


class Server:
    """mr_server: continuous-batching SpMV over a device-resident pool.
    Host arrays passed to add_matrix / submit are kept referenced here for
    as long as the server may read or write them."""

    def __init__(self, hbm_budget_bytes: int = 0, window_us: int = 200, max_batch: int = 64, lanes: int = 3,
                 sigma: int = 14, hub_cache: bool = False):
        L = lib()
        _server_sigs(L)
        cfg = ServerConfig(hbm_budget_bytes, window_us, max_batch, lanes, sigma, 1 if hub_cache else 0)
        h = C.c_void_p()
        check(L.mr_server_create(C.byref(cfg), C.byref(h)), "mr_server_create")
        self.h = h
        self._keep = []
        self._inflight = {}  # ticket -> (x, y): the server reads x / writes y until the request ends

    def add_matrix(self, rowptr, colidx, vals, perm_old2new=None) -> int:
        """vals: numpy float32 / float16, or a host torch bfloat16 tensor."""
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        colidx = np.ascontiguousarray(colidx, np.int32)
        if str(getattr(vals, "dtype", "")) == "torch.bfloat16":
            import torch
            if vals.is_cuda:
                raise ValueError("vals must be host memory")
            vals = vals.contiguous().view(torch.int16).numpy()  # the BF16 bits
            dt = MR_BF16
        elif vals.dtype == np.float32:
            dt = MR_F32
        elif vals.dtype == np.float16:
            dt = MR_F16
        else:
            raise ValueError("vals must be float32, float16 or a bfloat16 tensor")
        vals = np.ascontiguousarray(vals)
        perm = None if perm_old2new is None else np.ascontiguousarray(perm_old2new, np.int32)
        self._keep.append((rowptr, colidx, vals, perm))
        i = C.c_int32(0)
        check(lib().mr_server_add_matrix(self.h, rowptr.size - 1, colidx.size, rowptr.ctypes.data, colidx.ctypes.data,
                                         vals.ctypes.data, dt, None if perm is None else perm.ctypes.data,
                                         C.byref(i)), "mr_server_add_matrix")
        return i.value

    def submit(self, mid: int, x: np.ndarray, y: np.ndarray) -> int:
        t = C.c_uint64(0)
        check(lib().mr_server_submit(self.h, mid, x.ctypes.data, y.ctypes.data, C.byref(t)), "mr_server_submit")
        self._inflight[t.value] = (x, y)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 10000):
        lat = C.c_double(0)
        rc = lib().mr_server_wait(self.h, ticket, timeout_ms, C.byref(lat))
        if rc != MR_ERR_TIMEOUT:
            self._inflight.pop(ticket, None)
        return rc, lat.value

    def drain(self, timeout_ms: int = 60000):
        check(lib().mr_server_drain(self.h, timeout_ms), "mr_server_drain")
        self._inflight.clear()

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().mr_server_get_stats(self.h, C.byref(st)), "mr_server_get_stats")
        return st.as_dict()

    def reset_stats(self):
        check(lib().mr_server_reset_stats(self.h), "mr_server_reset_stats")

    def loadgen(self, ids, xs, ys, n_requests: int, rate: float, seed: int = 1, timeout_ms: int = 600000):
        ids_a = np.ascontiguousarray(ids, np.int32)
        xp = (C.c_void_p * len(xs))(*[a.ctypes.data for a in xs])
        yp = (C.c_void_p * len(ys))(*[a.ctypes.data for a in ys])
        check(lib().mr_server_loadgen(self.h, ids_a.ctypes.data, ids_a.size, n_requests, rate, seed, xp, yp,
                                      timeout_ms), "mr_server_loadgen")

    def close(self):
        if getattr(self, "h", None):
            lib().mr_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plain_requests(plans, views, perms, req_mat, xs, ys, stream=None):
    """mr_plain_requests: the requests one at a time (H2D, permute, MERBIT
    SpMV, un-permute, D2H, synchronise). plans / views / perms (device
    tensors perm[old] = new) per matrix; req_mat, xs, ys per request (host
    float32 arrays). Returns (elapsed_ms, per-request latencies in us)."""
    L = lib()
    _server_sigs(L)
    k = len(plans)
    ph = (C.c_void_p * k)(*[p.h.value for p in plans])
    vv = (CsrView * k)(*views)
    pp = (C.c_void_p * k)(*[_ptr(t) for t in perms])
    req = np.ascontiguousarray(req_mat, np.int32)
    xp = (C.c_void_p * req.size)(*[a.ctypes.data for a in xs])
    yp = (C.c_void_p * req.size)(*[a.ctypes.data for a in ys])
    lat = np.zeros(req.size, np.float64)
    ms = C.c_double(0)
    check(L.mr_plain_requests(k, ph, vv, pp, req.size, req.ctypes.data, xp, yp, _stream(stream), C.byref(ms),
                              lat.ctypes.data), "mr_plain_requests")
    return ms.value, lat


def gather_ceiling(colidx, vals, x, reps: int = 20, stream=None) -> float:
    """mr_gather_ceiling: ms per pass of the gather-only probe over (colidx,
    vals) device tensors and x."""
    L = lib()
    _sig(L.mr_gather_ceiling, C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32,
         C.POINTER(C.c_float), C.c_void_p)
    ms = C.c_float(0)
    check(L.mr_gather_ceiling(_ptr(colidx), _ptr(vals), colidx.numel(), _ptr(x), reps, C.byref(ms), _stream(stream)),
          "mr_gather_ceiling")
    return ms.value
