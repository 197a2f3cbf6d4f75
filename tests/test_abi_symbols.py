"""The C-ABI library loads without a GPU and exports every symbol its public
headers declare; argument checks reject bad input before touching a device."""
import ctypes as C
import os
import re

import pytest

from conftest import REPO


def _declared(header: str):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mr_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(M):
    lib = C.CDLL(M.LIBMR_PATH)
    missing = [s for s in _declared("mr.h") if not hasattr(lib, s)]
    assert not missing, f"declared in include/mr.h but not exported: {missing}"


def test_status_strings(M):
    L = M.lib()
    for code in range(0, 11):
        assert L.mr_status_string(code)
    assert L.mr_version() >= 10000


def test_null_arguments_rejected_without_gpu(M):
    L = M.lib()
    assert L.mr_spmv_csr(None, None, None, None) == M.MR_ERR_INVALID_ARG
    assert L.mr_merbit_plan_create(None, 14, 256, None, None) == M.MR_ERR_INVALID_ARG
    bad = M.CsrView(4, 4, -1, 1, 1, 1, 0)
    h = C.c_void_p()
    assert L.mr_merbit_plan_create(C.byref(bad), 14, 256, None, C.byref(h)) == M.MR_ERR_INVALID_ARG
    bad = M.CsrView(4, 4, 10, 1, 1, 1, 9)
    assert L.mr_spmv_csr(C.byref(bad), 1, 1, None) == M.MR_ERR_UNSUPPORTED
    ok = M.CsrView(4, 4, 10, 1, 1, 1, 0)
    assert L.mr_merbit_plan_create(C.byref(ok), 99, 256, None, C.byref(h)) == M.MR_ERR_INVALID_ARG
    assert L.mr_merbit_plan_create(C.byref(ok), 14, 96, None, C.byref(h)) == M.MR_ERR_UNSUPPORTED
    rect = M.CsrView(4, 5, 10, 1, 1, 1, 0)
    assert L.mr_permute_csr(C.byref(rect), 1, 1, 1, 1, None) == M.MR_ERR_INVALID_ARG
    assert L.mr_predict_speedup(7, None, None) == M.MR_ERR_INVALID_ARG
    raw = C.CDLL(M.LIBMR_PATH)
    assert raw.mr_gather_ceiling(None, None, C.c_int64(1000), None, 5, None, None) == M.MR_ERR_INVALID_ARG
    assert raw.mr_plain_requests(0, None, None, None, C.c_int64(0), None, None, None, None, None,
                                 None) == M.MR_ERR_INVALID_ARG


def test_pgorder_rejects_bad_input(M):
    import numpy as np
    with pytest.raises(M.MRError):
        M.pgorder(np.array([0, 1], np.int32), np.array([5], np.int32), 16, 5)
    with pytest.raises(M.MRError):
        M.pgorder(np.array([0, 1], np.int32), np.array([0], np.int32), 16, 0)
