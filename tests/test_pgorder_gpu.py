"""pGOrder on the GPU (mr_pgorder_gpu): the same permutation as the host
ordering (mr_pgorder, itself bit-identical to the reference's gorder4
tasks) on every matrix family, block size and window, including ragged last
blocks, empty rows, tiny matrices; rejects what its 16-bit queue cannot
hold instead of guessing."""
import numpy as np
import pytest

from conftest import csr_from_dense_pattern, csr_random

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _gpu(M, rp, ci, vsize, width):
    import torch
    A = M.view(_dev(rp), _dev(ci), _dev(np.ones(max(ci.size, 1), np.float32)))
    out = M.pgorder_gpu(A, vsize, width)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def mats(M):
    return {
        "rmat14": M.gen_rmat(scale=14, edge_factor=16, seed=2)[:2],
        "rmat12_ef4": M.gen_rmat(scale=12, edge_factor=4, seed=7)[:2],
        "lap96": M.gen_laplace2d(96, shuffle=True, seed=1)[:2],
        "chung_lu": M.gen_chung_lu(1 << 14, 2.1, 16.0, 1, 2000, seed=3)[:2],
        "band": M.gen_banded(5000, 33, seed=2)[:2],
        "random": csr_random(7000, 40, seed=8, empty_frac=0.3)[:2],
        "tiny": csr_from_dense_pattern([[1], [0, 1], []])[:2],
    }


@pytest.mark.parametrize("name", ["rmat14", "rmat12_ef4", "lap96", "chung_lu", "band", "random", "tiny"])
@pytest.mark.parametrize("vsize,width", [(0, 5), (256, 5), (1000, 3), (64, 1)])
def test_gpu_pgorder_equals_host(M, mats, name, vsize, width):
    rp, ci = mats[name]
    want = M.pgorder(rp, ci, vsize=vsize, width=width)
    got = _gpu(M, rp, ci, vsize, width)
    assert np.array_equal(got, want), (name, vsize, width)


def test_gpu_pgorder_rejects_oversized_blocks(M, mats):
    rp, ci = mats["rmat14"]
    with pytest.raises(M.MRError):
        _gpu(M, rp, ci, 40000, 5)


def test_gpu_pgorder_rmat_s18_and_timing(M):
    import time
    import torch
    rp, ci, _ = M.gen_rmat(scale=18, edge_factor=16, seed=1)
    t0 = time.perf_counter()
    want = M.pgorder(rp, ci, vsize=0, width=5)
    t_host = time.perf_counter() - t0
    _gpu(M, rp, ci, 0, 5)  # warm
    t0 = time.perf_counter()
    got = _gpu(M, rp, ci, 0, 5)
    t_gpu = time.perf_counter() - t0
    assert np.array_equal(got, want)
    print(f"s18 pGOrder host {t_host:.3f} s, GPU {t_gpu:.3f} s")
