"""Matrix Market ingestion with the reference's reader semantics and the
reference's local_swap augmentation (next-row items around the path)."""
import os

import numpy as np
import pytest

from conftest import REPO

HAVE_REF = os.path.exists(os.path.join(REPO, "oracle", "_ref", "libmr_ref.so"))


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_general_one_based(M, tmp_path):
    f = _write(tmp_path, "g.mtx", "%%MatrixMarket matrix coordinate real general\n% c\n3 3 4\n1 2 5.0\n3 1 2\n2 2 7\n1 3 1\n")
    rp, ci, v = M.read_mtx(f)
    # SpMV row = file column: file (1,2)->row 1 col 0; (3,1)->row 0 col 2; (2,2)->row 1 col 1; (1,3)->row 2 col 0
    assert rp.tolist() == [0, 1, 3, 4]
    assert ci.tolist() == [2, 0, 1, 0]
    assert np.all(v == 1.0)  # values forced to 1.0 (src/class.cu:61)
    rp, ci, v = M.read_mtx(f, keep_values=True)
    assert v.tolist() == [2.0, 5.0, 7.0, 1.0]


def test_symmetric_doubles_entries_including_diagonal(M, tmp_path):
    f = _write(tmp_path, "s.mtx", "%%MatrixMarket matrix coordinate pattern symmetric\n2 2 2\n1 1\n2 1\n")
    rp, ci, v = M.read_mtx(f)
    # entries (0,0), (1,0) and mirrored (0,0), (0,1): the diagonal appears twice
    assert rp.tolist() == [0, 3, 4]
    assert ci.tolist() == [0, 0, 1, 0]


def test_basezero_and_errors(M, tmp_path):
    f = _write(tmp_path, "z.mtx", "%%MatrixMarket basezero general\n2 2 1\n0 1\n")
    rp, ci, _ = M.read_mtx(f)
    assert rp.tolist() == [0, 0, 1] and ci.tolist() == [0]
    with pytest.raises(ValueError):
        M.read_mtx(str(tmp_path / "missing.mtx"))
    bad = _write(tmp_path, "b.mtx", "%%MatrixMarket general\n2 2 1\n5 1\n")
    with pytest.raises(ValueError):
        M.read_mtx(bad)


def test_generated_matrix_round_trip(M, tmp_path):
    rp, ci, v = M.gen_rmat(scale=10, edge_factor=4, seed=2)
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    lines = ["%%MatrixMarket matrix coordinate real general", f"{n} {n} {ci.size}"]
    # file holds the transpose, so that the reader's SpMV matrix is the original
    lines += [f"{c + 1} {r + 1} {float(val):.9g}" for r, c, val in zip(rows, ci, v)]
    f = _write(tmp_path, "r.mtx", "\n".join(lines) + "\n")
    rp2, ci2, v2 = M.read_mtx(f, keep_values=True)
    assert np.array_equal(rp2, rp) and np.array_equal(ci2, ci) and np.array_equal(v2, v)


@pytest.mark.skipif(not HAVE_REF, reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("n,rho,near,window,seed", [(1000, 0.1, 64, 256, 20260224), (5000, 0.3, 0, 10000, 7),
                                                    (4096, 0.9, 1024, 4096, 20260225), (10, 1.0, 20, 30, 1)])
def test_local_swap_matches_reference(M, O, n, rho, near, window, seed):
    assert np.array_equal(M.local_swap(n, rho, near, window, seed), O.ref_local_swap(n, rho, near, window, seed))
