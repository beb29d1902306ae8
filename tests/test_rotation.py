"""The PCA-balanced rotation's host steps against the reference library
(reference src/rotation.cpp): the Jacobi eigen-solver bit for bit, the
eigenvalue allocation to subspaces, and load()'s orthogonality check. The
GPU steps (means, covariance, rotating rows) are covered end to end by the
byte-identical training tests."""
import ctypes as C
import math

import numpy as np
import pytest

import qann_b200 as qb
from qann_b200 import _lib


def _spd(seed, d):
    rng = np.random.default_rng(seed)
    b = rng.normal(size=(d, d)) * (1.0 + np.arange(d) % 7)
    return b @ b.T / d


def _eigen(a):
    d = a.shape[0]
    a = np.ascontiguousarray(a, np.float64)
    values, vectors = np.empty(d), np.empty((d, d))
    _lib.check(_lib.lib.qg_symmetric_eigen(a.ctypes.data, d, values.ctypes.data, vectors.ctypes.data))
    return values, vectors


@pytest.mark.parametrize("d", [1, 2, 3, 8, 17, 64, 100])
def test_symmetric_eigen_bit_identical(ref, d):
    a = _spd(d, d)
    v1, w1 = _eigen(a)
    v2, w2 = ref.symmetric_eigen(a)
    assert v1.tobytes() == v2.tobytes()
    assert w1.tobytes() == w2.tobytes()


def test_symmetric_eigen_diagonal_and_zero_matrices(ref):
    for a in (np.diag([3.0, 1.0, 2.0, 2.0]), np.zeros((5, 5))):
        v1, w1 = _eigen(a)
        v2, w2 = ref.symmetric_eigen(a)
        assert v1.tobytes() == v2.tobytes() and w1.tobytes() == w2.tobytes()


def _allocation(values, vectors, m):
    """Eigenvalues largest first (stable), each into the open subspace with the
    smallest sum of logs (reference src/rotation.cpp:111-129)."""
    d = len(values)
    order = sorted(range(d), key=lambda e: -values[e])
    width = d // m
    filled, log_sum = [0] * m, [0.0] * m
    r = np.zeros((d, d), np.float32)
    for e in order:
        best = min((b for b in range(m) if filled[b] < width), key=lambda b: (log_sum[b], b))
        log_sum[best] += math.log(max(values[e], 1e-12))
        r[:, best * width + filled[best]] = vectors[:, e].astype(np.float32)
        filled[best] += 1
    return r


@pytest.mark.parametrize("d,m", [(8, 4), (16, 2), (24, 12), (64, 32), (100, 50)])
def test_balanced_rotation_allocation(ref, d, m):
    cov = _spd(100 + d, d)
    out = np.empty((d, d), np.float32)
    _lib.check(_lib.lib.qg_balanced_rotation(cov.ctypes.data, d, m, out.ctypes.data))
    values, vectors = ref.symmetric_eigen(cov)
    assert out.tobytes() == _allocation(values, vectors, m).tobytes()
    np.testing.assert_allclose(out.T @ out, np.eye(d), atol=1e-5)


def test_balanced_rotation_rejects_bad_subspaces():
    cov = np.eye(6)
    out = np.empty((6, 6), np.float32)
    with pytest.raises(ValueError, match="divisible"):
        _lib.check(_lib.lib.qg_balanced_rotation(cov.ctypes.data, 6, 4, out.ctypes.data))


def test_rotated_fixture_loads_and_reports_rotation(golden):
    idx = qb.load(golden / "ref" / "v9_ip_refine_ivf_fs.qann")
    assert idx.base.pq_rotate


def test_load_rejects_non_orthogonal_rotation(golden, tmp_path):
    from oracle import qann_file
    path = golden / "ref" / "v9_ip_refine_ivf_fs.qann"
    rot = qann_file.read(path)["ivf"]["rotation"]
    b = bytearray(path.read_bytes())
    start = bytes(b).find(np.asarray(rot, np.float32).tobytes())
    assert start > 0
    scaled = (np.asarray(rot, np.float32) * 1.5).tobytes()
    b[start:start + len(scaled)] = scaled
    bad = tmp_path / "bad.qann"
    bad.write_bytes(bytes(b))
    with pytest.raises(RuntimeError, match="corrupt file: IVFIndex rotation is not orthogonal"):
        qb.load(bad)
