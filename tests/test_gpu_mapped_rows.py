"""load(mmap=True): a RefineIndex whose raw rows stay in the mapped file and
are read in place by the re-rank (host-mapped memory) returns exactly what
the same index loaded into GPU memory returns, and what the reference
returns; adds and compaction copy the rows into memory first and keep the
results equal."""
import filecmp

import numpy as np
import pytest

import qann_b200 as qb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["refine_l2", "refine_cos_l2", "refine_ip", "refine_l2_custom_del"])
def test_mapped_rows_same_results(golden, ref, name):
    path = golden / "gen" / f"{name}.qann"
    q = np.load(golden / "gen" / "queries.npy")
    mapped, plain = qb.load(path, mmap=True), qb.load(path)
    i1, d1 = mapped.batch_query(q, 10)
    assert mapped.rows_mapped in (1, 2)
    i0, d0 = plain.batch_query(q, 10)
    np.testing.assert_array_equal(i1, i0)
    assert d1.tobytes() == d0.tobytes()
    np.testing.assert_array_equal(i1, np.load(golden / "gen" / f"{name}_ids.npy"))
    ri, rd = ref.load(path).batch_query(q, 10)
    np.testing.assert_array_equal(i1, ri)
    assert d1.tobytes() == rd.tobytes()


def test_mapped_rows_read_in_place(golden):
    idx = qb.load(golden / "gen" / "refine_l2.qann", mmap=True)
    idx.batch_query(np.load(golden / "gen" / "queries.npy")[:4], 10)
    # 2 where the driver registers the mapped pages (or a private view of
    # them) for device reads
    import ctypes as C
    err = C.c_int64()
    qb.check(qb._lib.lib.qg_get_option(b"mapped_rows_error", C.byref(err)))
    assert idx.rows_mapped == 2, f"registration refused: cudaError codes {err.value}"


def test_mapped_rows_then_add_remove_compact(golden, tmp_path):
    path = golden / "gen" / "refine_l2.qann"
    q = np.load(golden / "gen" / "queries.npy")
    rng = np.random.default_rng(5)
    extra = rng.normal(size=(300, q.shape[1])).astype(np.float32)
    results = []
    for mmap in (True, False):
        idx = qb.load(path, mmap=mmap)
        idx.batch_query(q[:2], 10)   # the device copy (mapped rows) exists before the change
        idx.add(extra)
        assert idx.rows_mapped == 0
        idx.remove(np.arange(0, 200, 3))
        idx.compact()
        out = tmp_path / f"after_{int(mmap)}.qann"
        idx.save(out)
        results.append((idx.batch_query(q, 10), out))
    (a, fa), (b, fb) = results
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1].tobytes() == b[1].tobytes()
    assert filecmp.cmp(fa, fb, shallow=False)
