"""CPU checks of the boundary: the C-ABI library loads and exports every entry
point include/qann_gpu.h declares, argument errors match the reference's
exception classes, and `.qann` files round-trip byte for byte with qann."""
import filecmp
import pathlib
import re

import numpy as np
import pytest

import qann_b200 as qb
from qann_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "qann_gpu.h").read_text()
    declared = set(re.findall(r"\b(qg_[a-z_0-9]+)\s*\(", header))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(_lib.lib, name), name
    assert declared == set(_lib.EXPORTS)


def test_version():
    assert "sm_100a" in qb.version()


def test_constructor_errors_match_reference():
    with pytest.raises(ValueError, match="nlist"):
        qb.IVFIndex(16, 50)
    with pytest.raises(ValueError, match="nprobe"):
        qb.IVFIndex(16, 100, 101)
    with pytest.raises(ValueError, match="dim"):
        qb.FlatIndex(0)
    ivf = qb.IVFIndex(32, 100)
    with pytest.raises(ValueError):
        ivf.enable_pq(16, 256, fast_scan=True)
    with pytest.raises(ValueError):
        ivf.enable_pq(15, fast_scan=True)
    ivf.enable_pq(16, fast_scan=True)
    with pytest.raises(ValueError):
        ivf.pq_distance = qb.PQDistance.SDC
    with pytest.raises(RuntimeError, match="train"):
        ivf.add(np.zeros((3, 32), np.float32))


def test_refine_base_rules():
    base = qb.IVFIndex(16, 100)
    base.enable_pq(8, fast_scan=True)
    with pytest.raises(ValueError, match="k_factor"):
        qb.RefineIndex(base, 0)
    r = qb.RefineIndex(base, 4)
    with pytest.raises(ValueError, match="wrapped"):
        qb.RefineIndex(base, 4)
    with pytest.raises(ValueError, match="RefineIndex"):
        qb.RefineIndex(r, 2)
    custom = qb.FlatIndex(16, custom_ids=True)
    with pytest.raises(ValueError, match="custom ids"):
        qb.RefineIndex(custom)


def test_setters_validate():
    ivf = qb.IVFIndex(16, 100, 10)
    ivf.nprobe = 100
    assert ivf.nprobe == 100
    with pytest.raises(ValueError):
        ivf.nprobe = 0


def test_scan_options_validate():
    """Scan shape options (host state only: no kernel runs): each variant -1..2
    is kept, anything else is refused and leaves the setting as it was."""
    try:
        for variant in (-1, 0, 1, 2):
            qb.set_scan_options(autotune=False, variant=variant)
            assert qb.scan_options()["variant"] == variant
            assert qb.scan_options()["autotune"] == 0
        for bad in (-2, 3):
            with pytest.raises(ValueError, match="scan_variant"):
                qb.set_scan_options(variant=bad)
            assert qb.scan_options()["variant"] == 2
    finally:
        qb.set_scan_options(autotune=True, variant=-1)
    assert qb.scan_options()["variant"] == -1 and qb.scan_options()["autotune"] == 1


def test_filter_options_validate():
    """Tensor-core filter schedule options (host state only): a forced
    epilogue of 0, 8 or 16 warps is kept, anything else is refused and leaves
    the setting as it was."""
    try:
        for warps in (8, 16, 0):
            qb.set_filter_options(autotune=False, epilogue_warps=warps)
            assert qb.filter_options()["epilogue_warps"] == warps
            assert qb.filter_options()["autotune"] == 0
        for bad in (-1, 4, 12, 32):
            with pytest.raises(ValueError, match="filter_epilogue_warps"):
                qb.set_filter_options(epilogue_warps=bad)
            assert qb.filter_options()["epilogue_warps"] == 0
    finally:
        qb.set_filter_options(autotune=True, epilogue_warps=0)
    assert qb.filter_options()["autotune"] == 1


@pytest.mark.parametrize("name", ["gen/refine_l2.qann", "gen/ivf_cos_ip.qann", "gen/ivf_l2_custom_del.qann",
                                  "gen/refine_l2_custom_del.qann", "gen/refine_cos_l2.qann"])
def test_resave_is_byte_identical(golden, tmp_path, name):
    src = golden / name
    idx = qb.load(src)
    out = tmp_path / "x.qann"
    idx.save(out)
    assert filecmp.cmp(src, out, shallow=False)


@pytest.mark.parametrize("name", ["v4_ivf_fs", "v11_ivf_cos_fs", "v12_ivf_cos_l2", "v1_flat", "v2_refine"])
def test_old_versions_load(golden, name):
    idx = qb.load(golden / "ref" / f"{name}.qann")
    assert idx.size() > 0


def test_corrupt_files_raise(tmp_path, golden):
    b = (golden / "gen" / "ivf_l2.qann").read_bytes()
    p = tmp_path / "bad.qann"
    p.write_bytes(b"XXXX" + b[4:])
    with pytest.raises(RuntimeError, match="not a qann index file"):
        qb.load(p)
    p.write_bytes(b[: len(b) // 2])
    with pytest.raises(RuntimeError, match="truncated|corrupt"):
        qb.load(p)
    p.write_bytes(b + b"\0")
    with pytest.raises(RuntimeError, match="unexpected data"):
        qb.load(p)


def test_reference_reads_our_files(ref, golden, tmp_path):
    idx = qb.load(golden / "gen" / "refine_cos_ip.qann")
    out = tmp_path / "ours.qann"
    idx.save(out)
    r = ref.load(out)
    q = np.load(golden / "gen" / "queries.npy")
    ids, _ = r.batch_query(q, 10)
    np.testing.assert_array_equal(ids, np.load(golden / "gen" / "refine_cos_ip_ids.npy"))


def test_where_and_metadata_point_to_the_bitmap_entry_point():
    """where= and add(metadata=) need the reference's metadata store, which
    this library leaves to the caller; the errors name the bitmap query that
    takes the evaluated filter instead (no GPU needed: both are refused
    before any device work)."""
    import qann_b200 as qb
    idx = qb.IVFIndex(8, 100, 2)
    with pytest.raises(NotImplementedError, match="batch_query_bitmap"):
        idx.batch_query(np.zeros((1, 8), np.float32), 1, where={"a": 1})
    with pytest.raises(NotImplementedError, match="batch_query_bitmap"):
        idx.add(np.zeros((1, 8), np.float32), metadata=[{"a": 1}])


def test_mapped_load_keeps_rows_in_the_file_and_saves_the_same_bytes(golden, tmp_path):
    """load(mmap=True) leaves a RefineIndex's raw rows in the mapped file
    (format 10 and later) and writes them back unchanged; no GPU needed."""
    src = golden / "gen" / "refine_l2.qann"
    idx = qb.load(src, mmap=True)
    assert idx.rows_mapped == 1   # mapped; the device copy is made at the first search
    out = tmp_path / "again.qann"
    idx.save(out)
    assert filecmp.cmp(src, out, shallow=False)
    plain = qb.load(src)
    assert plain.rows_mapped == 0
    ivf = qb.load(golden / "gen" / "ivf_l2.qann", mmap=True)   # not a RefineIndex: read as usual
    out2 = tmp_path / "ivf.qann"
    ivf.save(out2)
    assert filecmp.cmp(golden / "gen" / "ivf_l2.qann", out2, shallow=False)
