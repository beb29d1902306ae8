"""The allocation-free fast-scan entry point against the allocating one.

qg_fast_scan_noalloc_dev serves callers that cannot let a library allocate
GPU memory (a process that reserves the device for its own pool, a host
framework whose allocator is the only one allowed, a latency-critical loop
where cudaMalloc's device synchronisation or an out-of-memory failure is not
acceptable). It must give exactly the sums of qg_fast_scan_dev, call after
call, from its one shared static scratch array.

This file sorts last so that a run stopping at the first failure has run
every other test first; it also passes on its own in a fresh process (the
first call sets the scratch address up).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _call(L, fn, luts, codes, lut_of, m, n):
    sums = torch.full((n,), -1, dtype=torch.int16, device="cuda")
    tl = torch.from_numpy(luts).cuda()
    tc = torch.from_numpy(codes).cuda()
    to = torch.from_numpy(lut_of).cuda()
    L.check(fn(tl.data_ptr(), luts.shape[0], m, tc.data_ptr(), to.data_ptr(), n, sums.data_ptr(),
               torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return sums.cpu().numpy().view(np.uint16)


def _pool_bytes():
    """(reserved, used, used high-water mark) of the device's default
    stream-ordered pool, and the device's free bytes."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    out = []
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
                 rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return tuple(out) + (torch.cuda.mem_get_info()[0],)


def _reset_pool_high_water():
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    from cuda.bindings import driver as drv
    attr = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    for value in (drv.cuuint64_t(0), 0):   # the binding's value type differs between releases
        try:
            err, = rt.cudaMemPoolSetAttribute(pool, attr, value)
            break
        except TypeError:
            continue
    assert err == rt.cudaError_t.cudaSuccess


def test_no_alloc_sums_equal_the_allocating_entry_point_twice_in_a_row():
    from qann_b200 import _lib as L
    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    for call, (m, n) in enumerate([(50, 64 * 37 + 5), (64, 64 * 200 + 63)]):
        rng = np.random.default_rng(1000 + call)
        nl = 5
        luts = rng.integers(0, 64, size=(nl, m, 16), dtype=np.uint8)
        codes = rng.integers(0, 16, size=(n, m), dtype=np.uint8)
        lut_of = rng.integers(0, nl, size=(n + 63) // 64, dtype=np.uint32)
        want = _call(L, L.lib.qg_fast_scan_dev, luts, codes, lut_of, m, n)
        got = _call(L, L.lib.qg_fast_scan_noalloc_dev, luts, codes, lut_of, m, n)
        # integer sums: the tolerance is exact equality
        np.testing.assert_array_equal(got, want)


def test_no_alloc_call_takes_no_device_memory():
    """After a first call (which loads the library's kernels and looks the
    scratch up), further calls leave the stream-ordered pool and the
    device's free memory exactly as they were."""
    from qann_b200 import _lib as L
    m, n = 64, 64 * 300 + 17
    rng = np.random.default_rng(7)
    luts = torch.from_numpy(rng.integers(0, 64, size=(3, m, 16), dtype=np.uint8)).cuda()
    codes = torch.from_numpy(rng.integers(0, 16, size=(n, m), dtype=np.uint8)).cuda()
    lut_of = torch.from_numpy(rng.integers(0, 3, size=(n + 63) // 64, dtype=np.uint32)).cuda()
    sums = torch.empty((n,), dtype=torch.int16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def call():
        L.check(L.lib.qg_fast_scan_noalloc_dev(luts.data_ptr(), 3, m, codes.data_ptr(), lut_of.data_ptr(), n,
                                               sums.data_ptr(), st))

    call()
    torch.cuda.synchronize()
    _reset_pool_high_water()
    before = _pool_bytes()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    after = _pool_bytes()
    assert after == before, (before, after)
    assert after[2] == after[1], "a stream-ordered allocation happened during the calls"


def test_no_alloc_reports_a_lut_index_out_of_range():
    """A LUT index beyond nluts is caught on the device and refused, in both
    the allocation-free and the allocating entry point, without a read
    outside the LUT buffer."""
    from qann_b200 import _lib as L
    m, n, nl = 16, 64 * 10, 4
    rng = np.random.default_rng(3)
    luts = rng.integers(0, 64, size=(nl, m, 16), dtype=np.uint8)
    codes = rng.integers(0, 16, size=(n, m), dtype=np.uint8)
    lut_of = rng.integers(0, nl, size=n // 64, dtype=np.uint32)
    lut_of[6] = nl
    lut_of[8] = 1 << 30
    for fn in (L.lib.qg_fast_scan_noalloc_dev, L.lib.qg_fast_scan_dev):
        with pytest.raises(ValueError, match=r"lut_of\[6\]"):
            _call(L, fn, luts, codes, lut_of, m, n)
    # the scratch and the library stay usable
    lut_of[6] = lut_of[8] = 0
    np.testing.assert_array_equal(_call(L, L.lib.qg_fast_scan_noalloc_dev, luts, codes, lut_of, m, n),
                                  _call(L, L.lib.qg_fast_scan_dev, luts, codes, lut_of, m, n))


def test_no_alloc_refuses_inputs_beyond_its_scratch():
    from qann_b200 import _lib as L
    # ~128 MB of repacked codes, beyond the 32 MiB scratch; and sizes whose
    # byte counts would wrap a 64-bit product
    for m, n in ((64, 4_000_000), (1024, 1 << 62), (4, (1 << 64) - 1)):
        rc = L.lib.qg_fast_scan_noalloc_dev(None, 1, m, None, None, n, None, None)
        assert rc == L.INVALID_ARGUMENT
        assert "scratch" in L.lib.qg_last_error().decode()
