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


def test_no_alloc_refuses_inputs_beyond_its_scratch():
    from qann_b200 import _lib as L
    m, n = 64, 4_000_000   # ~128 MB of repacked codes, beyond the 32 MiB scratch
    rc = L.lib.qg_fast_scan_noalloc_dev(None, 1, m, None, None, n, None, None)
    assert rc == L.INVALID_ARGUMENT
    assert "scratch" in L.lib.qg_last_error().decode()
