"""Kernel-level parity of the CUDA path with the reference, through the C ABI
on device memory: the uint8 LUT rounding and the integer code sums must be
bit-exact, and exact distances must equal the reference's AVX2 build's."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    from qann_b200 import _lib
    assert torch.cuda.is_available(), "the -m gpu tests need a CUDA device"
    return _lib


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("m", [2, 6, 16, 50, 64, 196, 1024])
def test_quantize_lut_bit_exact(L, ref, m):
    rng = np.random.default_rng(m)
    n = 64
    tables = rng.normal(size=(n, m, 16)).astype(np.float32) * rng.uniform(0.01, 100, size=(n, 1, 1)).astype(np.float32)
    tables[0] = 3.0   # all rows constant: scale 1
    tables[1, :, :8] = -np.float32(7.5)
    t = dev(tables)
    lut = torch.empty((n, m, 16), dtype=torch.uint8, device="cuda")
    sc = torch.empty(n, dtype=torch.float32, device="cuda")
    of = torch.empty(n, dtype=torch.float32, device="cuda")
    L.check(L.lib.qg_quantize_lut_dev(t.data_ptr(), n, m, lut.data_ptr(), sc.data_ptr(), of.data_ptr(), None))
    torch.cuda.synchronize()
    lut, sc, of = lut.cpu().numpy(), sc.cpu().numpy(), of.cpu().numpy()
    for i in range(n):
        rl, rs, ro = ref.quantize_lut(tables[i].ravel())
        np.testing.assert_array_equal(lut[i].ravel(), rl)
        assert sc[i].tobytes() == rs.tobytes() and of[i].tobytes() == ro.tobytes()


@pytest.mark.parametrize("m", [16, 50, 64])
def test_build_quantize_lut_bit_exact(L, ref, m):
    rng = np.random.default_rng(100 + m)
    n = 32
    B = rng.normal(size=(n, m, 16)).astype(np.float32)
    Cq = rng.normal(size=(n, m, 16)).astype(np.float32)
    A = rng.uniform(0, 5, size=n).astype(np.float32)
    lut = torch.empty((n, m, 16), dtype=torch.uint8, device="cuda")
    sc = torch.empty(n, dtype=torch.float32, device="cuda")
    of = torch.empty(n, dtype=torch.float32, device="cuda")
    b, c, a = dev(B), dev(Cq), dev(A)
    L.check(L.lib.qg_build_quantize_lut_dev(b.data_ptr(), c.data_ptr(), a.data_ptr(), n, m, lut.data_ptr(),
                                            sc.data_ptr(), of.data_ptr(), None))
    torch.cuda.synchronize()
    lut, sc, of = lut.cpu().numpy(), sc.cpu().numpy(), of.cpu().numpy()
    for i in range(n):
        _, rl, rs, ro = ref.build_quantize_lut(B[i].ravel(), Cq[i].ravel(), float(A[i]))
        np.testing.assert_array_equal(lut[i].ravel(), rl)
        assert sc[i].tobytes() == rs.tobytes() and of[i].tobytes() == ro.tobytes()


def fs_pack(codes):
    """The reference's fast-scan block layout (reference src/fast_scan.hpp:6-34)."""
    n, m = codes.shape
    nb = (n + 31) // 32
    out = np.zeros((nb, m, 16), np.uint8)
    for v in range(n):
        b, p = divmod(v, 32)
        if p < 16:
            out[b, :, p] |= codes[v]
        else:
            out[b, :, p - 16] |= codes[v] << 4
    return out


@pytest.mark.parametrize("m", [2, 6, 16, 50, 64, 196, 1024])
def test_fast_scan_sums_bit_exact(L, ref, m):
    rng = np.random.default_rng(200 + m)
    n = 64 * 5 + 17
    codes = rng.integers(0, 16, size=(n, m), dtype=np.uint8)
    nl = 3
    luts = rng.integers(0, 64, size=(nl, m, 16), dtype=np.uint8)
    if m == 1024:
        luts[0] = 63   # the all-63 overflow case
    lut_of = (np.arange((n + 63) // 64) % nl).astype(np.uint32)
    sums = torch.empty(n, dtype=torch.int16, device="cuda")
    tl, tc, to = dev(luts), dev(codes), dev(lut_of)
    L.check(L.lib.qg_fast_scan_dev(tl.data_ptr(), nl, m, tc.data_ptr(), to.data_ptr(), n, sums.data_ptr(), None))
    torch.cuda.synchronize()
    got = sums.cpu().numpy().view(np.uint16)
    blocks = fs_pack(codes)
    for b in range(blocks.shape[0]):
        v0 = b * 32
        lut = luts[lut_of[v0 // 64]].ravel()
        _, expect = ref.fast_scan_block_mask(lut, blocks[b].ravel(), m, 0)
        cnt = min(32, n - v0)
        np.testing.assert_array_equal(got[v0:v0 + cnt], expect[:cnt])


@pytest.mark.parametrize("dim", [1, 7, 8, 16, 31, 32, 33, 100, 128, 200])
@pytest.mark.parametrize("ip", [0, 1])
def test_exact_scores_match_avx2_build(L, ref, dim, ip):
    rng = np.random.default_rng(dim * 3 + ip)
    a = rng.normal(size=(37, dim)).astype(np.float32)
    b = rng.normal(size=(45, dim)).astype(np.float32)
    out = torch.empty((37, 45), dtype=torch.float32, device="cuda")
    ta, tb = dev(a), dev(b)
    L.check(L.lib.qg_exact_scores_dev(ta.data_ptr(), 37, tb.data_ptr(), 45, dim, ip, out.data_ptr(), None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for i in range(37):
        for j in range(45):
            e = -ref.inner_product(a[i], b[j]) if ip else ref.l2_distance(a[i], b[j])
            assert got[i, j].tobytes() == np.float32(e).tobytes(), (i, j, got[i, j], e)
