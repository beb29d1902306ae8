"""Pins the oracle (this project's C restatement, oracle/qann_oracle.c) to the
reference: the reference's own known-answer tests (reference
tests/test_fast_scan.cpp, tests/test_distance.cpp), its golden files, and the
reference library built from its sources (oracle/_ref) on seeded inputs.
CPU only."""
import numpy as np
import pytest

from oracle import oracle as orc
from oracle import qann_file


# ---- known answers from the reference's own tests ------------------------------------

def test_block_layout_known_bytes():
    # reference tests/test_fast_scan.cpp:35-44
    codes = np.zeros((32, 2), np.uint8)
    codes[0, 0], codes[16, 0], codes[5, 1], codes[31, 1] = 0x3, 0xA, 0x7, 0x1
    blk = np.zeros((2, 16), np.uint8)
    for v in range(32):
        for s in range(2):
            if v < 16:
                blk[s, v] |= codes[v, s]
            else:
                blk[s, v - 16] |= codes[v, s] << 4
    assert blk[0, 0] == 0xA3 and blk[1, 5] == 0x07 and blk[1, 15] == 0x10


def test_block_sum_known_answer():
    # reference tests/test_fast_scan.cpp:46-61: entry = s * 16 + j, code (v + s) % 16
    m = 4
    lut = np.arange(m * 16, dtype=np.uint8)
    blk = np.zeros((m, 16), np.uint8)
    for v in range(32):
        for s in range(m):
            c = (v + s) % 16
            blk[s, v % 16] |= c if v < 16 else c << 4
    _, out = orc.fast_scan_block_mask(lut, blk, m, 0)
    for v in range(32):
        assert out[v] == sum(s * 16 + (v + s) % 16 for s in range(m))


def test_quantize_constant_rows():
    # reference tests/test_fast_scan.cpp:115-124
    lut, scale, offset = orc.quantize_lut(np.full(4 * 16, 3.0, np.float32))
    assert scale == 1.0 and offset == 12.0 and not lut.any()


def test_quantize_negative_rows():
    # reference tests/test_fast_scan.cpp:126-144
    t = np.empty(32, np.float32)
    t[:16] = -500.0 + 10.0 * np.arange(16)
    t[16:] = -40.0 - 2.0 * np.arange(16)
    lut, scale, offset = orc.quantize_lut(t)
    assert scale == np.float32(63) / np.float32(150) and offset == -570.0
    assert lut[0] == 0 and lut[15] == 63 and lut[31] == 0
    assert lut[16] == np.rint(np.float32(30.0) * scale)


def test_quantize_rounds_half_to_even():
    # reference tests/test_fast_scan.cpp:397-414
    t = np.zeros(32, np.float32)
    t[1] = 63
    probes = [0.5, 1.5, 2.5, 62.5, np.nextafter(np.float32(0.5), np.float32(0)),
              np.nextafter(np.float32(0.5), np.float32(1)), np.nextafter(np.float32(1.5), np.float32(0)), 0.25, 3.0]
    t[17:26] = np.array(probes, np.float32)
    lut, scale, _ = orc.quantize_lut(t)
    assert scale == 1.0
    assert list(lut[17:26]) == [0, 2, 2, 62, 0, 1, 1, 0, 3]


@pytest.mark.parametrize("m,sd", [(4, 4), (50, 2), (64, 2)])
def test_coarse_plus_list_term_plus_inner_table_is_the_residual_adc(m, sd):
    # reference tests/test_distance.cpp:702-723: per subspace, A (the query-centroid
    # distance) + B (list term) + C (inner table) equals the ADC table of q - c
    # within 1e-3 (numpy-drawn codebook, query and centroid here)
    rng = np.random.default_rng(700 + m)
    yt = rng.normal(size=(m, sd, 16)).astype(np.float32)
    q, c = rng.normal(size=(2, m * sd)).astype(np.float32)
    adc = orc.adc_table(q - c, yt, m, sd).reshape(m, 16)
    inner = orc.inner_table(q, yt, m, sd).reshape(m, 16)
    lt = orc.list_term(c, yt, m, sd).reshape(m, 16)
    for s in range(m):
        a = orc.l2(q[s * sd:(s + 1) * sd], c[s * sd:(s + 1) * sd])
        np.testing.assert_allclose(a + lt[s] + inner[s], adc[s], rtol=0, atol=1e-3)


@pytest.mark.parametrize("m", [2, 6, 16, 64, 196, 256, 480, 1024])
def test_mask_at_limits(m):
    # reference tests/test_fast_scan.cpp:416-439 (inputs drawn by numpy here)
    rng = np.random.default_rng(m + 200)
    lut = rng.integers(0, 64, size=m * 16, dtype=np.uint8)
    blk = rng.integers(0, 256, size=m * 16, dtype=np.uint8)
    _, ref_sums = orc.fast_scan_block_mask(lut, blk, m, 0)
    srt = np.sort(ref_sums)
    for limit in (0, 65535, int(srt[0]), int(srt[10]), int(srt[31]), int(srt[20]) + 1):
        mask, sums = orc.fast_scan_block_mask(lut, blk, m, limit)
        np.testing.assert_array_equal(sums, ref_sums)
        for v in range(32):
            assert ((mask >> v) & 1) == (1 if ref_sums[v] < limit else 0)


# ---- the restatement against the reference library -------------------------------------

@pytest.mark.parametrize("dim", list(range(1, 70)) + [96, 100, 128, 200, 768])
def test_distances_bit_exact(ref, dim):
    rng = np.random.default_rng(dim)
    for _ in range(10):
        a, b = rng.normal(size=(2, dim)).astype(np.float32)
        assert orc.l2(a, b).tobytes() == ref.l2_distance(a, b).tobytes()
        assert orc.ip(a, b).tobytes() == ref.inner_product(a, b).tobytes()


@pytest.mark.parametrize("m,sd", [(16, 2), (50, 2), (64, 2), (8, 4), (32, 3)])
def test_pq_tables_and_encoder_bit_exact(ref, m, sd):
    rng = np.random.default_rng(m * 10 + sd)
    cen = rng.normal(size=(m, 16, sd)).astype(np.float32)
    yt = np.ascontiguousarray(cen.transpose(0, 2, 1))
    for _ in range(10):
        q, c = rng.normal(size=(2, m * sd)).astype(np.float32)
        inner, lt, adc = ref.pq_tables(cen, m, 16, q=q, coarse=c, adc=True)
        assert orc.inner_table(q, yt, m, sd).tobytes() == inner.tobytes()
        assert orc.list_term(c, yt, m, sd).tobytes() == lt.tobytes()
        assert orc.adc_table(q, yt, m, sd).tobytes() == adc.tobytes()
        x = rng.normal(size=(8, m * sd)).astype(np.float32)
        codes = ref.pq_encode(cen, m, 16, x)
        for i in range(8):
            np.testing.assert_array_equal(orc.encode16(x[i], yt, m, sd), codes[i])


@pytest.mark.parametrize("m", [2, 6, 16, 50, 64, 196, 1024])
def test_lut_rounding_bit_exact(ref, m):
    rng = np.random.default_rng(m)
    for _ in range(10):
        t = (rng.normal(size=m * 16) * rng.uniform(0.01, 100)).astype(np.float32)
        a, b = orc.quantize_lut(t), ref.quantize_lut(t)
        np.testing.assert_array_equal(a[0], b[0])
        assert a[1].tobytes() == b[1].tobytes() and a[2].tobytes() == b[2].tobytes()
        B, Cq = rng.normal(size=(2, m * 16)).astype(np.float32)
        A = float(rng.uniform(0, 3))
        for x, y in zip(orc.build_quantize_lut(B, Cq, A), ref.build_quantize_lut(B, Cq, A)):
            assert np.asarray(x).tobytes() == np.asarray(y).tobytes()


def test_topk_first_pushed_tie_rule(ref):
    # reference tests/test_distance.cpp:291-317, with numpy-drawn levels
    rng = np.random.default_rng(3)
    for k in (1, 10, 100):
        d = (0.5 * rng.integers(-4, 5, size=2000)).astype(np.float32)
        ids = np.arange(2000, dtype=np.uint64)
        got_ids, got_d = ref.topk_run(d, ids, k)
        order = np.argsort(d, kind="stable")[:k]
        exp = sorted(zip(d[order], order))
        assert [int(i) for i in got_ids] == [int(i) for _, i in exp]


# ---- whole fast-scan queries of the restatement vs the reference ---------------------------

GEN = ["l2", "l2_adc", "ip", "cos_ip", "cos_l2", "l2_custom_del"]


def _normalize(q):
    return np.stack([orc.normalize_row(r) for r in q])


def _finalize(d, s, labels, k, cosine):
    lab = s.astype(np.int64) if labels is None or labels.size == 0 else labels[s]
    keys = np.array([orc.np.frombuffer(x.tobytes(), np.uint32)[0] for x in d], np.uint32) if d.size else d
    # order by (distance, id) as take_sorted does
    order = sorted(range(len(d)), key=lambda i: (float(d[i]), int(lab[i])))[:k]
    ids = np.full(k, -1, np.int64)
    dist = np.full(k, np.inf, np.float32)
    for j, i in enumerate(order):
        ids[j] = lab[i]
        dist[j] = d[i] * np.float32(0.5) if cosine else d[i]
    return ids, dist


@pytest.mark.parametrize("name", GEN)
def test_oracle_ivf_queries_match_reference(golden, name):
    info = qann_file.read(golden / "gen" / f"ivf_{name}.qann")
    ivf = info["ivf"]
    arr = qann_file.arrays(ivf)
    q = np.load(golden / "gen" / "queries.npy")
    if ivf["metric"] == 1:
        q = _normalize(q)
    exp_ids = np.load(golden / "gen" / f"ivf_{name}_ids.npy")
    exp_d = np.load(golden / "gen" / f"ivf_{name}_dists.npy")
    labels = ivf["idmap"]["labels"]
    differ = 0
    for i in range(q.shape[0]):
        probes, pterm = qann_file.coarse(ivf, q[i], ivf["nprobe"])
        d0, s0 = arr.query(q[i], probes, pterm, 10, semantics=0)
        d1, s1 = arr.query(q[i], probes, pterm, 10, semantics=1)
        differ += not (np.array_equal(s0, s1) and d0.tobytes() == d1.tobytes())
        ids, dist = _finalize(d0, s0, labels, 10, ivf["metric"] == 1)
        np.testing.assert_array_equal(ids, exp_ids[i])
        assert dist.tobytes() == exp_d[i].tobytes()
    # the limit16 pre-filter may only matter at float-rounding edges
    assert differ <= 1
