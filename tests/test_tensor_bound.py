"""The error bound behind the tensor-core filter, checked on the CPU for its
input-rounding part: scores from bf16-rounded inputs (accumulated exactly
here) stay within the stated bound of the exact float32 scores the oracle
computes, with room to spare for the accumulation term the GPU adds."""
import numpy as np
import pytest

from oracle import oracle


def bf16(x):
    """Round float32 to bfloat16 (nearest, ties to even), back as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def bound_c(d):
    return 2.0 ** -7 + 2.0 ** -14 + d * 2.0 ** -19


@pytest.mark.parametrize("d", [16, 96, 100, 128])
@pytest.mark.parametrize("ip", [False, True])
def test_bf16_scores_within_bound(d, ip):
    rng = np.random.default_rng(d + ip)
    q = (rng.normal(size=(40, d)) * np.exp(rng.normal(0, 0.25, (40, 1)))).astype(np.float32)
    x = (rng.normal(size=(300, d)) * np.exp(rng.normal(0, 0.25, (300, 1)))).astype(np.float32)
    dot = bf16(q).astype(np.float64) @ bf16(x).astype(np.float64).T
    q2 = (q.astype(np.float64) ** 2).sum(1)[:, None]
    x2 = (x.astype(np.float64) ** 2).sum(1)[None, :]
    exact = np.array([[oracle.ip(a, b) if ip else oracle.l2(a, b) for b in x] for a in q], np.float64)
    est = -dot if ip else q2 + x2 - 2 * dot
    e = (bound_c(d) / (2 if ip else 1)) * (q2 + x2)
    err = np.abs(est - (-exact if ip else exact))
    assert (err <= e).all()
    assert err.max() < 0.9 * e.max()
