"""The split-int8 numerics on the CPU (no GPU): a numpy restatement of the
digit extraction and recombination that csrc/rho1_split_i8.cu performs, checked
for the properties the kernels rely on.

* digit_scale: the row scale 2^e keeps |x| < 0.9921875 2^e, so the top digit
  of X = rint(x 2^(39 - e)) is a signed byte (|a0| <= 127);
* digits16: the bit-pattern trick (fma with 1.5 2^52, + 0x80808080) and the
  byte permutes give five signed-byte planes whose weighted sum is X exactly,
  and the 16-byte plane words hold element 4q + i in byte i of word q;
* the six level sums (s + u = 0..5) stay inside int32 for K up to 26,000, and
  the recombination 256 S = (L0 256 + L1) 2^32 + (L2 256 + L3) 2^16 +
  (L4 256 + L5) with the scales 2^(eA - 23), 2^(eB - 31) reproduces the FP64
  dot product to ~1e-13 of |a||b| (levels 0..4 alone: ~3.5x worse).
"""
import math

import numpy as np
import pytest

FMA_BIAS = 0x4338000000000000  # bit pattern of 1.5 * 2^52


def byte_perm(x, y, sel):
    b = [(x >> (8 * i)) & 0xFF for i in range(4)] + [(y >> (8 * i)) & 0xFF for i in range(4)]
    return sum(b[(sel >> (4 * n)) & 7] << (8 * n) for n in range(4))


def digit_scale(m):
    e = 0
    if m > 0:
        f, e = math.frexp(m)
        if f >= 0.9921875:
            e += 1
    e = max(e, -960)
    return math.ldexp(1.0, 39 - e), math.ldexp(1.0, e - 23), e


def digits16(x, sc39):
    """Five 4-word planes of 16 values, as the kernel's digits16 builds them."""
    hi, lo = [], []
    for v in x:
        # fma(v, sc39, 1.5 2^52): v * sc39 rounded to an integer (|X| < 2^40)
        X = int(np.rint(np.longdouble(v) * np.longdouble(sc39)))
        xp = (FMA_BIAS + X) + (0x80808080 - FMA_BIAS)
        hi.append((xp >> 32) & 0xFFFFFFFF)
        lo.append(xp & 0xFFFFFFFF)
    planes = [[byte_perm(byte_perm(hi[4 * q], hi[4 * q + 1], 0x40), byte_perm(hi[4 * q + 2], hi[4 * q + 3], 0x40),
                         0x5410) for q in range(4)]]
    for s in range(1, 5):
        b = 4 - s
        sel = b | ((b + 4) << 4)
        planes.append([byte_perm(byte_perm(lo[4 * q], lo[4 * q + 1], sel), byte_perm(lo[4 * q + 2], lo[4 * q + 3], sel),
                                 0x5410) ^ 0x80808080 for q in range(4)])
    return planes


def signed_bytes(planes):
    d = np.zeros((5, 16), dtype=np.int64)
    for s in range(5):
        for q in range(4):
            for i in range(4):
                v = (planes[s][q] >> (8 * i)) & 0xFF
                d[s, 4 * q + i] = v - 256 if v >= 128 else v
    return d


def row_digits(x):
    sc39, s23, e = digit_scale(float(np.max(np.abs(x))))
    n = (len(x) + 15) // 16 * 16
    xp = np.zeros(n)
    xp[: len(x)] = x
    d = np.concatenate([signed_bytes(digits16(xp[i:i + 16], sc39)) for i in range(0, n, 16)], axis=1)
    return d, sc39, s23


def test_scale_keeps_top_digit_a_signed_byte():
    for m in (1.0, 0.9921875, 0.99, 0.5, 3e-300, 7.5e3):
        sc39, _, e = digit_scale(m)
        assert m * sc39 < 0.9921875 * 2.0 ** 39 + 1
        X = int(np.rint(np.longdouble(m) * np.longdouble(sc39)))
        assert -128 <= (X + 0x80808080) >> 32 <= 127
    assert digit_scale(0.0)[2] == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_digit_planes_reconstruct_the_rounded_row(seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(40) * 10.0 ** rng.uniform(-6, 6)
    x[rng.integers(0, 40)] = np.abs(x).max() * 0.99999  # an element at the scale's edge
    d, sc39, _ = row_digits(x)
    assert np.abs(d[0]).max() <= 127 and np.abs(d[1:]).max() <= 128
    X = sum(d[s] * 2 ** (8 * (4 - s)) for s in range(5))
    ref = np.rint(np.longdouble(np.concatenate([x, np.zeros(d.shape[1] - 40)])) * np.longdouble(sc39))
    assert np.array_equal(X, ref.astype(np.int64))


def _levels(da, db, n_levels):
    return [sum(int(np.dot(da[s], db[u])) for s in range(5) for u in range(5) if s + u == L) for L in range(n_levels)]


def _recombine6(L, sA, sB):
    hi = L[0] * 256 + L[1]
    mid = L[2] * 256 + L[3]
    lo = L[4] * 256 + L[5]
    return (float(hi) * 4294967296.0 + (float(mid) * 65536.0 + float(lo))) * sB * 0.00390625 * sA


@pytest.mark.parametrize("K", [1, 33, 350, 800, 2048])
def test_six_levels_reproduce_the_dot_product(K):
    rng = np.random.default_rng(K)
    errs6, errs5 = [], []
    for _ in range(6):
        a, b = rng.standard_normal(K), rng.standard_normal(K) * 1e-3
        da, _, sA = row_digits(a)
        db, _, sB = row_digits(b)
        L = _levels(da, db, 6)
        assert all(abs(v) < 2 ** 31 for v in L)
        ref = float(np.dot(np.longdouble(a), np.longdouble(b)))
        scale = np.linalg.norm(a) * np.linalg.norm(b)
        errs6.append(abs(_recombine6(L, sA, sB) - ref) / scale)
        errs5.append(abs(_recombine6(L[:5] + [0], sA, sB) - ref) / scale)
    assert max(errs6) < 2e-12
    if K >= 350:
        assert np.sqrt(np.mean(np.square(errs5))) > 2 * np.sqrt(np.mean(np.square(errs6)))


def test_level_bound_at_the_largest_k():
    """Five products of |a_s b_u| <= 2^14 per level and step: int32 holds K < 26,214."""
    assert 5 * 2 ** 14 * 26_000 < 2 ** 31
    assert 5 * 2 ** 14 * 2048 < 2 ** 31
