"""The 24-bit fixed-point digit arithmetic of the tensor-core reciprocal
space (mdff_b200/csrc/umma.cuh: digits24, QS; ewald_tc.cuh: level sums),
restated in integer numpy: every scaled value V = rn(v * QS), |v| <= 1, is
exactly d1 2^16 + d2 2^8 + d3 with int8 digits taken from the bytes of
(V + 0x808080) ^ 0x808080; the integer dot products of the digit slices,
grouped by digit weight, rebuild the exact integer dot product, and the six
products kept by the kernels miss it by the bounded low-weight terms only."""
import numpy as np

QS = 8355000


def digits(V):
    w = ((V.astype(np.int64) + 0x808080) & 0xFFFFFF) ^ 0x808080
    b = [((w >> s) & 0xFF).astype(np.int64) for s in (16, 8, 0)]
    return [np.where(x > 127, x - 256, x) for x in b]


def test_digit_decomposition_is_exact_and_in_range():
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.uniform(-1, 1, 200000), [-1.0, 1.0, 0.0, 1e-9, -1e-9]])
    V = np.rint(v * QS).astype(np.int64)
    d1, d2, d3 = digits(V)
    assert np.array_equal(d1 * 65536 + d2 * 256 + d3, V)
    assert d1.min() >= -127 and d1.max() <= 127
    assert d2.min() >= -128 and d2.max() <= 127 and d3.min() >= -128 and d3.max() <= 127
    # the whole range the kernels allow
    edge = np.array([-0x7F7F7F, 0x7F7F7F, -QS, QS], np.int64)
    e1, e2, e3 = digits(edge)
    assert np.array_equal(e1 * 65536 + e2 * 256 + e3, edge) and np.abs(e1).max() <= 127


def test_level_sums_rebuild_the_dot_product():
    rng = np.random.default_rng(1)
    K = 4 * 1800   # the largest K one structure-factor CTA accumulates
    a = np.rint(rng.uniform(-1, 1, K) * QS).astype(np.int64)
    b = np.rint(rng.uniform(-1, 1, K) * QS).astype(np.int64)
    da, db = digits(a), digits(b)
    exact = int(np.dot(a, b))
    lv = [0] * 5
    for i in range(3):
        for j in range(3):
            s = int(np.dot(da[i], db[j]))
            assert abs(s) < 2 ** 31 // 3      # three products share an S32 accumulator
            lv[i + j] += s
    assert sum(lv[L] << (8 * (4 - L)) for L in range(5)) == exact
    kept = (lv[0] << 32) + (lv[1] << 24) + (lv[2] << 16)
    # dropped: weights 2^8 and 1, at most 2 * 128 * 128 * 2^8 + 128^2 per term
    assert abs(kept - exact) <= K * (2 * 128 * 128 * 256 + 128 * 128)
    # relative to the scale of one term (QS^2) the dropped part is ~2^-23 per term or less
    assert abs(kept - exact) / (K * float(QS) ** 2) < 2.0 ** -23
