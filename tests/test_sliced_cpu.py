"""The arithmetic of the INT8 slicing used by the sliced trailing update,
restated in numpy: four balanced base-254 digits per element of a row scaled
by max |row| / 127 stay within int8, reconstruct the row to ~2^-32 of its
maximum, and the S32 level sums of ts-long dot products cannot overflow."""
import numpy as np

RADIX, TOP, SLICES = 254.0, 127.0, 4


def slice_rows(P):
    m = np.max(np.abs(P), axis=1, keepdims=True)
    c = np.where(m > 0, TOP / np.where(m > 0, m, 1), 0.0)
    x = P * c
    digits = []
    for _ in range(SLICES):
        d = np.clip(np.rint(x), -TOP, TOP)
        digits.append(d)
        x = (x - d) * RADIX
    return digits, m / TOP


def rebuild(digits, scale):
    v = np.zeros_like(digits[0])
    for d in reversed(digits):
        v = v / RADIX + d
    return v * scale


def test_digits_fit_int8_and_rebuild_the_rows():
    rng = np.random.default_rng(0)
    P = rng.standard_normal((256, 512)) * np.exp(rng.uniform(-20, 20, (256, 1)))
    P[3] = 0.0
    P[7, :] = np.where(np.arange(512) % 2, 1.0, -1.0)  # ties at every digit
    digits, scale = slice_rows(P)
    for d in digits:
        assert np.all(np.abs(d) <= 127) and np.all(d == np.rint(d))
    err = np.abs(rebuild(digits, scale) - P) / np.maximum(np.max(np.abs(P), axis=1, keepdims=True), 1e-300)
    assert err.max() < 0.51 * RADIX ** -3 / TOP + 1e-15  # half a unit of the last digit
    assert np.all(rebuild(digits, scale)[3] == 0)


def test_truncated_level_product_error_and_int32_headroom():
    rng = np.random.default_rng(1)
    ts = 512
    A = rng.standard_normal((64, ts))
    B = rng.standard_normal((64, ts))
    da, sa = slice_rows(A)
    db, sb = slice_rows(B)
    U = np.zeros((64, 64))
    for t in range(SLICES):
        lvl = sum(da[a] @ db[t - a].T for a in range(t + 1))
        assert np.abs(lvl).max() < 2 ** 31
        U += lvl * RADIX ** -t
    U *= sa * sb.T
    exact = A @ B.T
    bound = np.abs(A).max(axis=1, keepdims=True) * np.abs(B).max(axis=1, keepdims=True).T * ts
    assert np.max(np.abs(U - exact) / bound) < 4 * RADIX ** -3 / TOP
    # worst case of a level sum: 4 digit pairs of 127 x 127 per k, ts terms
    assert 4 * 127 * 127 * 16384 < 2 ** 31
