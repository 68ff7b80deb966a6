"""The arithmetic of the Cholesky-route split products (csrc/tc_gemm.cu) restated in numpy,
without a GPU: per-row power-of-two scaling to |x| <= 1/2, eight signed 7-bit slices
a_i = rint(r_i 2^7) of the successive remainders, exact integer sums of the slice products
grouped by s = i + j, and the FP64 rebuild sum_s 2^(e_row + e_col - 7 (s + 2)) C_s.  The rebuilt
product must agree with the FP64 product to FP64 rounding (the dropped slice pairs i + j >= 8
weigh 2^-56 relative), and every slice must fit a signed byte.  The BF16 three-piece split
(hi, mid, lo) must represent each entry to 2^-24 relative."""
import numpy as np


def _row_exponents(f):
    mx = np.max(np.abs(f), axis=0)
    _, ex = np.frexp(mx)
    return np.where(mx > 0, ex + 1, 0)


def _slices(f, e, nslice=8):
    x = np.ldexp(f, -e[None, :])
    out = []
    for _ in range(nslice):
        y = x * 128.0
        a = np.rint(y)
        out.append(a.astype(np.int64))
        x = y - a
    return out


def test_int8_slices_rebuild_fp64_product():
    rng = np.random.default_rng(3)
    k, m, n = 96, 40, 30
    u = rng.standard_normal((k, m)) * np.exp(rng.uniform(-8, 8, m))[None, :]
    v = rng.standard_normal((k, n)) * np.exp(rng.uniform(-8, 8, n))[None, :]
    eu, ev = _row_exponents(u), _row_exponents(v)
    su, sv = _slices(u, eu), _slices(v, ev)
    for a in su + sv:
        assert a.min() >= -128 and a.max() <= 127
    t = np.zeros((m, n))
    for s in range(8):
        cs = sum(su[i].T @ sv[s - i] for i in range(s + 1))   # exact in int64 (int32 on the GPU)
        assert np.abs(cs).max() < 2 ** 31
        t += np.ldexp(cs.astype(np.float64), -7 * (s + 2))
    t = np.ldexp(t, eu[:, None] + ev[None, :])
    ref = u.T @ v
    bound = np.abs(u).T @ np.abs(v)
    assert np.all(np.abs(t - ref) <= 1e-14 * bound)


def test_bf16_three_pieces_represent_entries():
    rng = np.random.default_rng(4)
    x = rng.standard_normal(10000) * np.exp(rng.uniform(-20, 20, 10000))

    def to_bf16(y):  # round to nearest even on the upper 16 bits of the FP32 value
        f = y.astype(np.float32).view(np.uint32)
        f = (f + 0x7FFF + ((f >> 16) & 1)) & 0xFFFF0000
        return f.view(np.float32).astype(np.float64)

    r = x.copy()
    acc = np.zeros_like(x)
    for _ in range(3):
        h = to_bf16(r)
        acc += h
        r = r - h
    assert np.all(np.abs(acc - x) <= 2.0 ** -23 * np.abs(x))
