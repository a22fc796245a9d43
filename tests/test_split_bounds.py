"""CPU check of the error analysis behind the split-precision products (no GPU).

The tensor-core kernels split every FP64 operand value into bf16 parts and sum exact products of
parts with FP32 accumulation:

* two-part split (BF16x3): v = hi + lo, hi = bf16(v), lo = bf16(v - hi); a block pair contributes
  lo.hi + hi.lo + hi.hi, and the whole contraction accumulates in FP32;
* three-part split (BF16x6): v = hi + mid + lo; a block pair contributes hi.lo + lo.hi + mid.mid +
  hi.mid + mid.hi + hi.hi in one FP32 tile (smallest first), and the pairs are summed in FP64.

This emulation rounds to bf16 directly from FP64 (round to nearest even, 8 significant bits), forms
the products of parts exactly, and rounds the running FP32 sum to nearest after every product.  Its
worst errors (about 5.6e-6 and 4.1e-8 of sum |a||b|) are 2-3 times below those measured on the B200
tensor cores (1.1e-5 and 1.2e-7), whose MMA accumulation rounds more coarsely.  The per-element
bounds that the GPU tests assert (2^-14 and 2^-20 of sum |a||b|) hold for both with margin, on
13 x 13 blocks padded to 16.
"""
import numpy as np


def bf16(v):
    """Round to 8 significant bits, ties to even (what __double2bfloat16 does for normal values)."""
    m, e = np.frexp(v)
    return np.ldexp(np.rint(m * 256.0) / 256.0, e)


def split2(v):
    h = bf16(v)
    return h, bf16(v - h)


def split3(v):
    h = bf16(v)
    r = v - h
    m = bf16(r)
    return h, m, bf16(r - m)


def fp32_dot_accumulate(acc, x, y):
    """acc (float32, shape (n, n)) += x @ y with the sum rounded to FP32 after every product."""
    for k in range(x.shape[1]):
        acc = (acc.astype(np.float64) + np.outer(x[:, k], y[k, :])).astype(np.float32)
    return acc


def random_terms(rng, n_terms, nd=13, pad=16):
    """Block pairs of one output block: values uniform[-1, 1] times exp(-r/3) for r in [0, 48]
    bohr (the synthetic inputs' envelope), padded with zeros to 16 x 16."""
    out = []
    for _ in range(n_terms):
        a = np.zeros((pad, pad)); b = np.zeros((pad, pad))
        a[:nd, :nd] = rng.uniform(-1, 1, (nd, nd)) * np.exp(-rng.uniform(0, 48) / 3.0)
        b[:nd, :nd] = rng.uniform(-1, 1, (nd, nd)) * np.exp(-rng.uniform(0, 48) / 3.0)
        out.append((a, b))
    return out


def exact_and_bound(terms):
    ref = sum(a @ b for a, b in terms)
    bound = sum(np.abs(a) @ np.abs(b) for a, b in terms)
    return ref, bound


def test_bf16_rounding_is_round_to_nearest_even_at_8_bits():
    assert bf16(1.0 + 2.0 ** -8) == 1.0                 # tie to even
    assert bf16(1.0 + 3 * 2.0 ** -8) == 1.0 + 2.0 ** -6    # tie to even (up)
    v = np.random.default_rng(0).uniform(-1, 1, 10000)
    # half an ulp of an 8-bit significand in [128, 256) relative to the value: at most 2^-8
    assert np.all(np.abs(bf16(v) - v) <= 2.0 ** -8 * np.abs(v))


def test_three_part_split_keeps_24_bits():
    v = np.random.default_rng(1).uniform(-1, 1, 100000) * 10.0 ** np.random.default_rng(2).uniform(-7, 0, 100000)
    h, m, l = split3(v)
    # each rounding keeps 8 bits of what is left: |v - h - m - l| <= 2^-24 |v|
    assert np.all(np.abs(v - (h + m + l)) <= 2.0 ** -24 * np.abs(v))


def test_two_part_split_product_bound():
    rng = np.random.default_rng(3)
    worst = 0.0
    for _ in range(4):
        terms = random_terms(rng, 24)
        ref, bound = exact_and_bound(terms)
        acc = np.zeros((16, 16), np.float32)
        for a, b in terms:
            ah, al = split2(a)
            bh, bl = split2(b)
            acc = fp32_dot_accumulate(acc, al, bh)
            acc = fp32_dot_accumulate(acc, ah, bl)
            acc = fp32_dot_accumulate(acc, ah, bh)
        err = np.abs(acc.astype(np.float64) - ref)
        worst = max(worst, float(np.max(err / np.maximum(bound, 1e-300))))
    assert worst <= 2.0 ** -14, worst
    assert worst > 2.0 ** -24          # the emulation really rounds


def test_three_part_split_product_bound():
    rng = np.random.default_rng(4)
    worst = 0.0
    for _ in range(4):
        terms = random_terms(rng, 24)
        ref, bound = exact_and_bound(terms)
        acc = np.zeros((16, 16))
        for a, b in terms:
            ah, am, al = split3(a)
            bh, bm, bl = split3(b)
            t = np.zeros((16, 16), np.float32)
            for x, y in ((ah, bl), (al, bh), (am, bm), (ah, bm), (am, bh), (ah, bh)):
                t = fp32_dot_accumulate(t, x, y)
            acc += t.astype(np.float64)
        err = np.abs(acc - ref)
        worst = max(worst, float(np.max(err / np.maximum(bound, 1e-300))))
    assert worst <= 2.0 ** -20, worst
    assert worst > 2.0 ** -40
