"""The precision model of the tensor-core value kernel, on the CPU.

The kernel evaluates a linear predictor sum_c a_c x_c on TF32 tensor cores
(10 explicit mantissa bits) by splitting both operands, v = hi + lo with
hi = TF32 rounding of v (to nearest, ties away: cvt.rna.tf32.f32) and lo =
TF32 rounding of v - hi, and summing a_hi x_lo + a_lo x_hi + a_hi x_hi (the
product of two TF32 values is exact in the FP32 accumulator's precision;
a_lo x_lo is dropped).  This restates that split in numpy and checks the
error bound the kernel's accuracy argument uses: each product within 2^-20
of |a x| (and within 2^-21 on average), where a single TF32 product is off by
up to 2^-11.  No GPU: it checks the arithmetic, the GPU tests check the
kernel against the oracle.
"""
import numpy as np


def tf32_rna(v):
    """Round f32 values to TF32 (10 explicit mantissa bits), to nearest with
    ties away from zero, keeping the f32 container."""
    b = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x1000) & 0xFFFFE000  # add half an ulp of the 13 dropped bits, truncate
    return b.astype(np.uint32).view(np.float32)


def split(v):
    v = np.asarray(v, np.float32)
    hi = tf32_rna(v)
    lo = tf32_rna((v - hi).astype(np.float32))
    return hi, lo


def test_tf32_rounding_keeps_ten_mantissa_bits():
    rng = np.random.default_rng(0)
    v = rng.normal(0, 3, 10000).astype(np.float32)
    h = tf32_rna(v)
    assert np.all((h.view(np.uint32) & 0x1FFF) == 0)
    rel = np.abs(h.astype(np.float64) - v) / np.abs(v)
    assert rel.max() <= 2.0 ** -11 * (1 + 1e-6)


def test_three_product_split_is_near_fp32():
    rng = np.random.default_rng(1)
    a = rng.normal(0, 1, 200000).astype(np.float32)
    x = (rng.normal(0, 1, 200000) * np.exp(rng.normal(0, 2, 200000))).astype(np.float32)
    ah, al = split(a)
    xh, xl = split(x)
    f64 = np.float64
    three = f64(ah) * f64(xl) + f64(al) * f64(xh) + f64(ah) * f64(xh)
    exact = f64(a) * f64(x)
    rel = np.abs(three - exact) / np.abs(exact)
    assert rel.max() <= 2.0 ** -20
    assert rel.mean() <= 2.0 ** -21
    one = f64(ah) * f64(xh)
    assert (np.abs(one - exact) / np.abs(exact)).max() > 2.0 ** -13


def test_split_of_a_dot_product_matches_fp32_accumulation():
    # a 17-term linear predictor: the split products summed in f64 are
    # within a few FP32 roundings of the exact sum, like an FP32 FMA chain
    rng = np.random.default_rng(2)
    A = rng.normal(0, 0.5, (512, 17)).astype(np.float32)
    X = rng.normal(0, 1, (17, 4096)).astype(np.float32)
    X[16] = 1.0  # the ones column of an intercept
    ah, al = split(A)
    xh, xl = split(X)
    f64 = np.float64
    eta = f64(ah) @ f64(xl) + f64(al) @ f64(xh) + f64(ah) @ f64(xh)
    exact = f64(A) @ f64(X)
    scale = np.abs(f64(A)) @ np.abs(f64(X))
    assert (np.abs(eta - exact) / scale).max() <= 2.0 ** -20
    # an FP32 multiply-add chain for comparison
    fma = np.zeros_like(exact, dtype=np.float32)
    for k in range(17):
        fma = (fma.astype(np.float64) + f64(A[:, k:k + 1]) * f64(X[k:k + 1, :])).astype(np.float32)
    assert (np.abs(fma - exact) / scale).max() <= 2.0 ** -20
