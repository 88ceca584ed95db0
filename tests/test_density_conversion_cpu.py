"""The forward plane pass converts the integer deposit a (units of 2^-23
particle weight) to the density contrast as (a - 2^u) 2^-u with one integer
subtraction and one int64 -> float rounding, where the particle mass is
2^(23 - u); k_acc_mesh computes float(a 2^-u - 1.0) in FP64. For every count
below 2^53 the two give the same bits: the FP64 value is exact, and rounding
commutes with the power-of-two scale."""
import numpy as np


def test_integer_and_fp64_conversions_give_the_same_floats():
    rng = np.random.default_rng(0)
    for unit in (23, 20, 14, 11):
        k = 2.0 ** -unit
        a = np.concatenate([rng.integers(0, 2 ** 50, 200_000, dtype=np.int64),
                            rng.integers(2 ** unit - 4096, 2 ** unit + 4096, 50_000, dtype=np.int64),
                            np.array([0, 1, 2 ** unit - 1, 2 ** unit, 2 ** unit + 1, 2 ** 53 - 1], dtype=np.int64)])
        fp64 = (a.astype(np.float64) * k - 1.0).astype(np.float32)
        integer = (a - (1 << unit)).astype(np.float32) * np.float32(k)
        assert np.array_equal(fp64.view(np.int32), integer.view(np.int32)), unit
