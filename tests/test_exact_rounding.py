"""The exact MPR's second normalization (unit_again in
collision-detection_b200/csrc/cc_mpr.cuh) takes sqrt(s) and RN(1/sqrt(s))
from the bits of s when s lies within 2^20 units in the last place of 1. IEEE
754 square root and division are correctly rounded on the CPU as on the GPU,
so the two bit formulas are checked here against numpy for every s in range.
"""
import numpy as np

ONE = np.int64(0x3FF0000000000000)
NEAR = 1 << 20


def _root_bits(e):
    return ONE + (e >> 1)


def _recip_bits(f):
    return np.where(f >= 0, ONE - 2 * f, ONE - (f >> 1))


def test_root_of_near_one_from_bits():
    e = np.arange(-NEAR, NEAR + 1, dtype=np.int64)
    s = (ONE + e).view(np.float64)
    assert np.array_equal(np.sqrt(s).view(np.int64), _root_bits(e))


def test_reciprocal_of_near_one_from_bits():
    e = np.arange(-NEAR, NEAR + 1, dtype=np.int64)
    f = e >> 1
    l = (ONE + f).view(np.float64)
    assert np.array_equal((1.0 / l).view(np.int64), _recip_bits(f))


def test_unit_vector_renormalized_from_bits():
    """The whole second normalization on vectors normalized once: the bit
    formulas plus one quotient each equal v / sqrt(v.v) in IEEE arithmetic."""
    rng = np.random.default_rng(7)
    v = rng.standard_normal((200_000, 3)) * np.exp(rng.uniform(-20, 20, (200_000, 1)))
    u = v / np.sqrt(((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2]))[:, None]
    s = (u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1]) + u[:, 2] * u[:, 2]
    e = s.view(np.int64) - ONE
    assert np.all(np.abs(e) <= NEAR)
    l = _root_bits(e).view(np.float64)
    assert np.array_equal(l, np.sqrt(s))
    assert np.array_equal(_recip_bits(e >> 1).view(np.float64), 1.0 / l)
    assert np.array_equal(u / l[:, None], u / np.sqrt(s)[:, None])
