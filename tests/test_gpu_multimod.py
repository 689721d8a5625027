"""The multi-modular driver end to end on the GPU: the integer matrix's
GF(p) images reduced by gbgpu_reduce_batch, lifted to Q on the host, equal
to an exact rational elimination (and a rank-deficient prime skipped)."""
from fractions import Fraction

import numpy as np
import pytest

from gb_b200 import multimod
from tests.helpers import exact_answer, small_integer_matrix

pytestmark = pytest.mark.gpu


def test_reduce_over_q_matches_exact_rational_answer():
    mat = small_integer_matrix()
    got = multimod.reduce_over_q(mat)
    assert got.fractions() == exact_answer(mat)
    assert got.primes_used >= 2


def test_reduce_over_q_skips_a_rank_deficient_prime():
    p0 = 2147483647  # the first prime tried; the Schur complement has determinant p0
    mat = multimod.IntegerMacaulay(
        1, 2, np.array([0, 1, 3, 6], dtype=np.int64),
        np.array([0, 0, 1, 0, 1, 2], dtype=np.int32),
        np.array([1, 1, 1, 1, 5, p0], dtype=np.int64))
    got = multimod.reduce_over_q(mat, batch=4)
    assert got.fractions() == [[(2, Fraction(1))], [(1, Fraction(1))]]
