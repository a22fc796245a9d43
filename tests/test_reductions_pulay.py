"""CPU checks of the host-side pieces shared by the chain: Pulay coefficients and exact sums.

The Pulay inverse is restated twice (C++ in the library, Python in the oracle) with the
same operation order as LAPACK's dsytf2/dsytri; both must agree bit for bit and match
scipy's LAPACK to rounding.  The oracle's exact sum must be order independent.
"""
import numpy as np
import pytest

import cq_b200
from lnv_oracle import OracleLNV, bk_inverse


def _sym(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    d = np.geomspace(1.0, cond, n) * rng.choice([-1.0, 1.0], size=n)
    return (Q * d) @ Q.T


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("seed", range(6))
def test_pulay_product_equals_oracle_restatement(n, seed):
    A = _sym(n, seed)
    a_lib = cq_b200.pulay_alphas(2 if n > 1 else 1, A, n, 5)
    a_orc = OracleLNV.do_pulay(2 if n > 1 else 1, A, n, 5)
    assert np.array_equal(a_lib, a_orc)
    a_lap = OracleLNV.do_pulay(2 if n > 1 else 1, A, n, 5, use_lapack=True)
    np.testing.assert_allclose(a_lib, a_lap, rtol=1e-9, atol=1e-12)


def test_bk_inverse_indefinite_and_2x2_pivots():
    # zero diagonal forces 2x2 pivots
    A = [[0.0, 2.0, 1.0], [2.0, 0.0, 3.0], [1.0, 3.0, 0.0]]
    inv = np.array(bk_inverse(A))
    np.testing.assert_allclose(inv @ np.array(A), np.eye(3), atol=1e-14)
    assert bk_inverse([[0.0, 0.0], [0.0, 0.0]]) is None


def test_exact_sum_is_order_independent():
    from cq_oracle import OracleSystem
    import cq_oracle
    lib = cq_oracle._load()
    o = OracleSystem.__new__(OracleSystem)
    o._lib = lib
    rng = np.random.default_rng(0)
    x = rng.normal(size=20000) * np.exp(rng.normal(scale=8, size=20000))
    y = rng.normal(size=20000)
    s = o.exact_dot(x, y)
    for seed in range(3):
        p = np.random.default_rng(seed).permutation(x.size)
        assert o.exact_dot(x[p], y[p]) == s
    import math
    assert abs(s - math.fsum(x * y)) <= 1e-15 * abs(s)
    assert o.exact_dot(np.zeros(5), np.ones(5)) == 0.0
    # exact cancellation inside the 150-bit window, truncation below it (by design)
    assert o.exact_dot(np.array([1e30, -1e30, 3.0])) == 3.0
    assert o.exact_dot(np.array([1e300, -1e300, 3.0])) == 0.0


def test_pulay_nan_matrix_is_singular():
    """A NaN pivot makes the Pulay matrix singular (dsytf2's INFO), as in the oracle: the mixing then
    keeps the newest iterate instead of reading outside the matrix."""
    import math
    import cq_b200
    from lnv_oracle import bk_inverse
    A = np.eye(3)
    A[0, 0] = float("nan")
    al = cq_b200.pulay_alphas(2, A, 3, 5)
    assert al[1] == 1.0 and al[0] == 0.0 and al[2] == 0.0
    assert bk_inverse([list(r) for r in A]) is None
    assert not math.isnan(al.sum())


def test_solve_cubic_library_equals_oracle():
    """The library's SolveCubic (host C++) and the oracle's restatement give the same bits."""
    rs = np.random.default_rng(7)
    for _ in range(2000):
        a, b, c = rs.normal(size=3) * rs.choice([0.1, 1.0, 10.0], 3)
        g = float(rs.choice([1e-3, 1.0, 1e6]))
        assert cq_b200.solve_cubic(a, b, c, g) == OracleLNV.solve_cubic(a, b, c, g)
