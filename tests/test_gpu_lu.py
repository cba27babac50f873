"""The dataflow LU (log det and inverse of logDetM_and_inv_M_hat,
simulation/organic_dense_matrix.c:580-595) on its failure path and at the
edges of its pivot reciprocal.

* Wait time-out: the test hook ephmc_test_lu_withhold_next keeps one panel's
  owner from setting its ready flag.  Every CTA that waits for that panel
  gives up after its bounded wait (2 s), the call returns EPHMC_ERR_TIMEOUT
  instead of hanging, and the next LU on the same context is correct.  No
  kernel is stopped or faulted: the wait simply runs out.
* Reciprocal: the pivot row is scaled by 1/d from two Newton-Raphson steps on
  the hardware approximation; subnormal pivots and pivots whose reciprocal is
  subnormal take the IEEE quotient.  On diagonal matrices the inverse's
  diagonal is that reciprocal, compared with numpy's 1/d to one unit in the
  last place, for random pivots over 600 decades and the extreme cases."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ctx(V):
    import ephmc
    l1 = int(round(V ** 0.5))
    return ephmc.Context(l1, V // l1, 1, [0.1, 0.1, 0.1], [0.0, 0.0, 0.0], -1.0, 0.1)


@pytest.mark.parametrize("V", [256, 1600])
def test_lu_wait_timeout_reports_and_recovers(gpu, V):
    """V = 256: one panel per CTA; V = 1600: two panels per CTA (the second
    in shared memory), the kernel of 1024 < V <= 2304."""
    import scipy.linalg as sl

    import ephmc
    lib = ephmc.load_library()
    lib.ephmc_test_lu_withhold_next.restype = None
    lib.ephmc_test_lu_withhold_next.argtypes = [C.c_int]
    rng = np.random.default_rng(5)
    with _ctx(V) as ctx:
        A = rng.standard_normal((V, V)) + 3 * np.eye(V)
        lib.ephmc_test_lu_withhold_next(3)
        with pytest.raises(ephmc.EphmcError) as e:
            ctx.logdet_inverse(A.copy())
        assert e.value.status == 8, e.value
        for _ in range(2):
            B = rng.standard_normal((V, V)) + 3 * np.eye(V)
            inv = B.copy()
            ld, sg, ipiv = ctx.logdet_inverse(inv)
            lu, piv = sl.lu_factor(B.T)  # the LU sees the array column-major
            assert np.array_equal(ipiv - 1, piv)
            s_np, ld_np = np.linalg.slogdet(B)
            assert abs(ld - ld_np) <= 1e-12 * abs(ld_np) and sg == int(s_np)
            assert np.max(np.abs(inv - np.linalg.inv(B))) <= 1e-10 * np.max(np.abs(np.linalg.inv(B)))


def test_lu_pivot_reciprocal_over_the_double_range(gpu):
    rng = np.random.default_rng(9)
    V = 256
    d = rng.standard_normal(V) * 10.0 ** rng.uniform(-300, 300, V)
    special = [1e-308, -1e-308, 2.3e-308, 1.5e308, -1.5e308, 1e307, 3.0, -7.0, 2.0 ** -1021, 2.0 ** 1021]
    d[:len(special)] = special
    with _ctx(V) as ctx:
        A = np.diag(d)
        inv = A.copy()
        ld, sg, _ = ctx.logdet_inverse(inv)
    got = np.diag(inv)
    want = 1.0 / d
    ulp = np.abs(got - want) / np.spacing(np.abs(want))
    print(f"reciprocal of {V} pivots: max {ulp.max():.2f} ulp, exact in {int(np.sum(got == want))}")
    assert np.all(ulp <= 1.0), d[ulp > 1.0]
    assert np.count_nonzero(inv - np.diag(got)) == 0
    assert abs(ld - np.sum(np.log(np.abs(d)))) <= 1e-13 * np.sum(np.abs(np.log(np.abs(d))))
    assert sg == int(np.prod(np.sign(d)))
