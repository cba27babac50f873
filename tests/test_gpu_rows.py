"""Lattice-structured kernels for L1 = 32 (one warp per vector, rows through
a register pipeline) against the thread-per-site FP64 kernels of the same
library, which the golden-vector tests pin to the reference.

Shapes cover the row pipeline's wrap-around: L2 = 2 and 3 (every row is
within the pipeline's lag of both ends), 5, and 32 (the 32 x 32 lattice of
the headline workload) at small Nt."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(2, 8, 4.0), (3, 12, 5.0), (5, 16, 8.0), (32, 16, 8.0)]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("l2,nt,beta", SHAPES)
def test_row_pipeline_mixed_force_against_fp64_adjoint(gpu, restated, l2, nt, beta):
    """The FP32 force of the mixed path (row-pipeline kernel at L1 = 32)
    against the FP64 adjoint force on the same configuration: log det equal to
    FP64 rounding, force within 1e-3 (the bound the mixed path meets on the
    thread-per-site kernel)."""
    import ephmc
    from oracle import Model
    m = Model.physical(32, l2, nt, beta)
    x = restated.random_x(7, m.dim)
    with ephmc.Context(32, l2, nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld64, pd64 = ctx.eval(x, mode="adjoint")
        ldm, pdm = ctx.eval(x, mode="mixed")
    assert abs(ldm - ld64) <= 1e-12 * abs(ld64) + 1e-13
    err = rel(pdm, pd64)
    print(f"32x{l2} Nt={nt}: mixed force rel err {err:.2e}")
    assert err <= 1e-3
