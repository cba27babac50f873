"""The register-strip sweep-1 kernel (L1 = 32 lattices, used by the adjoint
and mixed paths) against the reference path of the same library, whose
M_hat is bit-identical to the reference's: the two paths share nothing but
the LU, so agreement of log det and force pins the strip kernel's M_hat and
q stack.  Shapes: the smallest strip layout (32x4), a middle one and the
32x32 lattice of the headline workload, at small Nt and dtau = beta/Nt =
0.25 (the headline workload has 0.31).  At dtau >= 0.5 the Taylor-4 slice
polynomial is far from exp(-dtau H) and M_hat's condition number reaches
1e30: log det then depends on the summation order at the 1e-5 level, for
the reference as for any other order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(4, 8, 2.0), (8, 16, 4.0), (32, 16, 4.0)]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("l2,nt,beta", SHAPES)
def test_strip_sweep_adjoint_matches_reference_path(gpu, restated, l2, nt, beta):
    import ephmc
    from oracle import Model
    m = Model.physical(32, l2, nt, beta)
    x = restated.random_x(5, m.dim)
    with ephmc.Context(32, l2, nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld_r, pd_r = ctx.eval(x, mode="reference")
        ld_a, pd_a = ctx.eval(x, mode="adjoint")
        ld_m, pd_m = ctx.eval(x, mode="mixed")
    assert abs(ld_a - ld_r) <= 1e-12 * abs(ld_r) + 1e-12
    assert abs(ld_m - ld_r) <= 1e-12 * abs(ld_r) + 1e-12
    err_a, err_m = rel(pd_a, pd_r), rel(pd_m, pd_r)
    print(f"32x{l2} Nt={nt}: adjoint {err_a:.2e} mixed {err_m:.2e}")
    # measured: adjoint 2e-15, mixed 7e-7 on all three shapes
    assert err_a <= 1e-12
    assert err_m <= 1e-5


# Register-tile layouts of the same sweep for L1 != 32 (slices_tile.cu): L1 =
# 48 (3 columns per lane, 16 lanes per row), 24 (3 columns, 8 lanes), 16 and
# 12 (one column, 16 lanes; 12 of them hold sites), 8 (one column, 8 lanes).
TILE_SHAPES = [(48, 4, 8, 2.0), (48, 48, 16, 4.0), (24, 8, 8, 2.0), (24, 24, 16, 4.0), (16, 16, 16, 4.0),
               (12, 12, 16, 4.0), (8, 8, 16, 4.0), (8, 24, 8, 2.0)]


@pytest.mark.parametrize("l1,l2,nt,beta", TILE_SHAPES)
def test_tile_sweep_adjoint_matches_reference_path(gpu, restated, l1, l2, nt, beta):
    """Sweep 1, the y chain and the segment stacks of the adjoint and mixed
    paths run the register-tile kernel on these lattices, and for L1 <= 24
    the mixed force's sweep runs the register-tile adjoint (adjoint_tile.cu);
    the reference path keeps the reference's summation order.  Log det to
    1e-12, the FP64 adjoint force to 1e-12 and the mixed force to 1e-5 of the
    reference path's."""
    import ephmc
    from oracle import Model
    m = Model.physical(l1, l2, nt, beta)
    x = restated.random_x(7, m.dim)
    with ephmc.Context(l1, l2, nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld_r, pd_r = ctx.eval(x, mode="reference")
        ld_a, pd_a = ctx.eval(x, mode="adjoint")
        ld_m, pd_m = ctx.eval(x, mode="mixed")
    err_a, err_m = rel(pd_a, pd_r), rel(pd_m, pd_r)
    print(f"{l1}x{l2} Nt={nt}: log det {ld_a - ld_r:.2e}, adjoint {err_a:.2e}, mixed {err_m:.2e}")
    assert abs(ld_a - ld_r) <= 1e-12 * abs(ld_r) + 1e-12
    assert abs(ld_m - ld_r) <= 1e-12 * abs(ld_r) + 1e-12
    assert err_a <= 1e-12
    assert err_m <= 1e-5
