"""ephmc_ctx_autotune: launch shapes chosen by timing.  The shapes only
change how threads and CTAs share the work: the sweeps keep their summation
order, the LU its pivots; the LU's log det sums per-row terms grouped by
the CTA size, so a new LU shape can move it in the last bit (bounded here by
1e-14 relative).  The FP64 force differs at most by the order of its atomic
sums (bounded by 1e-10 of the largest entry).  The mixed force sums a CTA's
vectors in FP32 before its FP64 atomic, so a new vectors-per-CTA count
regroups FP32 sums (measured 2.5e-7; bounded by 1e-5)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,mode", [((12, 12, 16), "reference"), ((12, 12, 16), "adjoint"),
                                        ((12, 12, 16), "mixed"), ((32, 32, 16), "mixed")])
def test_autotuned_shapes_keep_the_results(gpu, restated, shape, mode):
    import ephmc
    from oracle import Model
    l1, l2, nt = shape
    m = Model.physical(l1, l2, nt, 5.0)
    x = restated.random_x(8, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld0, pd0 = ctx.eval(x, mode=mode)
        before, after, shapes = ctx.autotune(x, mode)
        ld1, pd1 = ctx.eval(x, mode=mode)
    print(f"{shape} {mode}: {before:.3f} -> {after:.3f} ms, shapes {shapes}")
    assert abs(ld1 - ld0) <= 1e-14 * abs(ld0)
    assert np.max(np.abs(pd1 - pd0)) <= (1e-5 if mode == "mixed" else 1e-10) * np.max(np.abs(pd0))
    # 0 keeps the rule's shape; the tuner only replaces it by a faster one
    assert all(v >= 0 for v in shapes)
    assert after <= 1.25 * before
    if l1 == 32:  # the strip kernels have fixed shapes: only the LU is tuned
        assert shapes[:4] == [0, 0, 0, 0]
