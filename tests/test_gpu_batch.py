"""ephmc_batch_eval: independent chains of uneven lattice, Nt, beta and
coupling evaluated together (the batched-chains configuration), against
ephmc_eval of each chain alone and against the reference for two of them.
The log det is the same computation in both (bit-identical).  The force
differs only by the order of its cross-CTA atomic sums, which also varies
between two single-chain evaluations: each chain's force is bounded by 100
times that run-to-run spread, or 1e-10 if larger."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (L1, L2, Nt, beta, lambda scale, flags)
CHAINS = [(8, 8, 16, 5.0, 1.0, None), (12, 12, 32, 10.0, 0.7, None), (16, 16, 64, 20.0, 1.3, None),
          (24, 24, 32, 12.0, 0.5, None), (32, 32, 64, 20.0, 1.0, None), (8, 12, 16, 6.0, 1.5, None),
          (16, 8, 32, 8.0, 1.0, (0, 0, 0, 1, 0, 0, 0)), (12, 12, 16, 5.0, 1.0, (0, 0, 0, 0, 1, 0, 0))]


def _models():
    from oracle import Model
    out = []
    for l1, l2, nt, beta, s, flags in CHAINS:
        out.append(Model.physical(l1, l2, nt, beta, lam=tuple(s * v for v in (0.3, 0.15, 0.15)),
                                  flags=flags or (0,) * 7))
    return out


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("mode", ["reference", "adjoint", "mixed"])
def test_batch_equals_single_chain_evaluations(gpu, restated, mode):
    import ephmc
    models = _models()
    xs = [restated.random_x(10 + i, m.dim) for i, m in enumerate(models)]
    ctxs = [ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, flags=m.flags) for m in models]
    try:
        single = [c.eval(x, mode=mode) for c, x in zip(ctxs, xs)]
        spread = [_rel(c.eval(x, mode=mode)[1], s[1]) for c, x, s in zip(ctxs, xs, single)]
        lds, pds = ephmc.batch_eval(ctxs, xs, mode=mode)
        for i, ((ld0, pd0), ld, pd) in enumerate(zip(single, lds, pds)):
            assert ld == ld0, (i, ld, ld0)
            err = _rel(pd, pd0)
            print(f"chain {i} {mode}: force {err:.1e} (run-to-run {spread[i]:.1e})")
            assert err <= max(1e-10, 100 * spread[i]), (i, err, spread[i])
        # twice more: state left by a batch does not leak into the next one
        lds2, pds2 = ephmc.batch_eval(ctxs, xs, mode=mode)
        assert np.array_equal(lds2, lds)
    finally:
        for c in ctxs:
            c.close()


def test_batch_against_reference(gpu, reference, restated):
    """Two chains of the batch against the reference compiled unmodified:
    log det to 1e-12, FP64 adjoint force to 1e-10."""
    import ephmc
    models = _models()[:2]
    xs = [restated.random_x(30 + i, m.dim) for i, m in enumerate(models)]
    ctxs = [ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) for m in models]
    try:
        lds, pds = ephmc.batch_eval(ctxs, xs, mode="adjoint")
    finally:
        for c in ctxs:
            c.close()
    reference.set_threads(1)
    for m, x, ld, pd in zip(models, xs, lds, pds):
        rc = reference.context(m)
        ld_r, pd_r = rc.eval(x)
        rc.close()
        assert abs(ld - ld_r) <= 1e-12 * abs(ld_r)
        assert _rel(pd, pd_r) <= 1e-10


def test_batch_rejects_duplicate_contexts(gpu, restated):
    import ephmc
    from oracle import Model
    m = Model.physical(8, 8, 16, 5.0)
    x = restated.random_x(1, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as c:
        with pytest.raises(ephmc.EphmcError) as e:
            ephmc.batch_eval([c, c], [x, x])
    assert e.value.status == 2 and "twice" in str(e.value)
