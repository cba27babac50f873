"""Checkpointed adjoint sweeps (ephmc_ctx_set_checkpoint): sweep 1 keeps the
FP64 propagator states only every C slices and sweep 2 recomputes each
segment from its checkpoint.  Recomputation repeats the same FP64
arithmetic, so the log det is bit-identical to the whole-stack evaluation
and the force differs only by the order of its FP64 atomic sums across CTAs,
which also varies from run to run: the tests bound the difference by 100
times the whole-stack path's own run-to-run spread (measured 4e-12 at
32x32) or 1e-10, whichever is larger.
Covered: the strip kernels (L1 = 32) and the generic kernels (12x12), Nt not
a multiple of C, C = 1 (every state checkpointed), C >= Nt (one segment), and
the 48x48 Nt = 128 configuration with C = 12 (its checkpoint interval), whose
context then holds under 1.2 GB instead of the 5.4 GB stack."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("shape", [(32, 32, 64, 20.0), (12, 12, 37, 10.0)])
@pytest.mark.parametrize("mode", ["adjoint"])
def test_checkpointed_force_equals_whole_stack(gpu, restated, shape, mode):
    import ephmc
    from oracle import Model
    l1, l2, nt, beta = shape
    m = Model.physical(l1, l2, nt, beta)
    x = restated.random_x(3, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld0, pd0 = ctx.eval(x, mode=mode)
        spread = max(_rel(ctx.eval(x, mode=mode)[1], pd0) for _ in range(3))
        tol = max(1e-10, 100 * spread)
        mem0 = ctx.memory()
        for C in (1, 8, 12, nt, nt + 5):
            ctx.set_checkpoint(C)
            ld, pd = ctx.eval(x, mode=mode)
            err = _rel(pd, pd0)
            print(f"{l1}x{l2} Nt={nt} {mode} C={C}: force {err:.2e} (run-to-run {spread:.1e}), "
                  f"memory {ctx.memory() / 1e6:.0f} MB (whole stack {mem0 / 1e6:.0f} MB)")
            assert ld == ld0, (C, ld, ld0)
            assert err <= tol, (C, err)
        ctx.set_checkpoint(0)
        ld, pd = ctx.eval(x, mode=mode)
        assert ld == ld0 and _rel(pd, pd0) <= tol


@pytest.mark.parametrize("shape", [(32, 32, 64, 20.0), (12, 12, 37, 10.0), (10, 10, 23, 8.0)])
def test_checkpointed_mixed_force_equals_segmented_whole_stack(gpu, restated, shape):
    """The mixed force's segments are the checkpoint interval: checkpointed
    (one FP32 region reused, segments bottom up, y chain in place) against
    the whole stack cut into the same segments (all regions, one launch).
    Same FP64 arithmetic for sweep 1, so the log det is bit-identical; the
    segments' FP64 start rows come from a batched GEMM in one case and single
    GEMMs in the other, which may round differently in the last bit before
    the FP32 sweep: the forces agree to 1e-6, and with segments of at most 16
    slices each is within 1e-5 of the FP64 force.  C >= Nt is one segment,
    the unsegmented FP32 sweep, whose error against FP64 (2e-3 at 32x32,
    Nt = 64) is what segmenting removes.  10x10 runs the shared-memory
    sweep (no register-strip or tile shape) segment by segment."""
    import ephmc
    from oracle import Model
    l1, l2, nt, beta = shape
    m = Model.physical(l1, l2, nt, beta)
    x = restated.random_x(3, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld64, pd64 = ctx.eval(x, mode="adjoint")
        for C in (1, 8, 12, nt, nt + 5) if l1 != 10 else (1, 2, 3, 8, nt):
            ctx.set_checkpoint(0)
            ctx.set_segment(C)
            ld_w, pd_w = ctx.eval(x, mode="mixed")
            mem_w = ctx.memory()
            ctx.set_checkpoint(C)
            ld, pd = ctx.eval(x, mode="mixed")
            err, err64 = _rel(pd, pd_w), _rel(pd, pd64)
            print(f"{l1}x{l2} Nt={nt} mixed C={C}: checkpointed vs whole {err:.2e}, vs FP64 {err64:.2e}, "
                  f"memory {ctx.memory() / 1e6:.0f} MB (whole stack {mem_w / 1e6:.0f} MB)")
            assert ld == ld_w, (C, ld, ld_w)
            assert abs(ld - ld64) <= 1e-12 * abs(ld64)
            assert err <= 1e-6, (C, err)
            if C <= 16:
                assert err64 <= 1e-5 and _rel(pd_w, pd64) <= 1e-5, (C, err64)


def test_checkpointed_single_particle_and_device_buffers(gpu, restated):
    """SINGLE_PARTICLE (y starts from the identity) through the checkpointed
    sweep, device-resident x and force."""
    import torch

    import ephmc
    from oracle import Model
    m = Model.physical(8, 8, 20, 5.0, flags=(0, 0, 0, 1, 0, 0, 0))
    x = restated.random_x(4, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, flags=m.flags) as ctx:
        ld0, pd0 = ctx.eval(x, mode="adjoint")
        ctx.set_checkpoint(6)
        xd = torch.from_numpy(x).cuda()
        pd = torch.empty_like(xd)
        ld, _ = ctx.eval(xd, pd, mode="adjoint")
    assert ld == ld0 and _rel(pd.cpu().numpy(), pd0) <= 1e-10


def test_cfg2_checkpoint_memory(gpu, restated):
    """48x48 (V = 2304), Nt = 128, beta = 40, checkpoints every 12 slices:
    10 FP64 checkpoints + a 12-slice segment (0.93 GB) instead of the
    5.4 GB stack; the context goes from 7.1 GB to 1.3 GB (measured 1.26);
    mixed force as with the whole stack."""
    import ephmc
    from oracle import Model
    m = Model.physical(48, 48, 128, 40.0)
    x = restated.random_x(5, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ctx.set_segment(12)  # the mixed force's segments: those of the checkpoints below
        ld0, pd0 = ctx.eval(x, mode="mixed")
        full = ctx.memory()
        t0 = ctx.timings()
        ctx.set_checkpoint(12)
        ld, pd = ctx.eval(x, mode="mixed")
        ck = ctx.memory()
        t1 = ctx.timings()
    print(f"48x48 Nt=128: memory {full / 1e9:.2f} GB -> {ck / 1e9:.2f} GB; force phase {t0[2]:.1f} -> {t1[2]:.1f} ms, "
          f"M_hat {t0[0]:.1f} -> {t1[0]:.1f} ms")
    assert ld == ld0 and _rel(pd, pd0) <= 1e-6
    assert ck < 1.3e9 and full > 4 * ck
