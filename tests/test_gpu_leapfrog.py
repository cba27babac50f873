"""ephmc_leapfrog (the MD part of a trajectory, simulation/organic_hmc.c:167-190,
issued without host waits) against the same leapfrog written with the
synchronous calls: ephmc_eval for the force, ephmc_fa_evolve (or x += h p
without Fourier acceleration) for update_x, and p += h p_dot on the host.
Both run the same kernels; the force's cross-CTA atomic sums may differ in
order, so x and p agree to 1e-8 after the trajectory.  The drop-in chain
tests (test_gpu_dropin.py) run this path too, inside the reference's own
organic_main against the reference program."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _emulate(ctx, x, p, steps, traj, mode, no_fa):
    x, p = x.copy(), p.copy()
    h = traj / steps if steps else 2 * traj

    def update_x(w):
        if no_fa:
            x[:] += w * p
        else:
            ctx.fa_evolve(x, p, w)

    update_x(0.5 * h)
    for s in range(1, steps + 1):
        _, pd = ctx.eval(x, mode=mode)
        p += h * pd
        update_x((0.5 if s == steps else 1.0) * h)
    return x, p


@pytest.mark.parametrize("no_fa", [False, True])
@pytest.mark.parametrize("mode", ["reference", "adjoint", "mixed"])
def test_leapfrog_equals_synchronous_steps(gpu, restated, mode, no_fa):
    import torch

    import ephmc
    from oracle import Model
    flags = (0, 0, 0, 0, 0, 1, 0) if no_fa else (0,) * 7
    m = Model.physical(12, 12, 16, 5.0, flags=flags)
    x0 = restated.random_x(3, m.dim) * 0.3
    p0 = restated.random_x(4, m.dim)
    steps, traj = 5, 0.4
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, flags=flags) as ctx:
        # momenta of the accelerated distribution (sample_fourier_momenta): with
        # unscaled N(0,1) momenta the slowest mode (freq2 ~ 2e-4) moves x by
        # hundreds in one step and the force becomes chaotic
        if not no_fa:
            ctx.fa_scale_momenta(p0)
        xe, pe = _emulate(ctx, x0, p0, steps, traj, mode, no_fa)
        xd, pd = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(p0.copy()).cuda()
        neg = ctx.leapfrog(xd, pd, steps, traj, mode)
        xg, pg = xd.cpu().numpy(), pd.cpu().numpy()
        # a second call continues from the state the first left
        neg2 = ctx.leapfrog(xd, pd, steps, traj, mode)
    ex = np.max(np.abs(xg - xe)) / np.max(np.abs(xe))
    ep = np.max(np.abs(pg - pe)) / np.max(np.abs(pe))
    print(f"{mode} no_fa={no_fa}: x {ex:.1e}, p {ep:.1e}")
    assert ex <= 1e-8 and ep <= 1e-8
    assert neg == 0 and neg2 == 0
    assert np.isfinite(xd.cpu().numpy()).all()


def test_leapfrog_rejects_what_needs_the_host(gpu, restated):
    """SINGLE_PARTICLE scales the force by exp(-log det): that path stays
    synchronous, and host buffers are refused."""
    import torch

    import ephmc
    from oracle import Model
    m = Model.physical(6, 6, 8, 5.0, flags=(0, 0, 0, 1, 0, 0, 0))
    x = torch.zeros(m.dim, dtype=torch.float64, device="cuda")
    p = torch.zeros_like(x)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, flags=m.flags) as ctx:
        with pytest.raises(ephmc.EphmcError) as e:
            ctx.leapfrog(x, p, 2, 0.1)
        assert e.value.status == 7
    m = Model.physical(6, 6, 8, 5.0)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        with pytest.raises(ephmc.EphmcError) as e:
            ctx.leapfrog(np.zeros(m.dim), np.zeros(m.dim), 2, 0.1)
        assert e.value.status == 2


@pytest.mark.parametrize("mode", ["reference", "adjoint", "mixed"])
def test_leapfrog_graph_equals_leapfrog(gpu, restated, mode):
    """ephmc_leapfrog_graph against ephmc_leapfrog from the same start: the
    first call (capture, then launch) and the second (replay) both give the
    direct path's x and p.  After a change of the couplings the next call
    captures again and still agrees.  Every trajectory starts from the same
    (x, p): from this start the dynamics amplifies the rounding-level order
    of the force's atomic sums by about 1e4 per trajectory, so chained
    trajectories would compare nothing but that."""
    import torch

    import ephmc
    from oracle import Model
    m = Model.physical(12, 12, 16, 5.0)
    x0 = restated.random_x(5, m.dim) * 0.3
    p0 = restated.random_x(6, m.dim)

    def run(ctx, graph):
        x, p = torch.from_numpy(x0.copy()).cuda(), torch.from_numpy(p0.copy()).cuda()
        ctx.leapfrog(x, p, 4, 0.3, mode, graph=graph)
        return x.cpu().numpy(), p.cpu().numpy()

    def close(a, b):
        return (np.max(np.abs(a[0] - b[0])) <= 1e-12 * np.max(np.abs(b[0])) and
                np.max(np.abs(a[1] - b[1])) <= 1e-12 * np.max(np.abs(b[1])))

    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ctx.fa_scale_momenta(p0)
        # fixed buffers, as a caller replaying the graph uses them
        xb = torch.empty(m.dim, dtype=torch.float64, device="cuda")
        pb = torch.empty_like(xb)

        def run_fixed(graph):
            xb.copy_(torch.from_numpy(x0))
            pb.copy_(torch.from_numpy(p0))
            ctx.leapfrog(xb, pb, 4, 0.3, mode, graph=graph)
            return xb.cpu().numpy(), pb.cpu().numpy()

        direct = run_fixed(False)
        first = run_fixed(True)    # capture + launch
        second = run_fixed(True)   # replay
        assert close(first, direct) and close(second, direct)
        # new couplings: the captured graph is stale and must not be replayed
        t_new = np.ascontiguousarray(0.9 * m.t)
        k_new = np.ascontiguousarray(m.kappa)
        ctx.lib.ephmc_ctx_set_params(ctx.h, t_new.ctypes.data, k_new.ctypes.data, m.mu, m.omega, 1)
        direct2 = run_fixed(False)
        assert not close(direct2, direct)
        assert close(run_fixed(True), direct2)
        del run
