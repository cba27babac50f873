"""The adjoint force as the gradient of log det through torch.autograd
(tests/autograd_harness.py): against the reference's own force, against
central finite differences, and inside a composite action."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["adjoint", "mixed"])
def test_autograd_gradient_is_the_reference_force(gpu, reference, restated, mode):
    """d log det / dx by backward() equals the reference's p_dot / flavors
    (6x6, Nt = 16, beta = 5, two flavours): FP64 adjoint to 1e-10, mixed to
    1e-5 of the largest entry."""
    import torch

    import ephmc
    from autograd_harness import LogDet
    from oracle import Model
    m = Model.physical(6, 6, 16, 5.0, flavors=2)
    x0 = restated.random_x(11, m.dim)
    reference.set_threads(1)
    rc = reference.context(m)
    ld_r, pd_r = rc.eval(x0)
    rc.close()
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, flavors=2) as ctx:
        x = torch.from_numpy(x0.copy()).cuda().requires_grad_(True)
        ld = LogDet.apply(x, ctx, mode)
        ld.backward()
        g = x.grad.cpu().numpy()
    assert abs(ld.item() - ld_r) <= 1e-12 * abs(ld_r)
    err = np.max(np.abs(g - pd_r / 2)) / np.max(np.abs(pd_r / 2))
    assert err <= (1e-5 if mode == "mixed" else 1e-10), err


def test_autograd_composite_action_against_finite_differences(gpu, restated):
    """S(x) = -flavors log det M(x) + 0.5 w . x^2 differentiated by autograd
    (the library's adjoint for the first term, torch for the second), against
    central differences of S on 24 entries, step 1e-5."""
    import torch

    import ephmc
    from autograd_harness import LogDet
    from oracle import Model
    m = Model.physical(6, 6, 16, 5.0)
    x0 = restated.random_x(12, m.dim)
    w = np.random.default_rng(1).uniform(0.5, 1.5, m.dim)
    wt = torch.from_numpy(w).cuda()
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        def action(xt):
            return -LogDet.apply(xt, ctx, "adjoint") + 0.5 * (wt * xt * xt).sum()

        x = torch.from_numpy(x0.copy()).cuda().requires_grad_(True)
        action(x).backward()
        g = x.grad.cpu().numpy()
        idx = np.random.default_rng(2).choice(m.dim, 24, replace=False)
        h = 1e-5
        fd = []
        with torch.no_grad():
            for i in idx:
                xp = torch.from_numpy(x0.copy()).cuda()
                xp[i] += h
                xm = torch.from_numpy(x0.copy()).cuda()
                xm[i] -= h
                fd.append((action(xp) - action(xm)).item() / (2 * h))
    fd = np.array(fd)
    err = np.max(np.abs(g[idx] - fd)) / np.max(np.abs(fd))
    print(f"composite action: autograd vs central differences {err:.2e}")
    assert err <= 1e-6
