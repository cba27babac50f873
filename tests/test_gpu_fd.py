"""The force against central finite differences of the log det, the check of
simulation/organic_hmc.c:20-54 (check_force), on 64 randomly chosen
(slice, site, link) entries of an N(0,1) phonon field with step 1e-4, on a
48x48 lattice (the lattice of the checkpointing configuration; V = 2304 also
runs the LU's multi-launch path for V > 1024) with Nt = 64, beta = 20
(dtau = 0.3125, the 32x32 workload's), where the raw slice product that the
reference factors resolves log det well.  At that configuration's
beta = 40, Nt = 128 it does not (the log det moves by rounding noise of
about 1e-6 under a 1e-4 step, for the reference as for the unstabilised
path); that case runs with the re-stabilised chain in test_gpu_stabilize.py.

    f_i = flavors (log det M(x + h e_i) - log det M(x - h e_i)) / (2 h)

is compared with the FP64 force of the reference algorithm, the FP64 adjoint
force (one CTA per vector at this size: nine vectors of V doubles and the
hopping table fill 216 of the 227 KB of shared memory) and the mixed force
on the same entries."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_force_matches_central_differences(gpu, restated):
    import torch

    import ephmc
    from oracle import Model
    m = Model.physical(48, 48, 64, 20.0)
    x = restated.random_x(3, m.dim)
    rng = np.random.default_rng(17)
    idx = rng.choice(m.dim, size=64, replace=False)
    h = 1e-4
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega, m.flavors) as ctx:
        _, pda = ctx.eval(x, mode="adjoint")
        _, pd64 = ctx.eval(x, mode="reference")
        _, pdm = ctx.eval(x, mode="mixed")
        V = ctx.V
        xd = torch.from_numpy(x.copy()).cuda()
        Md = torch.empty(V * V, dtype=torch.float64, device="cuda")
        fd = np.empty(len(idx))
        for n, i in enumerate(idx):
            keep = float(x[i])
            ld = []
            for s in (+1.0, -1.0):
                xd[i] = keep + s * h
                ctx.construct_M_hat(xd, Md)
                ld.append(ctx.logdet_inverse(Md)[0])
            xd[i] = keep
            fd[n] = m.flavors * (ld[0] - ld[1]) / (2 * h)
    scale = np.max(np.abs(fd))
    err64 = float(np.max(np.abs(pd64[idx] - fd)) / scale)
    erra = float(np.max(np.abs(pda[idx] - fd)) / scale)
    errm = float(np.max(np.abs(pdm[idx] - fd)) / scale)
    print(f"48x48 Nt=64 beta=20: FD vs FP64 reference {err64:.2e}, vs FP64 adjoint {erra:.2e}, vs mixed {errm:.2e} "
          f"(max |f| {scale:.3e})")
    # the adjoint path builds M_hat with the register-tile sweep, which sums in
    # another order than the reference path: the two forces differ by M_hat's
    # rounding amplified by its conditioning (measured 1.1e-8 of max |f|)
    assert float(np.max(np.abs(pda - pd64))) <= 1e-7 * float(np.max(np.abs(pd64)))
    # measured 1.7e-5 (the mixed force: 8.5e-4 unsegmented).  The FD quotient itself is good to about
    # (rounding of log det ~ 2e-10) / (2 h) ~ 1e-6 absolute, 1.5e-5 of max |f|.
    assert err64 <= 1e-4
    assert errm <= 1e-4
    assert errm <= 1e-2
