"""CPU tests of the Python host layer (package ``ephmc``) that needs no GPU.

The neighbour table a caller builds with ``ephmc.lattice`` must be the
reference's construct_triangular table (simulation/organic_lattice.c), and
``ephmc.convert_params`` must give organic_main's lattice units
(simulation/organic_main.c:99-116), bit for bit: both feed the library
directly when a host program drives it from Python."""
import hashlib

import numpy as np
import pytest

from conftest import golden

SMALL = [(1, 1), (1, 4), (4, 1), (2, 2), (2, 3), (3, 4), (6, 6)]
LARGE = [(32, 32), (48, 48), (64, 64), (8, 12)]


@pytest.mark.parametrize("l1,l2", SMALL)
def test_host_lattice_is_the_reference_table(l1, l2):
    import ephmc
    g = golden("rng_lattice.npz")
    nnt = ephmc.lattice(l1, l2)
    assert nnt.dtype == np.uint32 and nnt.shape == (12 * l1 * l2,)
    assert np.array_equal(nnt, g[f"nnt_{l1}x{l2}"])


@pytest.mark.parametrize("l1,l2", LARGE)
def test_host_lattice_large_hash(l1, l2):
    import ephmc
    g = golden("rng_lattice.npz")
    assert hashlib.sha256(ephmc.lattice(l1, l2).tobytes()).hexdigest() == str(g[f"nnt_sha256_{l1}x{l2}"])


@pytest.mark.parametrize("beta,nt,static", [(20.0, 64, False), (10.0, 16, False), (40.0, 128, False),
                                            (40.0, 512, True)])
def test_host_convert_params_equals_the_oracle(beta, nt, static):
    import ephmc
    import oracle
    J, lam, mu0, om0 = (1.0, -0.5, -0.5), (0.3, 0.15, 0.15), -3.0, 0.05
    a = ephmc.convert_params(beta, nt, J, lam, mu0, om0, static_disorder=static)
    b = oracle.convert_params(beta, nt, J, lam, mu0, om0, static_disorder=static)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))


def test_no_gpu_fails_loudly():
    """Without a CUDA device every handle's creation raises EphmcError with the
    library's status and message: nothing falls back to a CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import ephmc
    t, kappa, mu, omega = ephmc.convert_params(10.0, 16, (1.0, -0.5, -0.5), (0.3, 0.15, 0.15), -3.0, 0.05)
    with pytest.raises(ephmc.EphmcError, match="ephmc_ctx_create: status 9"):
        ephmc.Context(4, 4, 16, t, kappa, mu, omega)
    cm = ephmc.contraction_matrix((1.0, 0.0), (0.5, 0.8660254))
    with pytest.raises(ephmc.EphmcError, match="ephmc_tl_create: status 9"):
        ephmc.TransLoc(4, 4, 16, t, kappa, mu, cm)
    sigma, widths = np.ones(16), np.array([0.1])
    with pytest.raises(ephmc.EphmcError, match="status 9"):
        ephmc.conv_sigma_w(sigma, 0.1, widths)
    with pytest.raises(ephmc.EphmcError, match="status 9"):
        ephmc.conv_sigma_t(sigma, 0.1, widths, 8)
