"""CPU tests: the oracle restatement pinned against the reference's golden vectors.

The fixtures in tests/golden/ come from the reference's own C sources compiled
unmodified (tests/golden/make_golden.py).  Where the reference library itself
is available (oracle/_ref), the restatement is also compared live.
"""
import hashlib

import numpy as np
import pytest

from conftest import golden, model_from_golden


def test_mt19937_64_stream(restated):
    g = golden("rng_lattice.npz")
    for s in (1, 5489, 2 ** 40 + 7):
        restated.lib.or_mt_seed(s)
        u = np.array([restated.lib.or_mt_real2() for _ in range(32)])
        assert np.array_equal(u, g[f"uniform_{s}"]), s


def test_box_muller_normals_odd_and_even(restated):
    g = golden("rng_lattice.npz")
    assert np.array_equal(restated.random_x(1, 9), g["normals_1_n9"])
    assert np.array_equal(restated.random_x(3, 10), g["normals_3_n10"])


@pytest.mark.parametrize("l1,l2", [(1, 1), (1, 4), (4, 1), (2, 2), (2, 3), (3, 4), (6, 6)])
def test_lattice_bit_exact(restated, l1, l2):
    g = golden("rng_lattice.npz")
    assert np.array_equal(restated.lattice(l1, l2), g[f"nnt_{l1}x{l2}"])


@pytest.mark.parametrize("l1,l2", [(32, 32), (48, 48), (64, 64), (8, 12)])
def test_lattice_large_hash(restated, l1, l2):
    g = golden("rng_lattice.npz")
    assert hashlib.sha256(restated.lattice(l1, l2).tobytes()).hexdigest() == str(g[f"nnt_sha256_{l1}x{l2}"])


WELL_CONDITIONED = ["small_L6_Nt64", "rect_L4x3_Nt16", "odd_L5x6_Nt12", "tiny_L2x2_Nt4", "line_L1x4_Nt5",
                    "single_slice_L3x3_Nt1"]


@pytest.mark.parametrize("name", WELL_CONDITIONED)
def test_restated_eval_matches_reference_fixture(restated, name):
    g = golden(f"eval_{name}.npz")
    m = model_from_golden(g)
    for n, seed in enumerate(g["seeds"]):
        x = restated.random_x(int(seed), m.dim)
        M = restated.construct_M_hat(m, x)
        assert np.array_equal(M, g["M_hat"][n]), "M_hat must be bit-identical to the reference"
        ld, pd, Mi, sign = restated.eval_reference(m, x)
        assert abs(ld - g["logdet"][n]) <= 1e-12 * abs(g["logdet"][n]) + 1e-13
        tol = max(1e-10, 10 * float(g["force_spread_max"][n]))
        assert np.max(np.abs(pd - g["force"][n])) <= tol * np.max(np.abs(g["force"][n]))
        assert np.max(np.abs(Mi - g["M_inv"][n])) <= 1e-10 * np.max(np.abs(g["M_inv"][n]))


@pytest.mark.parametrize("name", WELL_CONDITIONED)
def test_restated_adjoint_matches_reference_fixture(restated, name):
    g = golden(f"eval_{name}.npz")
    m = model_from_golden(g)
    x = restated.random_x(int(g["seeds"][0]), m.dim)
    ld, pd = restated.eval_adjoint(m, x)
    tol = max(1e-10, 10 * float(g["force_spread_max"][0]))
    assert abs(ld - g["logdet"][0]) <= 1e-12 * abs(g["logdet"][0]) + 1e-13
    assert np.max(np.abs(pd - g["force"][0])) <= tol * np.max(np.abs(g["force"][0]))


def test_mid_size_reference_fixture(restated):
    g = golden("eval_mid_L16_Nt64.npz")
    m = model_from_golden(g)
    x = restated.random_x(1, m.dim)
    M = restated.construct_M_hat(m, x)
    assert hashlib.sha256(M.tobytes()).hexdigest() == str(g["M_hat_sha256"][0])


def test_cfg0_is_outside_the_taylor_regime(restated):
    """The literal small config (dtau = 0.625) is ill-conditioned: the
    reference's own 1- and N-thread runs disagree in the force at O(1).  What
    is reproducible is M_hat (bitwise) and the magnitude of log det."""
    g = golden("eval_cfg0_L6_Nt16_beta10.npz")
    m = model_from_golden(g)
    x = restated.random_x(1, m.dim)
    assert np.array_equal(restated.construct_M_hat(m, x), g["M_hat"][0])
    assert float(g["force_spread_max"][0]) > 1e-3
    ld, _, _, _ = restated.eval_reference(m, x)
    assert abs(ld - g["logdet"][0]) <= 5e-3 * abs(g["logdet"][0])


def test_fa_routines_match_reference_fixture(restated):
    g = golden("fa_bosons.npz")
    for (L, nt) in ((4, 16), (6, 64), (3, 5)):
        tag = f"L{L}_Nt{nt}"
        om = float(g[f"{tag}_omega"])
        ns = L * L
        xe, pe = restated.evolve_bosons(g[f"{tag}_x"], g[f"{tag}_p"], om, ns, nt, 0.3)
        assert np.allclose(xe, g[f"{tag}_x_evolved"], rtol=0, atol=1e-12)
        assert np.allclose(pe, g[f"{tag}_p_evolved"], rtol=0, atol=1e-12)
        pm = restated.sample_fourier_momenta(31, om, ns, nt)
        assert np.allclose(pm, g[f"{tag}_p_sampled_seed31"], rtol=0, atol=1e-12)
        e = restated.energy_fourier_momenta(pm, om, ns, nt)
        assert abs(e - float(g[f"{tag}_energy_of_p_sampled"])) <= 1e-12 * abs(e)
        xf = restated.sample_free_bosons(41, om, ns, nt)
        assert np.allclose(xf, g[f"{tag}_x_free_seed41"], rtol=0, atol=1e-12)
        assert abs(restated.higher_matsubaras_norm(g[f"{tag}_x"], ns, nt) - float(g[f"{tag}_higher_matsubara_x"])) < 1e-10
        h = restated.hamilton(g[f"{tag}_x"], 1.5, 2.5, om, 1, ns, nt)
        assert abs(h - float(g[f"{tag}_hamilton_x"])) <= 1e-12 * abs(h)


def test_free_fermion_log_det_is_analytic(restated):
    """lambda = 0: every B_t = p(mu + K) is diagonal in momentum space, so
    log det(1 + prod B_t) = sum_k log(1 + p(eps_k)^Nt) with
    eps_k = mu + 2 sum_a t_a cos(k.e_a) and p the product of the two pair
    quadratics (the free-electron pin of simulation/organic_hmc.R:68-109)."""
    from oracle import Model
    L1, L2, nt = 6, 4, 16
    m = Model.physical(L1, L2, nt, 4.0, lam=(0.0, 0.0, 0.0), mu0=0.5)
    x = restated.random_x(3, m.dim)  # irrelevant at kappa = 0
    ld, pd, _, _ = restated.eval_reference(m, x)
    al, aq = np.zeros(2), np.zeros(2)
    coeff = np.array([1.8294933739891903 + 0.9404019519941707j, 0.1705066260108097 + 1.5785318126884535j])
    a = 0.5 * coeff / 2
    al, aq = 2 * a.real, np.abs(a) ** 2
    k1 = 2 * np.pi * np.arange(L1) / L1
    k2 = 2 * np.pi * np.arange(L2) / L2
    K1, K2 = np.meshgrid(k1, k2, indexing="ij")
    t = m.t
    # links: right (e1), top-right (e2), top-left (e2 - e1)
    eps = m.mu + 2 * (t[0] * np.cos(K1) + t[1] * np.cos(K2) + t[2] * np.cos(K2 - K1))
    p = (1 + al[0] * eps + aq[0] * eps ** 2) * (1 + al[1] * eps + aq[1] * eps ** 2)
    exact = np.sum(np.log1p(p ** nt))
    assert abs(ld - exact) <= 1e-11 * abs(exact)
    assert np.all(pd == 0.0)


def test_restated_live_against_reference(restated, reference):
    from oracle import Model
    m = Model.physical(4, 5, 8, 3.0)
    x = reference.random_x(17, m.dim)
    ctx = reference.context(m)
    reference.set_threads(1)
    ld_r, pd_r, Mp_r, Mi_r = ctx.eval(x, want_M=True)
    ld, pd, Mi, _ = restated.eval_reference(m, x)
    assert np.array_equal(restated.construct_M_hat(m, x), Mp_r)
    assert abs(ld - ld_r) <= 1e-13 * abs(ld_r)
    assert np.max(np.abs(pd - pd_r)) <= 1e-11 * np.max(np.abs(pd_r))
    G_r = ctx.all_QM1P(x, Mi_r)
    G = restated.all_G(m, x, Mi_r)
    assert np.array_equal(G, G_r), "log-depth sharing must be bit-identical given the same inverse"
    for t in (0, 3, 7):
        assert np.array_equal(restated.refine(m, x, G[t], t), ctx.refine(x, G_r[t], t))


def test_reference_classical_acceleration_step_matches_its_formula(reference):
    """The reference's evolve_bosons_approx_step (through oracle/ref_driver.c)
    equals x + irfft((h / freq2_k) rfft(p)) per series, with
    freq2_k = w + (2 sin(pi k / Nt))^2 / w and w = sqrt(cfa_mass^2 + omega^2)
    (simulation/organic_bosons.c:152-177)."""
    from oracle import RefFA
    ns, nt = 4, 16
    fa = RefFA(reference, ns, nt)
    rng = np.random.default_rng(1)
    ld = 3 * ns
    x, p = rng.standard_normal(ld * nt), rng.standard_normal(ld * nt)
    fa.set(x, p)
    omega, h, mass = 0.3, 0.2, 0.5
    fa.approx_step(omega, h, mass)
    xr, pr = fa.get()
    w = np.sqrt(mass ** 2 + omega ** 2)
    k = np.arange(nt // 2 + 1)
    f2 = w + (2 * np.sin(np.pi * k / nt)) ** 2 / w
    xn = x.reshape(nt, ld) + np.fft.irfft((h / f2)[:, None] * np.fft.rfft(p.reshape(nt, ld), axis=0), n=nt, axis=0)
    assert np.max(np.abs(xr - xn.ravel())) <= 1e-13
    assert np.array_equal(pr, p)


TL_CASES = ["L6x5_nb64", "L8x8_nb128", "L5x7_nb32_beta10", "L6x6_nb64_mu-3"]


def _tl_case(g, tag):
    return dict(l1=int(g[f"{tag}_l1"]), l2=int(g[f"{tag}_l2"]), nbins=int(g[f"{tag}_nbins"]), t=g[f"{tag}_t"],
                kappa=g[f"{tag}_kappa"], mu=float(g[f"{tag}_mu"]), contr_mat=g[f"{tag}_contr_mat"],
                width=float(g[f"{tag}_width"]))


@pytest.mark.parametrize("tag", TL_CASES)
def test_trans_loc_restatement_matches_reference_fixture(tag):
    """The numpy restatement of hist_trans_loc against the reference's own
    output (tests/golden/trans_loc.npz, simulation/organic_trans_loc.c:25-83)
    on the reference's bond fields: histograms within 1e-10 of the largest bin
    (measured 1e-13), partition sums within 1e-12."""
    from oracle import trans_loc_sample
    g = golden("trans_loc.npz")
    c = _tl_case(g, tag)
    xs = g[f"{tag}_x"]
    h = np.zeros(c["nbins"])
    z = []
    for x in xs:
        hs, zs = trans_loc_sample(x, **c)
        h += hs
        z.append(zs)
    ref = g[f"{tag}_greens"]
    assert np.max(np.abs(h - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert np.allclose(z, g[f"{tag}_z"], rtol=1e-12, atol=0)
    # the mu0 = -3 case is the one whose default width leaves bins past the end
    assert bool(g[f"{tag}_overflow"]) == (tag == "L6x6_nb64_mu-3")


def test_trans_loc_reference_reproduces_its_fixture(reference):
    """The fixture generator's call, repeated on this host: the same MT19937-64
    bond fields bit for bit and the same histogram to 1e-12 (OpenBLAS may pick
    other kernels on another CPU)."""
    g = golden("trans_loc.npz")
    tag = "L6x5_nb64"
    c = _tl_case(g, tag)
    reference.set_threads(1)
    h, z, xs, ov = reference.trans_loc_samples(int(g[f"{tag}_seed"]), c["l1"], c["l2"], c["nbins"], c["t"],
                                               c["kappa"], c["mu"], c["contr_mat"], c["width"], len(g[f"{tag}_z"]))
    assert np.array_equal(xs, g[f"{tag}_x"])
    assert np.max(np.abs(h - g[f"{tag}_greens"])) <= 1e-12 * np.max(np.abs(h))
    assert np.allclose(z, g[f"{tag}_z"], rtol=1e-13, atol=0) and not ov


def test_trans_loc_degenerate_spectrum_is_ill_posed_in_the_reference(reference):
    """Without disorder (lambda = 0) a 4x4 lattice has exactly degenerate
    levels.  The reference keeps pairs with E_j >= E_i, so an exactly tied
    pair counts twice and a pair split by one ulp once: bin 0 then depends on
    the eigensolver's rounding.  LAPACK's dsyev (the reference) and numpy's
    eigh disagree there by up to a factor 2, while every other bin agrees.
    Parity cases therefore carry disorder."""
    from oracle import contraction_matrix, convert_params, trans_loc_sample
    t, kappa, mu, _ = convert_params(10.0, 32, lam=(0, 0, 0), mu0=0.0, static_disorder=True)
    cm = contraction_matrix((1.0, 0.0), (0.5, 0.8660254))
    width = (-2 * mu + 8 * np.abs(kappa).sum()) / 32 * 1.0137
    reference.set_threads(1)
    h, _, xs, _ = reference.trans_loc_samples(7, 4, 4, 32, t, kappa, mu, cm, width, 1)
    r, _ = trans_loc_sample(xs[0], 4, 4, 32, t, kappa, mu, cm, width)
    assert np.max(np.abs(h[1:] - r[1:])) <= 1e-10 * np.max(np.abs(h))


@pytest.mark.parametrize("tag", ["L8x8_nb128", "L16x16_nb512"])
def test_conv_restatement_matches_reference_fixture(tag):
    """organic_conv's smearing and tanh-sinh time transform restated in numpy
    against the reference's smeared_sigma_w / smeared_sigma_t
    (simulation/organic_conv.c:92-121, tests/golden/conv.npz): 1e-13
    (measured 1.3e-15)."""
    from oracle import conv_sigma_t, conv_sigma_w
    g = golden("conv.npz")
    sig, h, wd, nt = g[f"{tag}_sigma"], float(g[f"{tag}_h"]), g[f"{tag}_widths"], int(g[f"{tag}_nt"])
    assert np.allclose(conv_sigma_w(sig, h, wd), g[f"{tag}_w"], rtol=1e-13, atol=0)
    assert np.allclose(conv_sigma_t(sig, h, wd, nt), g[f"{tag}_t"], rtol=1e-13, atol=0)
