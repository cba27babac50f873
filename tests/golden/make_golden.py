"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own C sources, compiled unmodified into
oracle/_ref/libephref.so (``make -C oracle ref``), and stores the outputs as
small .npz files.  Run it in a checkout that has the reference sources
(it is not run by the tests; the fixtures are committed):

    python tests/golden/make_golden.py [--skip-cfg1] [--only trans_loc|conv]

Every evaluation is done twice, with 1 and with N OpenMP/OpenBLAS threads;
the spread between the two (the reference's own reproducibility, which comes
from OpenBLAS's LU reduction order) is stored beside the values and anchors
the parity tolerances of the GPU tests.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Model, Reference, rel_max  # noqa: E402

NTHREADS = max(2, min(8, os.cpu_count() or 2))


def spread(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(rel_max(a, b)), float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def eval_pair(ref: Reference, m: Model, seed: int, want_M=True):
    x = ref.random_x(seed, m.dim)
    ctx = ref.context(m)
    ref.set_threads(1)
    ld1, pd1, Mp1, Mi1 = ctx.eval(x, want_M=True)
    t1 = ctx.last_time()
    ref.set_threads(NTHREADS)
    ldN, pdN, MpN, MiN = ctx.eval(x, want_M=True)
    tN = ctx.last_time()
    ctx.close()
    out = dict(seed=seed, logdet=ld1, logdet_mt=ldN, force=pd1, t_1thr=t1, t_mthr=tN, threads=NTHREADS)
    out["force_spread_max"], out["force_spread_norm"] = spread(pdN, pd1)
    out["minv_spread_max"], _ = spread(MiN, Mi1)
    out["logdet_spread"] = abs(ldN - ld1) / max(abs(ld1), 1e-300)
    assert np.array_equal(Mp1, MpN), "M_hat must not depend on the thread count"
    if want_M:
        out["M_hat"] = Mp1
        out["M_inv"] = Mi1
    else:
        out["M_hat_sha256"] = hashlib.sha256(np.ascontiguousarray(Mp1).tobytes()).hexdigest()
    return x, out


def model_meta(m: Model):
    return dict(l1=m.l1, l2=m.l2, nt=m.nt, t=m.t, kappa=m.kappa, mu=m.mu, omega=m.omega, flavors=m.flavors,
                beta=m.beta)


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KB)")


def gen_rng_lattice(ref: Reference):
    d = {}
    for s in (1, 5489, 2 ** 40 + 7):
        d[f"uniform_{s}"] = ref.uniforms(s, 32)
    d["normals_1_n9"] = ref.random_x(1, 9)
    d["normals_3_n10"] = ref.random_x(3, 10)
    for (l1, l2) in ((1, 1), (1, 4), (4, 1), (2, 2), (2, 3), (3, 4), (6, 6)):
        d[f"nnt_{l1}x{l2}"] = ref.lattice(l1, l2)
    for (l1, l2) in ((32, 32), (48, 48), (64, 64), (8, 12)):
        d[f"nnt_sha256_{l1}x{l2}"] = np.array(hashlib.sha256(ref.lattice(l1, l2).tobytes()).hexdigest())
    save("rng_lattice.npz", **d)


def gen_evals(ref: Reference):
    cases = [
        ("small_L6_Nt64", Model.physical(6, 6, 64, 20.0), (1, 2, 3), True),
        ("rect_L4x3_Nt16", Model.physical(4, 3, 16, 5.0), (7,), True),
        ("odd_L5x6_Nt12", Model.physical(5, 6, 12, 4.0), (11,), True),
        ("tiny_L2x2_Nt4", Model.physical(2, 2, 4, 2.0), (5,), True),
        ("line_L1x4_Nt5", Model.physical(1, 4, 5, 2.0), (9,), True),
        ("single_slice_L3x3_Nt1", Model.physical(3, 3, 1, 0.5), (4,), True),
        ("cfg0_L6_Nt16_beta10", Model.physical(6, 6, 16, 10.0), (1,), True),
        ("mid_L16_Nt64", Model.physical(16, 16, 64, 20.0), (1,), False),
    ]
    for name, m, seeds, want_M in cases:
        res = []
        for s in seeds:
            t0 = time.time()
            x, o = eval_pair(ref, m, s, want_M)
            res.append(o)
            print(f"{name} seed {s}: logdet {o['logdet']:.12g} spread {o['force_spread_max']:.2e} ({time.time() - t0:.1f}s)")
        d = model_meta(m)
        d["seeds"] = np.array(seeds)
        for key in res[0]:
            if key == "seed":
                continue
            vals = [r[key] for r in res]
            d[key] = np.array(vals) if not isinstance(vals[0], str) else np.array(vals)
        save(f"eval_{name}.npz", **d)


def gen_cfg1(ref: Reference, nseeds: int):
    """32x32, Nt=64, beta=20: 50 fixed configurations, logdet + action + force summaries."""
    m = Model.physical(32, 32, 64, 20.0)
    rng = np.random.default_rng(20240601)
    sample_idx = np.sort(rng.choice(m.dim, 256, replace=False))
    logdet, spread_f, spread_fn, ham, fnorm, fsum, fsample, tt = [], [], [], [], [], [], [], []
    full = None
    ctx = ref.context(m)
    for s in range(1, nseeds + 1):
        x = ref.random_x(s, m.dim)
        ref.set_threads(NTHREADS)
        t0 = time.time()
        ld, pd = ctx.eval(x)
        tt.append(ctx.last_time())
        if s <= 2:
            ref.set_threads(1)
            ld1, pd1 = ctx.eval(x)
            a, b = spread(pd, pd1)
            spread_f.append(a)
            spread_fn.append(b)
        if s == 1:
            full = pd.copy()
        logdet.append(ld)
        ham.append(ref.hamilton(x, ld, 0.0, m.omega, 1, m.ns, m.nt))
        fnorm.append(np.linalg.norm(pd))
        fsum.append(pd.sum())
        fsample.append(pd[sample_idx])
        print(f"cfg1 seed {s}: logdet {ld:.13g} ({time.time() - t0:.1f}s)")
    ctx.close()
    d = model_meta(m)
    d.update(seeds=np.arange(1, nseeds + 1), logdet=np.array(logdet), hamilton=np.array(ham),
             force_norm=np.array(fnorm), force_sum=np.array(fsum), force_sample=np.array(fsample),
             sample_idx=sample_idx, force_seed1=full, force_spread_max=np.array(spread_f),
             force_spread_norm=np.array(spread_fn), t_eval_mthr=np.array(tt), threads=NTHREADS)
    save("eval_cfg1_L32_Nt64.npz", **d)


def gen_fa(ref: Reference):
    d = {}
    for (L, nt) in ((4, 16), (6, 64), (3, 5)):
        m = Model.physical(L, L, nt, 10.0)
        ns = m.ns
        fa = ref.fa(ns, nt)
        x = ref.random_x(21, 3 * ns * nt)
        p = ref.random_x(22, 3 * ns * nt)
        fa.set(x, p)
        fa.evolve(m.omega, 0.3)
        xe, pe = fa.get()
        fa.sample_momenta(31, m.omega)
        _, pm = fa.get()
        en = fa.energy(m.omega)
        fa.sample_free(41, m.omega)
        xf, _ = fa.get()
        tag = f"L{L}_Nt{nt}"
        d.update({f"{tag}_omega": m.omega, f"{tag}_x": x, f"{tag}_p": p, f"{tag}_x_evolved": xe,
                  f"{tag}_p_evolved": pe, f"{tag}_p_sampled_seed31": pm, f"{tag}_energy_of_p_sampled": en,
                  f"{tag}_x_free_seed41": xf,
                  f"{tag}_higher_matsubara_x": ref.higher_matsubaras_norm(x, ns, nt),
                  f"{tag}_hamilton_x": ref.hamilton(x, 1.5, 2.5, m.omega, 1, ns, nt)})
        fa.close()
    save("fa_bosons.npz", **d)


# static-disorder cases: (l1, l2, bins, beta, mu0, lambda, samples, seed); beta, mu0
# and lambda in input.txt units, converted as organic_main does with STATIC_DISORDER
TL_CASES = {
    "L6x5_nb64": (6, 5, 64, 40.0, 0.0, (0.3, 0.15, 0.15), 3, 7),
    "L8x8_nb128": (8, 8, 128, 40.0, 0.0, (0.3, 0.15, 0.15), 2, 8),
    "L5x7_nb32_beta10": (5, 7, 32, 10.0, 0.5, (0.2, 0.1, 0.3), 3, 9),
    # mu0 = -3: the default width does not cover the band; the reference writes
    # bins past the end of greens (into the results behind it), the in-range
    # bins are what both compute
    "L6x6_nb64_mu-3": (6, 6, 64, 40.0, -3.0, (0.3, 0.15, 0.15), 2, 10),
}
TL_A, TL_B = (1.0, 0.0), (0.5, 0.8660254)


def gen_trans_loc(ref: Reference):
    from oracle import contraction_matrix, convert_params
    d = {"unit_a": np.array(TL_A), "unit_b": np.array(TL_B)}
    cm = contraction_matrix(TL_A, TL_B)
    for tag, (l1, l2, nb, beta, mu0, lam, ns, seed) in TL_CASES.items():
        t, kappa, mu, _ = convert_params(beta, nb, lam=lam, mu0=mu0, static_disorder=True)
        width = (-2 * mu + 8 * np.abs(kappa).sum()) / nb
        ref.set_threads(1)
        g, z, xs, ov = ref.trans_loc_samples(seed, l1, l2, nb, t, kappa, mu, cm, width, ns)
        d.update({f"{tag}_l1": l1, f"{tag}_l2": l2, f"{tag}_nbins": nb, f"{tag}_t": t, f"{tag}_kappa": kappa,
                  f"{tag}_mu": mu, f"{tag}_width": width, f"{tag}_contr_mat": cm, f"{tag}_x": xs,
                  f"{tag}_greens": g, f"{tag}_z": z, f"{tag}_overflow": ov, f"{tag}_seed": seed})
    save("trans_loc.npz", **d)


def gen_conv(ref: Reference):
    """organic_conv's smearing and time transform (simulation/organic_conv.c)
    on two TL histograms: the 8x8 fixture case (128 bins) and a 16x16 lattice
    with 512 bins; widths of the reference's smear.txt (beta = 40, nt = 48)."""
    from oracle import contraction_matrix, convert_params
    d = {}
    g = np.load(os.path.join(HERE, "trans_loc.npz"))
    cm = contraction_matrix(TL_A, TL_B)
    t, kappa, mu, _ = convert_params(40.0, 512, lam=(0.3, 0.15, 0.15), mu0=0.0, static_disorder=True)
    w512 = (-2 * mu + 8 * np.abs(kappa).sum()) / 512
    ref.set_threads(1)
    g512, _, _, _ = ref.trans_loc_samples(11, 16, 16, 512, t, kappa, mu, cm, w512, 2)
    cases = {"L8x8_nb128": (g["L8x8_nb128_greens"] / 2, float(g["L8x8_nb128_width"])),
             "L16x16_nb512": (g512 / 2, w512)}
    beta, nt = 40.0, 48
    widths = np.array([0, 2.7e-3, 6e-3, 1.0]) * beta
    for tag, (sig, h) in cases.items():
        d.update({f"{tag}_sigma": sig, f"{tag}_h": h, f"{tag}_widths": widths, f"{tag}_nt": nt,
                  f"{tag}_w": ref.conv_sigma_w(sig, h, widths), f"{tag}_t": ref.conv_sigma_t(sig, h, widths, nt),
                  f"{tag}_t_matsubara32": ref.conv_sigma_t(sig, h, widths, nt, 32)})
    save("conv.npz", **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-cfg1", action="store_true")
    ap.add_argument("--cfg1-seeds", type=int, default=50)
    ap.add_argument("--only", choices=["trans_loc", "conv"], default=None)
    a = ap.parse_args()
    ref = Reference()
    if a.only == "trans_loc":
        gen_trans_loc(ref)
        return
    if a.only == "conv":
        gen_conv(ref)
        return
    gen_rng_lattice(ref)
    gen_fa(ref)
    gen_evals(ref)
    gen_trans_loc(ref)
    gen_conv(ref)
    if not a.skip_cfg1:
        gen_cfg1(ref, a.cfg1_seeds)


if __name__ == "__main__":
    main()
