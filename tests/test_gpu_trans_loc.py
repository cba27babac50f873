"""Static-disorder (transient localisation) mode on the GPU against the
reference: hist_trans_loc / run_trans_loc (simulation/organic_trans_loc.c:25-114).

Tolerances: the reference diagonalises with LAPACK dsyev, the GPU path with
cuSOLVER dsyevd, and the matrix elements are summed in other orders.  Every
binned quantity is quadratic in each eigenvector and summed over whole
(near-)degenerate groups, so it does not depend on the eigensolver's basis
choice.  The histograms agree to about 1e-13 of the largest bin; the tests
allow 1e-10.  Disorder is always on: an exactly degenerate spectrum makes the
reference's bin 0 depend on eigenvalue rounding (see
test_trans_loc_degenerate_spectrum_is_ill_posed_in_the_reference)."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ORACLE, golden

pytestmark = pytest.mark.gpu

TL_CASES = ["L6x5_nb64", "L8x8_nb128", "L5x7_nb32_beta10", "L6x6_nb64_mu-3"]


def _case(g, tag):
    return dict(l1=int(g[f"{tag}_l1"]), l2=int(g[f"{tag}_l2"]), nbins=int(g[f"{tag}_nbins"]), t=g[f"{tag}_t"],
                kappa=g[f"{tag}_kappa"], mu=float(g[f"{tag}_mu"]), contr_mat=g[f"{tag}_contr_mat"])


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("tag", TL_CASES)
def test_tl_matches_reference_fixture(gpu, tag):
    """Histogram and partition sums of the reference's own samples (its bond
    fields, tests/golden/trans_loc.npz), one sample per call and all samples
    in one call."""
    import ephmc
    g = golden("trans_loc.npz")
    c = _case(g, tag)
    xs = np.ascontiguousarray(g[f"{tag}_x"])
    width = float(g[f"{tag}_width"])
    with ephmc.TransLoc(**c) as tl:
        assert tl.default_width() == width
        h1 = np.zeros(c["nbins"])
        z1 = [tl.run(x[None, :].copy(), width, hist=h1)[1][0] for x in xs]
        hb, zb = tl.run(xs, width)
    ref, zr = g[f"{tag}_greens"], g[f"{tag}_z"]
    for h, z in ((h1, np.array(z1)), (hb, zb)):
        assert _rel(h, ref) <= 1e-10, f"{tag}: histogram {_rel(h, ref):.2e}"
        assert np.allclose(z, zr, rtol=1e-12, atol=0), f"{tag}: partition sums {np.max(np.abs(z / zr - 1)):.2e}"


def test_tl_lanes_streams_and_device_buffers(gpu):
    """Five samples on three concurrent lanes, with bond fields, histogram and
    partition sums in device memory and a caller stream, against one lane on
    host buffers: the same results up to the order of the atomic sums."""
    import torch

    import ephmc
    g = golden("trans_loc.npz")
    tag = "L8x8_nb128"
    c = _case(g, tag)
    rng = np.random.default_rng(3)
    xs = rng.standard_normal((5, 3 * c["l1"] * c["l2"]))
    with ephmc.TransLoc(**c, lanes=1) as a:
        width = a.default_width()
        ha, za = a.run(xs, width)
    with ephmc.TransLoc(**c, lanes=3) as b:
        s = torch.cuda.Stream()
        b.set_stream(s.cuda_stream)
        xd = torch.from_numpy(xs).cuda()
        hd = torch.full((c["nbins"],), 0.5, dtype=torch.float64, device="cuda")  # accumulates on top
        zd = torch.zeros(5, dtype=torch.float64, device="cuda")
        b.run(xd, width, hd, zd)
        s.synchronize()
        hb, zb = hd.cpu().numpy() - 0.5, zd.cpu().numpy()
    assert _rel(hb, ha) <= 1e-12
    assert np.allclose(zb, za, rtol=1e-14, atol=0)


def test_tl_larger_lattice_matches_restatement(gpu):
    """32 x 32 sites (V = 1024, the HMC workload's lattice), 512 bins, beta =
    40, one sample, against the numpy restatement of hist_trans_loc (pinned to
    the reference by the CPU tests)."""
    import ephmc
    from oracle import contraction_matrix, convert_params, trans_loc_sample
    t, kappa, mu, _ = convert_params(40.0, 512, mu0=0.0, static_disorder=True)
    cm = contraction_matrix((1.0, 0.0), (0.5, 0.8660254))
    x = np.random.default_rng(5).standard_normal(3 * 1024)
    with ephmc.TransLoc(32, 32, 512, t, kappa, mu, cm) as tl:
        width = tl.default_width()
        h, z = tl.run(x[None, :].copy(), width)
    r, zr = trans_loc_sample(x, 32, 32, 512, t, kappa, mu, cm, width)
    print(f"32x32, 512 bins: histogram {_rel(h, r):.2e}, Z {abs(z[0] / zr - 1):.2e}")
    assert _rel(h, r) <= 1e-10
    assert abs(z[0] / zr - 1) <= 1e-12


def test_tl_argument_errors(gpu):
    """A missing contraction matrix (the reference dereferences it), a zero
    width and a missing histogram are rejected with EPHMC_ERR_ARG and a
    message; the handle stays usable."""
    import ephmc
    lib = ephmc.load_library()
    t = np.array([-40.0, 20.0, 20.0])
    k = np.array([-12.0, 3.0, 3.0])
    h = C.c_void_p()
    st = lib.ephmc_tl_create(C.byref(h), 4, 4, 16, t.ctypes.data, k.ctypes.data, -40.0, None, 1, 0)
    assert st == 2 and b"contraction matrix" in lib.ephmc_last_error_message()
    assert not h.value
    cm = np.array([1.0, 0.75, -0.25, 0.0, 0.4330127, 0.4330127])
    with ephmc.TransLoc(4, 4, 16, t, k, -40.0, cm) as tl:
        x = np.zeros((1, 48))
        hist = np.zeros(16)
        z = np.zeros(1)
        assert lib.ephmc_tl_run(tl.h, x.ctypes.data, 1, 0.0, hist.ctypes.data, z.ctypes.data) == 2
        assert lib.ephmc_tl_run(tl.h, x.ctypes.data, 1, 1.0, None, z.ctypes.data) == 2
        tl.run(x, 1.0, hist, z)
        # x = 0: the clean lattice, whose partition sum is that of the hopping band
        assert z[0] > 0 and np.isfinite(hist).all()


INPUT_TL = """6 6
64
40
1 -0.5 -0.5
0.3 0.15 0.15
0
0.05
5 0
0
4 1
1 0
0.5 0.8660254
1
STATIC_DISORDER
"""


def _read_sigma(path):
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], dtype=np.uint32)[0])
    width = float(np.frombuffer(raw[4:12], dtype=np.float64)[0])
    return n, width, np.frombuffer(raw[12:], dtype=np.float64)


def test_reference_organic_main_static_disorder(gpu, reference):
    """The reference's organic_main.c with STATIC_DISORDER linked to the GPU
    library (run_trans_loc and hist_trans_loc from libephmc_cuda.so) against
    the reference program on the same MT19937-64 seed: the same partition sum
    per sample in results.csv (1e-12), the same greens.bin header (bins and
    width, bit for bit) and histogram (1e-10 of the largest bin)."""
    exe = os.path.join(ORACLE, "_ref", "organic_main_ephmc")
    if not os.path.exists(exe):
        pytest.skip("drop-in program not built (make -C oracle dropin)")
    with tempfile.TemporaryDirectory() as d:
        inp = os.path.join(d, "input.txt")
        open(inp, "w").write(INPUT_TL)
        r_res, r_sig = os.path.join(d, "ref_res.csv"), os.path.join(d, "ref_sigma.bin")
        g_res, g_sig = os.path.join(d, "gpu_res.csv"), os.path.join(d, "gpu_sigma.bin")
        reference.set_threads(1)
        reference.run_main(13, inp, r_res, r_sig)
        env = dict(os.environ, EPHMC_SEED="13", EPHMC_TL_LANES="2")
        out = subprocess.run([exe, inp, g_res, g_sig], env=env, capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr
        assert "ERROR" not in out.stdout, out.stdout
        zr = np.loadtxt(r_res)
        zg = np.loadtxt(g_res)
        nr, wr, hr = _read_sigma(r_sig)
        ng, wg, hg = _read_sigma(g_sig)
    assert zr.shape == zg.shape == (4,)
    assert np.allclose(zg, zr, rtol=1e-12, atol=0)
    assert (ng, wg) == (nr, wr) == (64, wr)
    assert _rel(hg, hr) <= 1e-10


def test_tl_many_bins_and_odd_lattice(gpu):
    """Histograms past the shared-memory limit (12 000 bins: the binning
    kernel's global-atomic variant) and a 7x5 lattice with 5 samples on 3
    lanes, against the numpy restatement."""
    import ephmc
    from oracle import contraction_matrix, convert_params, trans_loc_sample
    cm = contraction_matrix((1.0, 0.0), (0.5, 0.8660254))
    rng = np.random.default_rng(21)
    for (l1, l2, nbins, lanes, ns) in ((6, 6, 12000, 1, 2), (7, 5, 48, 3, 5)):
        t, kappa, mu, _ = convert_params(20.0, nbins, mu0=0.0, static_disorder=True)
        xs = rng.standard_normal((ns, 3 * l1 * l2))
        with ephmc.TransLoc(l1, l2, nbins, t, kappa, mu, cm, lanes=lanes) as tl:
            w = tl.default_width()
            h, z = tl.run(xs, w)
        ref = np.zeros(nbins)
        zr = []
        for x in xs:
            hs, zs = trans_loc_sample(x, l1, l2, nbins, t, kappa, mu, cm, w)
            ref += hs
            zr.append(zs)
        assert _rel(h, ref) <= 1e-10, (l1, l2, nbins, _rel(h, ref))
        assert np.allclose(z, zr, rtol=1e-12, atol=0)
