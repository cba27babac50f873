"""organic_conv on the GPU (ephmc_conv_sigma_w / ephmc_conv_sigma_t and the
organic_conv program built over them) against the reference's own
smeared_sigma_w / smeared_sigma_t (simulation/organic_conv.c:92-121) and its
program (:123-164).  The GPU sums run in the reference's order; the
differences come from the device's exp/sinh/cosh/tanh (a few ulp), so the
tolerance is 1e-12 relative."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import PKG, golden

pytestmark = pytest.mark.gpu

CASES = ["L8x8_nb128", "L16x16_nb512"]


@pytest.mark.parametrize("tag", CASES)
def test_conv_matches_reference_fixture(gpu, tag):
    import ephmc
    g = golden("conv.npz")
    sig, h, wd, nt = g[f"{tag}_sigma"], float(g[f"{tag}_h"]), g[f"{tag}_widths"], int(g[f"{tag}_nt"])
    w = ephmc.conv_sigma_w(sig, h, wd)
    t = ephmc.conv_sigma_t(sig, h, wd, nt)
    tm = ephmc.conv_sigma_t(sig, h, wd, nt, 32)
    for name, a, r in (("sigma_w", w, g[f"{tag}_w"]), ("sigma_t", t, g[f"{tag}_t"]),
                       ("sigma_t Matsubara", tm, g[f"{tag}_t_matsubara32"])):
        rel = np.max(np.abs(a - r) / np.maximum(np.abs(r), 1e-300))
        print(f"{tag} {name}: {rel:.2e}")
        assert rel <= 1e-12, (name, rel)


def test_conv_device_buffers_and_errors(gpu):
    import ctypes as C

    import torch

    import ephmc
    lib = ephmc.load_library()
    g = golden("conv.npz")
    tag = "L8x8_nb128"
    sig = torch.from_numpy(g[f"{tag}_sigma"]).cuda()
    wd = torch.from_numpy(g[f"{tag}_widths"]).cuda()
    out = torch.empty(128 * 4, dtype=torch.float64, device="cuda")
    h = float(g[f"{tag}_h"])
    assert lib.ephmc_conv_sigma_w(sig.data_ptr(), 128, h, wd.data_ptr(), 4, out.data_ptr()) == 0
    assert np.allclose(out.cpu().numpy().reshape(128, 4), g[f"{tag}_w"], rtol=1e-12, atol=0)
    assert lib.ephmc_conv_sigma_w(sig.data_ptr(), 128, 0.0, wd.data_ptr(), 4, out.data_ptr()) == 2
    assert lib.ephmc_conv_sigma_t(sig.data_ptr(), 128, h, wd.data_ptr(), 4, 0, 0, out.data_ptr()) == 2
    assert b"arguments" in lib.ephmc_last_error_message()
    del C


def _write_greens(path, sigma, h):
    with open(path, "wb") as f:
        f.write(np.uint32(len(sigma)).tobytes())
        f.write(np.float64(h).tobytes())
        f.write(np.ascontiguousarray(sigma, dtype=np.float64).tobytes())


def _read_csv(path):
    rows = [r for r in open(path).read().strip().split("\n") if r.strip()]
    return np.array([[float(v) for v in r.split()] for r in rows])


def test_organic_conv_program_against_reference_program(gpu, reference):
    """The command-line program (greens.bin, smear.txt -> greens_smeared.csv,
    corr_smeared.csv) against the reference's organic_conv on the same files,
    with the reference's smear.txt contents (beta 40, nt 48, widths 0,
    2.7e-3, 6e-3, 1).  Both print %g (6 significant digits): values agree to
    that precision."""
    exe = os.path.join(PKG, "lib", "organic_conv")
    assert os.path.exists(exe), "organic_conv program not built (electron-phonon-hmc_b200/build.py)"
    g = golden("conv.npz")
    tag = "L16x16_nb512"
    with tempfile.TemporaryDirectory() as d:
        gb, sm = os.path.join(d, "greens.bin"), os.path.join(d, "smear.txt")
        _write_greens(gb, g[f"{tag}_sigma"], float(g[f"{tag}_h"]))
        open(sm, "w").write("40 48\n0\n2.7e-3\n6e-3\n1\n")
        rw, rt = os.path.join(d, "ref_w.csv"), os.path.join(d, "ref_t.csv")
        gw, gt = os.path.join(d, "gpu_w.csv"), os.path.join(d, "gpu_t.csv")
        reference.run_conv(gb, sm, rw, rt)
        out = subprocess.run([exe, gb, sm, gw, gt], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        a, b = _read_csv(rw), _read_csv(gw)
        at, bt = _read_csv(rt), _read_csv(gt)
    assert a.shape == b.shape == (512, 5) and at.shape == bt.shape == (25, 5)
    assert np.allclose(b, a, rtol=1e-5, atol=1e-300)
    assert np.allclose(bt, at, rtol=1e-5, atol=1e-300)


def test_conv_unsmeared_width_only(gpu):
    """Width 0 alone (the histogram read back bin by bin, organic_conv.c:97-101)
    and the t = 1/2 end point, against the restatement."""
    import ephmc
    from oracle import conv_sigma_t, conv_sigma_w
    g = golden("conv.npz")
    sig, h = g["L8x8_nb128_sigma"], float(g["L8x8_nb128_h"])
    w = ephmc.conv_sigma_w(sig, h, [0.0])
    assert np.allclose(w, conv_sigma_w(sig, h, [0.0]), rtol=1e-13, atol=0)
    t = ephmc.conv_sigma_t(sig, h, [0.0, 5.0], 2)
    r = conv_sigma_t(sig, h, [0.0, 5.0], 2)
    assert t.shape == (2, 2) and np.allclose(t, r, rtol=1e-12, atol=0)
