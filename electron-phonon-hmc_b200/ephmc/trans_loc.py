"""Python handle for the static-disorder (transient localisation) histograms,
the GPU form of hist_trans_loc / run_trans_loc
(simulation/organic_trans_loc.c:25-114), over ephmc_tl_* of libephmc_cuda.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load_library, ptr


def conv_sigma_w(sigma, h, widths):
    """Smeared conductivity of organic_conv (simulation/organic_conv.c:92-111)
    at every bin's frequency: [n][len(widths)] (ephmc_conv_sigma_w)."""
    lib = load_library()
    sg = np.ascontiguousarray(sigma, dtype=np.float64)
    wd = np.ascontiguousarray(widths, dtype=np.float64)
    out = np.empty((len(sg), len(wd)))
    check(lib.ephmc_conv_sigma_w(sg.ctypes.data, len(sg), float(h), wd.ctypes.data, len(wd), out.ctypes.data),
          "ephmc_conv_sigma_w")
    return out


def conv_sigma_t(sigma, h, widths, nt, nt_matsubara=0):
    """Euclidean-time transform of organic_conv (:113-121) at t = i/nt,
    i <= nt/2: [nt/2+1][len(widths)] (ephmc_conv_sigma_t)."""
    lib = load_library()
    sg = np.ascontiguousarray(sigma, dtype=np.float64)
    wd = np.ascontiguousarray(widths, dtype=np.float64)
    out = np.empty((nt // 2 + 1, len(wd)))
    check(lib.ephmc_conv_sigma_t(sg.ctypes.data, len(sg), float(h), wd.ctypes.data, len(wd), int(nt),
                                 int(nt_matsubara), out.ctypes.data), "ephmc_conv_sigma_t")
    return out


def contraction_matrix(a, b):
    """construct_contraction_mat (simulation/organic_lattice.c:48-60) for the
    triangular lattice: rows c = 0, 1 (Cartesian), columns k = right, top
    right, top left."""
    m = np.empty(6)
    for c in range(2):
        m[3 * c] = a[c]
        m[3 * c + 1] = .5 * (a[c] + b[c])
        m[3 * c + 2] = .5 * (-a[c] + b[c])
    return m


class TransLoc:
    """One ephmc_tl handle: a lattice, nbins frequency bins and the couplings
    as run_trans_loc receives them.  ``lanes`` samples run concurrently."""

    def __init__(self, l1, l2, nbins, t, kappa, mu, contr_mat, lanes=1, device=0):
        self.lib = load_library()
        self.l1, self.l2, self.nbins = int(l1), int(l2), int(nbins)
        self.V = self.l1 * self.l2
        self.dim = 3 * self.V
        self._t = np.ascontiguousarray(t, dtype=np.float64)
        self._k = np.ascontiguousarray(kappa, dtype=np.float64)
        self._m = np.ascontiguousarray(contr_mat, dtype=np.float64)
        h = C.c_void_p()
        check(self.lib.ephmc_tl_create(C.byref(h), self.l1, self.l2, self.nbins, self._t.ctypes.data,
                                       self._k.ctypes.data, float(mu), self._m.ctypes.data, int(lanes), int(device)),
              "ephmc_tl_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ephmc_tl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream):
        check(self.lib.ephmc_tl_set_stream(self.h, C.c_void_p(int(stream))), "ephmc_tl_set_stream")

    def default_width(self):
        w = C.c_double(0.0)
        check(self.lib.ephmc_tl_default_width(self.h, C.byref(w)), "ephmc_tl_default_width")
        return w.value

    def run(self, x, width=None, hist=None, z=None):
        """Samples x[n][3V] (numpy or CUDA tensor): hist += the summed sample
        histograms, z[n] = partition sums / V.  Returns (hist, z)."""
        n = int(x.shape[0]) if x.ndim == 2 else 1
        if width is None:
            width = self.default_width()
        if hist is None:
            hist = np.zeros(self.nbins)
        if z is None and isinstance(x, np.ndarray):
            z = np.empty(n)
        check(self.lib.ephmc_tl_run(self.h, ptr(x), n, float(width), ptr(hist), ptr(z)), "ephmc_tl_run")
        return hist, z

    def last_timings(self):
        """Device ms of lane 0's first sample of the last run: Hamiltonian,
        eigensolver, current operators, products, binning."""
        ms = (C.c_float * 5)()
        check(self.lib.ephmc_tl_last_timings(self.h, ms), "ephmc_tl_last_timings")
        return list(ms)
