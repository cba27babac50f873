"""Python handle for one device context (ephmc_ctx) -- one lattice, one set of
couplings, all work buffers resident on one GPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import MODES, Flags, check, load_library, ptr

ROOM_TEMPERATURE = 0.025  # simulation/organic_main.c:17


def convert_params(beta, nt, J, lam, mu0, omega0, static_disorder=False):
    """Lattice units exactly as organic_main (simulation/organic_main.c:99-116)."""
    x_avg = 1.0 if static_disorder else float(np.sqrt(0.5 / np.tanh(0.5 * omega0 / ROOM_TEMPERATURE)))
    b = -beta if static_disorder else beta / nt
    mu = mu0 * b
    omega = omega0 * b
    t = np.zeros(3)
    kappa = np.zeros(3)
    for k in range(3):
        t[k] = J[k] * b
        kappa[k] = lam[k] * t[k] / x_avg
        mu -= 2 * abs(t[k])
    return t, kappa, float(mu), float(omega)


def lattice(l1, l2):
    """Neighbour table of the periodic triangular lattice (construct_triangular layout)."""
    V = l1 * l2
    nnt = np.empty(12 * V, dtype=np.uint32)
    idx = np.arange(V)
    a, b = idx % l1, idx // l1
    right = b * l1 + (a + 1) % l1
    left = b * l1 + (a + l1 - 1) % l1
    up = ((b + 1) % l2) * l1
    down = ((b + l2 - 1) % l2) * l1
    s = nnt[:6 * V].reshape(V, 6)
    s[:, 0], s[:, 1] = right, left
    s[:, 2], s[:, 3] = up + a, down + a
    s[:, 4], s[:, 5] = up + (a + l1 - 1) % l1, down + (a + 1) % l1
    lk = nnt[6 * V:].reshape(V, 6)
    lk[:, 0], lk[:, 1] = 3 * idx, 3 * s[:, 1]
    lk[:, 2], lk[:, 3] = 3 * idx + 1, 3 * s[:, 3] + 1
    lk[:, 4], lk[:, 5] = 3 * idx + 2, 3 * s[:, 5] + 2
    return nnt


def _flags(flags):
    if flags is None:
        return None
    if isinstance(flags, Flags):
        return flags
    f = Flags()
    names = [n for n, _ in Flags._fields_]
    if isinstance(flags, dict):
        for k, v in flags.items():
            setattr(f, k, v)
    else:
        for n, v in zip(names, flags):
            setattr(f, n, v)
    return f


class Context:
    """One ephmc_ctx.  Buffers passed to methods may be numpy arrays (host:
    staged by the library) or CUDA torch tensors (used in place)."""

    def __init__(self, l1, l2, nt, t, kappa, mu, omega, flavors=1, flags=None, device=0):
        self.lib = load_library()
        self.l1, self.l2, self.nt = int(l1), int(l2), int(nt)
        self.V = self.l1 * self.l2
        self.dim = 3 * self.V * self.nt
        self.flavors = int(flavors)
        self._t = np.ascontiguousarray(t, dtype=np.float64)
        self._k = np.ascontiguousarray(kappa, dtype=np.float64)
        self._flags = _flags(flags)
        h = C.c_void_p()
        st = self.lib.ephmc_ctx_create(C.byref(h), self.l1, self.l2, self.nt, self._t.ctypes.data,
                                       self._k.ctypes.data, float(mu), float(omega), self.flavors,
                                       C.byref(self._flags) if self._flags is not None else None, int(device))
        check(st, "ephmc_ctx_create")
        self.h = h
        self.mu, self.omega = float(mu), float(omega)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ephmc_ctx_destroy(self.h)
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

    # ------------------------------------------------------------ fermion side
    def eval(self, x, p_dot=None, mode="reference"):
        """One force+logdet evaluation; returns (logdet, p_dot)."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        if p_dot is None:
            p_dot = np.empty(self.dim) if isinstance(x, np.ndarray) else None
        ld = C.c_double(0.0)
        check(self.lib.ephmc_eval(self.h, ptr(x), ptr(p_dot), C.byref(ld), m), "ephmc_eval")
        return ld.value, p_dot

    def construct_M_hat(self, x, out=None):
        if out is None:
            out = np.empty((self.V, self.V))
        check(self.lib.ephmc_construct_M_hat(self.h, ptr(x), ptr(out)), "ephmc_construct_M_hat")
        return out

    def logdet_inverse(self, M):
        """In place: M becomes its inverse. Returns (logdet, sign, ipiv 1-based)."""
        ipiv = np.empty(self.V, dtype=np.int32)
        ld, sg = C.c_double(0.0), C.c_int(0)
        check(self.lib.ephmc_logdet_inverse(self.h, ptr(M), ipiv.ctypes.data, C.byref(ld), C.byref(sg)),
              "ephmc_logdet_inverse")
        return ld.value, sg.value, ipiv

    def inverse(self, out=None):
        if out is None:
            out = np.empty((self.V, self.V))
        check(self.lib.ephmc_ctx_get_inverse(self.h, ptr(out)), "ephmc_ctx_get_inverse")
        return out

    def timings(self):
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        check(self.lib.ephmc_ctx_last_timings(self.h, C.byref(a), C.byref(b), C.byref(c)), "timings")
        return a.value, b.value, c.value

    def warnings(self):
        return self.lib.ephmc_last_warnings()

    def leapfrog(self, x, p, steps, traj_length, mode="mixed", graph=False):
        """ephmc_leapfrog (or, with graph=True, ephmc_leapfrog_graph) on device
        tensors x, p (updated in place); returns the number of steps with a
        negative determinant."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        neg = C.c_uint(0)
        fn = self.lib.ephmc_leapfrog_graph if graph else self.lib.ephmc_leapfrog
        check(fn(self.h, ptr(x), ptr(p), int(steps), float(traj_length), m, C.byref(neg)),
              "ephmc_leapfrog_graph" if graph else "ephmc_leapfrog")
        return neg.value

    def set_segment(self, length):
        """Segment length of the mixed force (0: the built-in min(Nt, 16))."""
        check(self.lib.ephmc_ctx_set_segment(self.h, int(length)), "ephmc_ctx_set_segment")

    def set_stabilize(self, on=True):
        """FP64 re-stabilised slice chain for the adjoint and mixed paths."""
        check(self.lib.ephmc_ctx_set_stabilize(self.h, int(bool(on))), "ephmc_ctx_set_stabilize")

    def logdet(self, x, mode="adjoint"):
        """log|det M_hat| alone (ephmc_eval without a force output)."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        ld = C.c_double(0.0)
        check(self.lib.ephmc_eval(self.h, ptr(x), None, C.byref(ld), m), "ephmc_eval")
        return ld.value

    def set_checkpoint(self, interval):
        """Checkpointed adjoint sweeps every `interval` slices (0: whole stack)."""
        check(self.lib.ephmc_ctx_set_checkpoint(self.h, int(interval)), "ephmc_ctx_set_checkpoint")

    def autotune(self, x, mode="mixed"):
        """ephmc_ctx_autotune on field x; returns (ms_before, ms_after, shapes)."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        a, b = C.c_float(0), C.c_float(0)
        check(self.lib.ephmc_ctx_autotune(self.h, ptr(x), m, C.byref(a), C.byref(b)), "ephmc_ctx_autotune")
        out = (C.c_int * 5)()
        check(self.lib.ephmc_ctx_tuning(self.h, out), "ephmc_ctx_tuning")
        return a.value, b.value, list(out)

    def memory(self):
        """Device bytes the context holds."""
        b = C.c_size_t(0)
        check(self.lib.ephmc_ctx_memory(self.h, C.byref(b)), "ephmc_ctx_memory")
        return b.value

    # ------------------------------------------------------------ phonon side
    def fa_evolve(self, x, p, h):
        check(self.lib.ephmc_fa_evolve(self.h, ptr(x), ptr(p), float(h)), "ephmc_fa_evolve")

    def fa_approx_step(self, x, p, h):
        """Kinetic step of classical Fourier acceleration (x in place)."""
        check(self.lib.ephmc_fa_approx_step(self.h, ptr(x), ptr(p), float(h)), "ephmc_fa_approx_step")

    def fa_scale_momenta(self, p):
        check(self.lib.ephmc_fa_scale_momenta(self.h, ptr(p)), "ephmc_fa_scale_momenta")

    def fa_scale_free_bosons(self, x):
        check(self.lib.ephmc_fa_scale_free_bosons(self.h, ptr(x)), "ephmc_fa_scale_free_bosons")

    def fa_energy(self, p):
        e = C.c_double(0.0)
        check(self.lib.ephmc_fa_energy(self.h, ptr(p), C.byref(e)), "ephmc_fa_energy")
        return e.value

    def hamilton(self, x, logdet, energyP):
        H = C.c_double(0.0)
        check(self.lib.ephmc_hamilton(self.h, ptr(x), float(logdet), float(energyP), C.byref(H)), "ephmc_hamilton")
        return H.value


def batch_eval(contexts, xs, p_dots=None, mode="mixed"):
    """ephmc_batch_eval: one force+logdet evaluation of every chain (context
    i on field xs[i]), all chains issued before any host wait.  xs and
    p_dots: numpy arrays or CUDA tensors; p_dots defaults to new host arrays
    for host fields (None entries for device fields).  Returns (logdets,
    p_dots)."""
    lib = load_library()
    n = len(contexts)
    m = MODES[mode] if isinstance(mode, str) else int(mode)
    if p_dots is None:
        p_dots = [np.empty(c.dim) if isinstance(x, np.ndarray) else None for c, x in zip(contexts, xs)]
    hs = (C.c_void_p * n)(*[c.h.value if isinstance(c.h, C.c_void_p) else c.h for c in contexts])
    xp = (C.c_void_p * n)(*[ptr(x) for x in xs])
    pp = (C.c_void_p * n)(*[ptr(p) if p is not None else None for p in p_dots])
    ld = (C.c_double * n)()
    check(lib.ephmc_batch_eval(hs, xp, pp, ld, n, m), "ephmc_batch_eval")
    return np.array(ld[:]), p_dots
