"""ctypes access to the two CPU oracles -- TEST INFRASTRUCTURE ONLY.

* ``Restated``  -> ``oracle/liboracle.so``: the project's plain-C restatement of
  the hot path (``oracle/ephmc_oracle.c``), no third-party dependencies.
* ``Reference`` -> ``oracle/_ref/libephref.so``: the reference's own C sources
  compiled unmodified (``oracle/Makefile``), the pin for the restatement and the
  timed CPU baseline.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm import this module, as the checker.  The product path never
does.  Both libraries are built by ``make -C oracle`` (``build()`` in
``__graft_entry__.py`` runs it).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_SO = os.path.join(HERE, "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libephref.so")

_D, _U, _P, _I = C.c_double, C.c_uint, C.c_void_p, C.c_int

# couplings of the benchmark workloads in physical units (organic_main input.txt
# semantics): J, lambda, mu0, omega0
J_DEFAULT = (1.0, -0.5, -0.5)
LAMBDA_DEFAULT = (0.3, 0.15, 0.15)
MU0_DEFAULT = -3.0
OMEGA0_DEFAULT = 0.05


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def convert_params(beta, nt, J=J_DEFAULT, lam=LAMBDA_DEFAULT, mu0=MU0_DEFAULT,
                   omega0=OMEGA0_DEFAULT, static_disorder=False):
    """Lattice-unit parameters exactly as organic_main (simulation/organic_main.c:99-116)."""
    x_avg = 1.0 if static_disorder else float(np.sqrt(0.5 / np.tanh(0.5 * omega0 / 0.025)))
    b = -beta if static_disorder else beta / nt
    mu = mu0 * b
    omega = omega0 * b
    t = [0.0, 0.0, 0.0]
    kappa = [0.0, 0.0, 0.0]
    for k in range(3):
        t[k] = J[k] * b
        kappa[k] = lam[k] * t[k] / x_avg
        mu -= 2 * abs(t[k])
    return np.array(t), np.array(kappa), float(mu), float(omega)


@dataclass
class Model:
    """One parameter point of the path: lattice, slices and lattice-unit couplings."""
    l1: int
    l2: int
    nt: int
    t: np.ndarray
    kappa: np.ndarray
    mu: float
    omega: float
    flavors: int = 1
    flags: tuple = (0, 0, 0, 0, 0, 0, 0)
    beta: float = field(default=float("nan"))

    @property
    def ns(self):
        return self.l1 * self.l2

    @property
    def dim(self):
        return 3 * self.ns * self.nt

    @classmethod
    def physical(cls, L1, L2, nt, beta, J=J_DEFAULT, lam=LAMBDA_DEFAULT,
                 mu0=MU0_DEFAULT, omega0=OMEGA0_DEFAULT, flavors=1, flags=(0,) * 7):
        t, kappa, mu, omega = convert_params(beta, nt, J, lam, mu0, omega0)
        return cls(L1, L2, nt, t, kappa, mu, omega, flavors, tuple(flags), beta)


class _Lib:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: run `make -C oracle`")
        self.lib = C.CDLL(path)

    def _sig(self, name, res, args):
        f = getattr(self.lib, name)
        f.restype = res
        f.argtypes = args
        return f


class Restated(_Lib):
    """The project's C restatement (oracle/ephmc_oracle.c)."""

    def __init__(self, path=RESTATED_SO):
        super().__init__(path)
        s = self._sig
        s("or_mt_seed", None, [C.c_ulonglong])
        s("or_mt_real2", _D, [])
        s("or_normals", None, [_P, _U])
        s("or_lattice", None, [_U, _U, _P])
        s("or_model_new", _P, [_U, _U, _U, _P, _P, _D, _D, _U, _P])
        s("or_model_free", None, [_P])
        s("or_apply_mu_K_v", None, [_P, _P, _P, _P])
        s("or_apply_exp_M", None, [_P, _P, _P, _I, _I])
        s("or_construct_M_hat", None, [_P, _P, _P])
        s("or_logdet_inverse", _D, [_P, _U, C.POINTER(C.c_int)])
        s("or_all_G", None, [_P, _P, _P, _P])
        s("or_refine", None, [_P, _P, _P, _U])
        s("or_eval_reference", _D, [_P, _P, _P, _P, C.POINTER(C.c_int)])
        s("or_eval_adjoint", _D, [_P, _P, _P, _I])
        s("or_hamilton", _D, [_P, _D, _D, _D, _U, _U, _U])
        s("or_check_force", _D, [_P, _P, _P])
        s("or_rdft_forward", None, [_P, _P, _U, _U])
        s("or_rdft_inverse", None, [_P, _P, _U, _U])
        s("or_evolve_bosons", None, [_P, _P, _D, _U, _U, _D])
        s("or_sample_fourier_momenta", None, [_P, _D, _U, _U])
        s("or_energy_fourier_momenta", _D, [_P, _D, _U, _U])
        s("or_sample_free_bosons", None, [_P, _D, _U, _U])
        s("or_higher_matsubaras_norm", _D, [_P, _U, _U])

    # -- RNG / lattice
    def random_x(self, seed, n):
        x = np.empty(n)
        self.lib.or_mt_seed(seed)
        self.lib.or_normals(_ptr(x), n)
        return x

    def lattice(self, l1, l2):
        nnt = np.empty(12 * l1 * l2, dtype=np.uint32)
        self.lib.or_lattice(l1, l2, _ptr(nnt))
        return nnt

    # -- model handle
    def _model(self, m: Model):
        t = np.ascontiguousarray(m.t, dtype=np.float64)
        k = np.ascontiguousarray(m.kappa, dtype=np.float64)
        f = np.ascontiguousarray(m.flags, dtype=np.int32)
        return self.lib.or_model_new(m.l1, m.l2, m.nt, _ptr(t), _ptr(k), m.mu, m.omega, m.flavors, _ptr(f))

    def construct_M_hat(self, m: Model, x):
        h = self._model(m)
        M = np.empty((m.ns, m.ns))
        self.lib.or_construct_M_hat(h, _ptr(np.ascontiguousarray(x)), _ptr(M))
        self.lib.or_model_free(h)
        return M

    def apply_mu_K_v(self, m: Model, x_slice, v):
        h = self._model(m)
        w = np.empty(m.ns)
        self.lib.or_apply_mu_K_v(h, _ptr(np.ascontiguousarray(x_slice)), _ptr(np.ascontiguousarray(v)), _ptr(w))
        self.lib.or_model_free(h)
        return w

    def logdet_inverse(self, M):
        A = np.array(M, dtype=np.float64, order="C", copy=True)
        sign = C.c_int(0)
        ld = self.lib.or_logdet_inverse(_ptr(A), A.shape[0], C.byref(sign))
        return ld, sign.value, A

    def eval_reference(self, m: Model, x):
        h = self._model(m)
        pd = np.empty(m.dim)
        Mi = np.empty((m.ns, m.ns))
        sign = C.c_int(0)
        ld = self.lib.or_eval_reference(h, _ptr(np.ascontiguousarray(x)), _ptr(pd), _ptr(Mi), C.byref(sign))
        self.lib.or_model_free(h)
        return ld, pd, Mi, sign.value

    def eval_adjoint(self, m: Model, x, single=False):
        h = self._model(m)
        pd = np.empty(m.dim)
        ld = self.lib.or_eval_adjoint(h, _ptr(np.ascontiguousarray(x)), _ptr(pd), int(single))
        self.lib.or_model_free(h)
        return ld, pd

    def all_G(self, m: Model, x, M_inv):
        h = self._model(m)
        G = np.empty((m.nt, m.ns, m.ns))
        self.lib.or_all_G(h, _ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(M_inv)), _ptr(G))
        self.lib.or_model_free(h)
        return G

    def refine(self, m: Model, x, G_t, t):
        h = self._model(m)
        G = np.array(G_t, dtype=np.float64, order="C", copy=True)
        self.lib.or_refine(h, _ptr(np.ascontiguousarray(x)), _ptr(G), t)
        self.lib.or_model_free(h)
        return G

    def hamilton(self, x, logdet, energyP, omega, flavors, ns, nt):
        return self.lib.or_hamilton(_ptr(np.ascontiguousarray(x)), logdet, energyP, omega, flavors, ns, nt)

    def check_force(self, m: Model, x, p_dot):
        h = self._model(m)
        r = self.lib.or_check_force(h, _ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(p_dot)))
        self.lib.or_model_free(h)
        return r

    # -- Fourier acceleration
    def evolve_bosons(self, x, p, omega, ns, nt, h):
        x = np.array(x, dtype=np.float64, copy=True)
        p = np.array(p, dtype=np.float64, copy=True)
        self.lib.or_evolve_bosons(_ptr(x), _ptr(p), omega, ns, nt, h)
        return x, p

    def sample_fourier_momenta(self, seed, omega, ns, nt):
        self.lib.or_mt_seed(seed)
        p = np.empty(3 * ns * nt)
        self.lib.or_sample_fourier_momenta(_ptr(p), omega, ns, nt)
        return p

    def energy_fourier_momenta(self, p, omega, ns, nt):
        return self.lib.or_energy_fourier_momenta(_ptr(np.ascontiguousarray(p)), omega, ns, nt)

    def sample_free_bosons(self, seed, omega, ns, nt):
        self.lib.or_mt_seed(seed)
        x = np.empty(3 * ns * nt)
        self.lib.or_sample_free_bosons(_ptr(x), omega, ns, nt)
        return x

    def higher_matsubaras_norm(self, x, ns, nt):
        return self.lib.or_higher_matsubaras_norm(_ptr(np.ascontiguousarray(x)), ns, nt)

    def rdft_forward(self, x, ld, nt):
        Xc = np.empty((nt // 2 + 1) * ld * 2)
        self.lib.or_rdft_forward(_ptr(np.ascontiguousarray(x)), _ptr(Xc), ld, nt)
        return Xc


class Reference(_Lib):
    """The reference's own C code compiled unmodified (oracle/_ref/libephref.so)."""

    def __init__(self, path=REFERENCE_SO):
        super().__init__(path)
        s = self._sig
        s("ref_init", None, [])
        s("ref_set_threads", None, [_I])
        s("ref_max_threads", _I, [])
        s("ref_set_seed_time", None, [C.c_ulong])
        s("ref_init_genrand64", None, [C.c_ulong])
        s("ref_genrand64_real2", _D, [])
        s("ref_random_vector", None, [C.c_ulong, _P, _U])
        s("ref_lattice", None, [_U, _U, _P, C.POINTER(C.c_uint), C.POINTER(C.c_uint)])
        s("ref_ctx_new", _P, [_U, _U, _U, _P, _P, _D, _D, _U, _P])
        s("ref_ctx_free", None, [_P])
        s("ref_ctx_eval", _D, [_P, _P, _P, _P, _P])
        s("ref_ctx_last_time", _D, [_P])
        s("ref_ctx_construct_M_hat", None, [_P, _P, _P])
        s("ref_ctx_apply_exp", None, [_P, _P, _P, _I, _I])
        s("ref_ctx_apply_mu_K_v", None, [_P, _P, _P, _P])
        s("ref_ctx_all_QM1P", None, [_P, _P, _P, _P])
        s("ref_ctx_refine", None, [_P, _P, _P, _I])
        s("ref_ctx_logdet_inv", _D, [_P, _P])
        s("ref_hamilton", _D, [_P, _D, _D, _D, _U, _U, _U])
        s("ref_ctx_check_force", _D, [_P, _P, _P])
        s("ref_fa_new", _P, [_U, _U])
        s("ref_fa_free", None, [_P])
        s("ref_fa_set", None, [_P, _P, _P])
        s("ref_fa_get", None, [_P, _P, _P])
        s("ref_fa_evolve", None, [_P, _D, _D])
        s("ref_fa_sample_momenta", None, [_P, _D, _P])
        s("ref_fa_energy", _D, [_P, _D])
        s("ref_fa_sample_free", None, [_P, _D])
        s("ref_fa_approx_step", None, [_P, _D, _D, _D])
        s("ref_fa_update_x", None, [_P, _P, _D, _D, _D, _P, _U, _D])
        s("ref_higher_matsubaras_norm", _D, [_P, _U, _U])
        s("ref_boson_force", None, [_P, _P, _D, _U, _U, _I])
        s("ref_run_main", _I, [C.c_ulong, C.c_char_p, C.c_char_p, C.c_char_p])
        s("ref_ctx_cc_correlator", None, [_P, _P, _P, _D, _P])
        s("ref_trans_loc_samples", _I, [C.c_ulong, _U, _U, _U, _P, _P, _D, _P, _D, _U, _P, _P, _P])
        s("ref_run_trans_loc", _U, [C.c_ulong, _U, _U, _U, _P, _P, _D, _P, _U, C.c_char_p, C.c_char_p, _P])
        s("smeared_sigma_w", _D, [_D, _P, _D, _D, _U])
        s("smeared_sigma_t", _D, [_D, _P, _D, _D, _U, _U])
        s("ref_run_conv", _I, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p])
        self.lib.ref_init()

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def random_x(self, seed, n):
        x = np.empty(n)
        self.lib.ref_random_vector(seed, _ptr(x), n)
        return x

    def uniforms(self, seed, n):
        self.lib.ref_init_genrand64(seed)
        return np.array([self.lib.ref_genrand64_real2() for _ in range(n)])

    def lattice(self, l1, l2):
        nnt = np.empty(12 * l1 * l2, dtype=np.uint32)
        ns, nn = C.c_uint(), C.c_uint()
        self.lib.ref_lattice(l1, l2, _ptr(nnt), C.byref(ns), C.byref(nn))
        return nnt

    def trans_loc_samples(self, seed, l1, l2, nbins, t, kappa, mu, contr_mat, width, nsamples):
        """hist_trans_loc x nsamples on the stream seeded with `seed`
        (simulation/organic_trans_loc.c:25-83, 102-103).  Returns (greens
        summed over samples, z per sample, bond fields [nsamples][3V], whether
        a bin past the end was written)."""
        g = np.zeros(nbins)
        z = np.empty(nsamples)
        xs = np.empty((nsamples, 3 * l1 * l2))
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        t, kappa, contr_mat = f64(t), f64(kappa), f64(contr_mat)
        ov = self.lib.ref_trans_loc_samples(seed, l1, l2, nbins, _ptr(t), _ptr(kappa), mu, _ptr(contr_mat), width,
                                            nsamples, _ptr(g), _ptr(z), _ptr(xs))
        return g, z, xs, bool(ov)

    def conv_sigma_w(self, sigma, h, widths):
        """smeared_sigma_w (simulation/organic_conv.c:92-111) at omega = i h for
        every bin i and width: [n][len(widths)]."""
        sg = np.ascontiguousarray(sigma, dtype=np.float64)
        n = len(sg)
        return np.array([[self.lib.smeared_sigma_w(i * h, _ptr(sg), w, h, n) for w in widths] for i in range(n)])

    def conv_sigma_t(self, sigma, h, widths, nt, nt_matsubara=0):
        """smeared_sigma_t (:113-121) at t = i / nt, i <= nt/2: [nt/2+1][len(widths)]."""
        sg = np.ascontiguousarray(sigma, dtype=np.float64)
        n = len(sg)
        return np.array([[self.lib.smeared_sigma_t(i / nt, _ptr(sg), w, h, n, nt_matsubara) for w in widths]
                         for i in range(nt // 2 + 1)])

    def run_conv(self, greens, smear, out_w, out_t=None):
        """organic_conv's main (simulation/organic_conv.c:123-164)."""
        return self.lib.ref_run_conv(greens.encode(), smear.encode(), out_w.encode(),
                                     out_t.encode() if out_t else None)

    def run_trans_loc(self, seed, l1, l2, nbins, t, kappa, mu, contr_mat, meas, res_name, corr_name):
        """run_trans_loc (simulation/organic_trans_loc.c:85-114), time(NULL) = seed."""
        g = np.zeros(nbins + meas)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        t, kappa, contr_mat = f64(t), f64(kappa), f64(contr_mat)
        n = self.lib.ref_run_trans_loc(seed, l1, l2, nbins, _ptr(t), _ptr(kappa), mu, _ptr(contr_mat), meas,
                                       res_name.encode() if res_name else None,
                                       corr_name.encode() if corr_name else None, _ptr(g))
        return g, n

    def context(self, m: Model):
        return RefContext(self, m)

    def hamilton(self, x, logdet, energyP, omega, flavors, ns, nt):
        return self.lib.ref_hamilton(_ptr(np.ascontiguousarray(x)), logdet, energyP, omega, flavors, ns, nt)

    def fa(self, ns, nt):
        return RefFA(self, ns, nt)

    def higher_matsubaras_norm(self, x, ns, nt):
        return self.lib.ref_higher_matsubaras_norm(_ptr(np.ascontiguousarray(x)), ns, nt)

    def run_main(self, seed, input_path, res_path, corr_path=None):
        return self.lib.ref_run_main(seed, input_path.encode(), res_path.encode(),
                                     corr_path.encode() if corr_path else None)


class RefContext:
    """Persistent reference buffers for repeated evaluations of one Model."""

    def __init__(self, ref: Reference, m: Model):
        self.ref, self.m = ref, m
        t = np.ascontiguousarray(m.t, dtype=np.float64)
        k = np.ascontiguousarray(m.kappa, dtype=np.float64)
        f = np.ascontiguousarray(m.flags, dtype=np.int32)
        self.h = ref.lib.ref_ctx_new(m.l1, m.l2, m.nt, _ptr(t), _ptr(k), m.mu, m.omega, m.flavors, _ptr(f))

    def close(self):
        if self.h:
            self.ref.lib.ref_ctx_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def eval(self, x, want_M=False):
        """construct_M_hat + logDetM_and_inv_M_hat + force (simulation/organic_hmc.c:177-180)."""
        pd = np.empty(self.m.dim)
        Mpre = np.empty((self.m.ns, self.m.ns)) if want_M else None
        Mi = np.empty((self.m.ns, self.m.ns)) if want_M else None
        ld = self.ref.lib.ref_ctx_eval(self.h, _ptr(np.ascontiguousarray(x)), _ptr(pd), _ptr(Mpre), _ptr(Mi))
        return (ld, pd, Mpre, Mi) if want_M else (ld, pd)

    def last_time(self):
        return self.ref.lib.ref_ctx_last_time(self.h)

    def construct_M_hat(self, x):
        M = np.empty((self.m.ns, self.m.ns))
        self.ref.lib.ref_ctx_construct_M_hat(self.h, _ptr(np.ascontiguousarray(x)), _ptr(M))
        return M

    def apply_exp(self, x_slice, M, revert=0, stop=2):
        M = np.array(M, dtype=np.float64, order="C", copy=True)
        self.ref.lib.ref_ctx_apply_exp(self.h, _ptr(np.ascontiguousarray(x_slice)), _ptr(M), revert, stop)
        return M

    def apply_mu_K_v(self, x_slice, v):
        w = np.empty(self.m.ns)
        self.ref.lib.ref_ctx_apply_mu_K_v(self.h, _ptr(np.ascontiguousarray(x_slice)), _ptr(np.ascontiguousarray(v)), _ptr(w))
        return w

    def all_QM1P(self, x, M_inv):
        G = np.empty((self.m.nt, self.m.ns, self.m.ns))
        self.ref.lib.ref_ctx_all_QM1P(self.h, _ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(M_inv)), _ptr(G))
        return G

    def refine(self, x, G_t, t):
        G = np.array(G_t, dtype=np.float64, order="C", copy=True)
        self.ref.lib.ref_ctx_refine(self.h, _ptr(np.ascontiguousarray(x)), _ptr(G), t)
        return G

    def logdet_inv(self, M):
        A = np.array(M, dtype=np.float64, order="C", copy=True)
        ld = self.ref.lib.ref_ctx_logdet_inv(self.h, _ptr(A))
        return ld, A

    def check_force(self, x, p_dot):
        return self.ref.lib.ref_ctx_check_force(self.h, _ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(p_dot)))

    def cc_correlator(self, x, M_inv, logdet):
        g = np.empty(self.m.nt * 9)
        self.ref.lib.ref_ctx_cc_correlator(self.h, _ptr(np.ascontiguousarray(x)), _ptr(np.ascontiguousarray(M_inv)), logdet, _ptr(g))
        return g


class RefFA:
    """Reference Fourier-acceleration routines bound to [x|p] and [xc|pc] plans."""

    def __init__(self, ref: Reference, ns, nt):
        self.ref, self.ns, self.nt = ref, ns, nt
        self.h = ref.lib.ref_fa_new(ns, nt)

    def close(self):
        if self.h:
            self.ref.lib.ref_fa_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, x=None, p=None):
        self.ref.lib.ref_fa_set(self.h, _ptr(None if x is None else np.ascontiguousarray(x)),
                                _ptr(None if p is None else np.ascontiguousarray(p)))

    def get(self):
        n = 3 * self.ns * self.nt
        x, p = np.empty(n), np.empty(n)
        self.ref.lib.ref_fa_get(self.h, _ptr(x), _ptr(p))
        return x, p

    def evolve(self, omega, h):
        self.ref.lib.ref_fa_evolve(self.h, omega, h)

    def sample_momenta(self, seed, omega, flags=(0,) * 7):
        self.ref.lib.ref_init_genrand64(seed)
        f = np.ascontiguousarray(flags, dtype=np.int32)
        self.ref.lib.ref_fa_sample_momenta(self.h, omega, _ptr(f))

    def energy(self, omega):
        return self.ref.lib.ref_fa_energy(self.h, omega)

    def approx_step(self, omega, h, cfa_mass):
        self.ref.lib.ref_fa_approx_step(self.h, omega, h, cfa_mass)

    def update_x(self, omega, h, half, flags=(0,) * 7, cfa_steps=1, cfa_mass=0.0):
        p_dot = np.zeros(3 * self.ns * self.nt)
        f = np.ascontiguousarray(flags, dtype=np.int32)
        self.ref.lib.ref_fa_update_x(self.h, _ptr(p_dot), omega, h, half, _ptr(f), cfa_steps, cfa_mass)

    def sample_free(self, seed, omega):
        self.ref.lib.ref_init_genrand64(seed)
        self.ref.lib.ref_fa_sample_free(self.h, omega)


def rel_max(a, b):
    """max |a-b| / max |b| (0 when both are zero)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if a.size else 0.0
    return 0.0 if den == 0 and num == 0 else num / den


# ---------------------------------------------------------------------- static disorder (TL mode)
def contraction_matrix(a, b):
    """construct_contraction_mat (simulation/organic_lattice.c:48-60), n = 3."""
    m = np.empty(6)
    for c in range(2):
        m[3 * c] = a[c]
        m[3 * c + 1] = .5 * (a[c] + b[c])
        m[3 * c + 2] = .5 * (-a[c] + b[c])
    return m


def forward_neighbours(l1, l2):
    """nnt[6i + 2k] of construct_triangular (simulation/organic_lattice.c:10-46):
    site i = a + l1 b, link 0 right, 1 up, 2 up-left; returns [V][3]."""
    i = np.arange(l1 * l2)
    a, b = i % l1, i // l1
    up = ((b + 1) % l2) * l1
    return np.stack([b * l1 + (a + 1) % l1, up + a, up + (a + l1 - 1) % l1], axis=1)


def trans_loc_sample(x, l1, l2, nbins, t, kappa, mu, contr_mat, width):
    """One sample of hist_trans_loc (simulation/organic_trans_loc.c:25-83)
    restated with dense numpy matrices, for small lattices:
      H = -mu 1 + K(x)                 construct_hamilton (organic_dense_matrix.c:218-224)
      I_k: w[i] += f v[n], w[n] -= f v[i]    apply_current_to_v (:226-249)
      P_k[j, i] = psi_j . I_k psi_i; I = sum_c (sum_k mat[c,k] P_k)^2 (contr_gr_mat)
      every pair E_j >= E_i adds (e^-E_i + e^-E_j) I / (width V) to bin
      (unsigned)((E_j - E_i)/width + .5); bins past the end are dropped here.
    Returns (histogram, partition sum / V)."""
    V = l1 * l2
    nb = forward_neighbours(l1, l2)
    fac = np.asarray(t)[None, :] - np.asarray(kappa)[None, :] * np.asarray(x).reshape(V, 3)
    H = np.zeros((V, V))
    H[np.arange(V), np.arange(V)] += -mu
    cur = np.zeros((3, V, V))
    for k in range(3):
        np.add.at(H, (np.arange(V), nb[:, k]), fac[:, k])
        np.add.at(H, (nb[:, k], np.arange(V)), fac[:, k])
        np.add.at(cur[k], (np.arange(V), nb[:, k]), fac[:, k])
        np.add.at(cur[k], (nb[:, k], np.arange(V)), -fac[:, k])
    ev, psi = np.linalg.eigh(H)
    m = np.asarray(contr_mat).reshape(2, 3)
    P = np.stack([psi.T @ cur[k] @ psi for k in range(3)])  # P[k, j, i]
    I = sum((m[c, 0] * P[0] + m[c, 1] * P[1] + m[c, 2] * P[2]) ** 2 for c in range(2))
    jj, ii = np.meshgrid(np.arange(V), np.arange(V), indexing="ij")
    keep = ev[jj] >= ev[ii]
    w = (np.exp(-ev[ii]) + np.exp(-ev[jj])) * I / (width * V)
    bins = np.floor((ev[jj] - ev[ii]) / width + .5)
    keep &= bins < nbins
    hist = np.zeros(nbins)
    np.add.at(hist, bins[keep].astype(np.int64), w[keep])
    return hist, float(np.sum(np.exp(-ev)) / V)


# ---------------------------------------------------------------------- organic_conv restated
HALF_PI_REF = 1.570796326794897  # simulation/organic_aux.h:10
PI_REF = 3.141592653589793


def _tanhc(x):
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(x != 0, np.tanh(x) / np.where(x != 0, x, 1.0), 1.0)


def _sigma_of_w(w, t, omega, width):
    """sigma_of_w (simulation/organic_conv.c:9-17)."""
    effW = -(w * width + omega)
    tt = t * effW
    with np.errstate(over="ignore"):
        return np.exp(tt) / (1 + w * w) * (1 + np.exp(effW - 2 * tt)) / (1 + np.exp(effW))


def _integral_sigma(t, omega, width):
    """calc_integral_sigma (:19-49) for an array of omega: tanh-sinh, step
    0.03, at most 200 nodes, each element stopping at its first term below
    DBL_EPSILON times its running sum."""
    omega = np.asarray(omega, dtype=np.float64)
    if t > .5:
        t = 1 - t
    if t == 0:
        return np.full(omega.shape, PI_REF)
    h = 0.03
    s = HALF_PI_REF * _sigma_of_w(0.0, t, omega, width)
    active = np.ones(omega.shape, dtype=bool)
    for i in range(1, 200):
        x = i * h
        sh_x = HALF_PI_REF * np.sinh(x)
        ch_x = HALF_PI_REF * np.cosh(x)
        w = np.sinh(sh_x)
        val = _sigma_of_w(w, t, omega, width) + _sigma_of_w(w, t, -omega, width)
        term = val * (ch_x * np.cosh(sh_x))
        active &= term >= 2.220446049250313e-16 * s
        if not active.any():
            break
        s = np.where(active, s + term, s)
    return h * s


def conv_sigma_w(sigma, h, widths):
    """smeared_sigma_w (simulation/organic_conv.c:92-111) for every bin's
    frequency i h and every width: [n][len(widths)]."""
    sigma = np.asarray(sigma, dtype=np.float64)
    n = len(sigma)
    om = np.arange(n) * h
    x0 = np.arange(n) * h
    out = np.empty((n, len(widths)))
    pre = PI_REF * .5 * _tanhc(.5 * om)
    for k, wd in enumerate(widths):
        if wd == 0:
            out[:, k] = np.where(np.arange(n) == 0, sigma, pre * sigma)
            continue
        d1 = om[:, None] - x0[None, :]
        d2 = om[:, None] + x0[None, :]
        ker = wd / (PI_REF * (wd * wd + d1 * d1)) + wd / (PI_REF * (wd * wd + d2 * d2))
        out[:, k] = pre * h * (ker @ sigma)
    return out


def conv_sigma_t(sigma, h, widths, nt):
    """smeared_sigma_t (:113-121) with the tanh-sinh kernel (eval_GK_kernel
    with nt = 0, :65-75) at t = i/nt, i <= nt/2: [nt/2+1][len(widths)]."""
    sigma = np.asarray(sigma, dtype=np.float64)
    om = np.arange(len(sigma)) * h
    out = np.empty((nt // 2 + 1, len(widths)))
    for i in range(nt // 2 + 1):
        t = i / nt
        for k, wd in enumerate(widths):
            ker = _sigma_of_w(0.0, t, om, 1.0) if wd == 0 else _integral_sigma(t, om, wd) / PI_REF
            out[i, k] = h * np.sum(sigma * ker)
    return out
