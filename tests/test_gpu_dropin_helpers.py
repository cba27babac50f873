"""Drop-in entry points beyond one evaluation, each against the reference's
own function (oracle/_ref, the reference's sources compiled unmodified),
called with host pointers as the reference's C host code calls them:

* construct_id, transpose, trace (simulation/organic_dense_matrix.c:47-93);
* apply_2nd_order_mu_K_to_v and apply_pair_expansion_mu_K_to_v (:168-194),
  bit for bit (the stencil sums in the reference's order);
* phonon_correlator (:526-545);
* check_force (simulation/organic_hmc.c:20-54): the finite-difference check
  of a force, both programs on the reference's force;
* cc_correlator (:451-524) at the 32x32, Nt = 64 workload on a fixed field
  and the same M_hat^-1, against the reference to 1e-10 of the largest
  entry, and timed."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

D, U, P, I = C.c_double, C.c_uint, C.c_void_p, C.c_int


class OrganicFlags(C.Structure):
    _fields_ = [("schur_form_inv", C.c_int), ("zero_filling", C.c_int), ("static_disorder", C.c_int),
                ("single_particle", C.c_int), ("constant_force", C.c_int), ("no_fourier_acc", C.c_int),
                ("classical_fourier_acc", C.c_int), ("cfa_steps", C.c_uint), ("cfa_mass", C.c_double)]


def _p(a):
    return a.ctypes.data


def _sigs(lib):
    lib.construct_id.argtypes = [P, U]
    lib.construct_id.restype = None
    lib.transpose.argtypes = [P, U]
    lib.transpose.restype = None
    lib.trace.argtypes = [P, U]
    lib.trace.restype = D
    lib.set_taylor_pair_order.argtypes = []
    lib.set_taylor_pair_order.restype = None
    # double complex a passes as two doubles in SSE registers (x86-64 System V)
    lib.apply_2nd_order_mu_K_to_v.argtypes = [P, P, P, P, P, D, P, U, U, D, D]
    lib.apply_2nd_order_mu_K_to_v.restype = None
    lib.apply_pair_expansion_mu_K_to_v.argtypes = [P, P, P, P, P, D, P, U, U, I, I]
    lib.apply_pair_expansion_mu_K_to_v.restype = None
    lib.phonon_correlator.argtypes = [P, U, U, U, P]
    lib.phonon_correlator.restype = None
    lib.check_force.argtypes = [P, P, P, P, P, P, P, P, D, D, U, P, U, U, U, P]
    lib.check_force.restype = D
    lib.cc_correlator.argtypes = [P, P, P, P, P, P, P, D, P, U, U, U, P, D, P]
    lib.cc_correlator.restype = None
    return lib


def _libs(reference):
    import ephmc
    return _sigs(ephmc.load_library()), _sigs(reference.lib)


def test_identity_transpose_trace(gpu, reference):
    gpu_lib, ref_lib = _libs(reference)
    rng = np.random.default_rng(3)
    n = 37
    for lib_pair in ((gpu_lib, ref_lib),):
        a = rng.standard_normal(n * n)
        outs = []
        for lib in lib_pair:
            m = a.copy()
            lib.transpose(_p(m), n)
            tr = lib.trace(_p(m), n)
            e = np.empty(n * n)
            lib.construct_id(_p(e), n)
            outs.append((m, tr, e))
        (mg, tg, eg), (mr, trr, er) = outs
        assert np.array_equal(mg, mr) and np.array_equal(mg.reshape(n, n), a.reshape(n, n).T)
        assert tg == trr
        assert np.array_equal(eg, er) and np.array_equal(eg.reshape(n, n), np.eye(n))


def test_pair_functions_bit_identical(gpu, reference, restated):
    from oracle import Model
    gpu_lib, ref_lib = _libs(reference)
    m = Model.physical(5, 4, 3, 2.0)
    nnt = restated.lattice(m.l1, m.l2)
    t, kap = np.array(m.t), np.array(m.kappa)
    x = restated.random_x(8, m.dim)
    xs = x[3 * m.ns: 6 * m.ns].copy()
    v0 = restated.random_x(9, m.ns)
    for lib in (gpu_lib, ref_lib):
        lib.set_taylor_pair_order()
    # a complex (two stencils) and a real (one stencil) pair coefficient
    for a in ((0.31, 0.17), (-0.42, 0.0)):
        res = []
        for lib in (gpu_lib, ref_lib):
            v, w = v0.copy(), np.empty(2 * m.ns)
            lib.apply_2nd_order_mu_K_to_v(_p(xs), _p(v), _p(w), _p(t), _p(kap), m.mu, _p(nnt), m.ns, 6, *a)
            res.append(v)
        assert np.array_equal(res[0], res[1]), a
    for revert, stop in ((0, 2), (0, 1), (0, 0), (1, -1), (1, 0), (1, 1)):
        res = []
        for lib in (gpu_lib, ref_lib):
            v, w = v0.copy(), np.empty(2 * m.ns)
            lib.apply_pair_expansion_mu_K_to_v(_p(xs), _p(v), _p(w), _p(t), _p(kap), m.mu, _p(nnt), m.ns, 6, revert,
                                               stop)
            res.append(v)
        assert np.array_equal(res[0], res[1]), (revert, stop)


def test_phonon_correlator(gpu, reference, restated):
    gpu_lib, ref_lib = _libs(reference)
    ns, nt = 20, 6
    x = restated.random_x(4, 3 * ns * nt)
    out = []
    for lib in (gpu_lib, ref_lib):
        g = np.empty(nt * 9)
        lib.phonon_correlator(_p(x.copy()), ns, 6, nt, _p(g))
        out.append(g)
    assert np.allclose(out[0], out[1], rtol=1e-14, atol=1e-15)


def test_check_force(gpu, reference, restated):
    """Both programs' finite-difference check of the same (reference) force
    on a 3x3 lattice, Nt = 4: sqrt(sum (p_dot - fd)^2 / sum (|p_dot| + |fd|)^2),
    which the reference expects near its FD accuracy (1e-10 .. 1e-8)."""
    from oracle import Model
    gpu_lib, _ = _libs(reference)
    m = Model.physical(3, 3, 4, 1.0)
    nnt = restated.lattice(m.l1, m.l2)
    t, kap = np.array(m.t), np.array(m.kappa)
    x = restated.random_x(12, m.dim)
    reference.set_threads(1)
    rc = reference.context(m)
    ld, pd = rc.eval(x)
    r_ref = rc.check_force(x.copy(), pd)
    rc.close()
    flags = OrganicFlags()
    M = np.empty(m.ns * m.ns)
    w = np.empty(5 * m.ns * m.ns)
    perm = np.zeros(max(m.ns, 2 * m.nt), dtype=np.int32)
    p = np.zeros(m.dim)
    xg = x.copy()
    r_gpu = gpu_lib.check_force(_p(xg), _p(p), _p(pd), _p(M), _p(w), _p(perm), _p(t), _p(kap), m.mu, m.omega,
                                m.flavors, _p(nnt), m.ns, 6, m.nt, C.byref(flags))
    print(f"check_force: GPU {r_gpu:.3e}, reference {r_ref:.3e}")
    assert np.array_equal(xg, x)  # x restored
    assert r_gpu <= 1e-7 and r_ref <= 1e-7
    assert abs(r_gpu - r_ref) <= 0.5 * r_ref + 1e-10


def test_cc_correlator_at_32x32(gpu, reference, restated):
    """32x32, Nt = 64, beta = 20, seed 1: the GPU cc_correlator (one R_t0
    stack, R_0t streamed slice by slice) against the reference's on the same
    field and the same M_hat^-1."""
    import ephmc
    from oracle import Model
    gpu_lib, _ = _libs(reference)
    m = Model.physical(32, 32, 64, 20.0)
    nnt = restated.lattice(m.l1, m.l2)
    t, kap = np.array(m.t), np.array(m.kappa)
    x = restated.random_x(1, m.dim)
    with ephmc.Context(m.l1, m.l2, m.nt, m.t, m.kappa, m.mu, m.omega) as ctx:
        ld, _ = ctx.eval(x, mode="adjoint")
        Mi = ctx.inverse()
    reference.set_threads(8)
    rc = reference.context(m)
    g_ref = rc.cc_correlator(x, Mi, ld)
    rc.close()
    flags = OrganicFlags()
    Rt0 = np.empty(m.nt * m.ns * m.ns)
    R0t = np.empty(m.ns * m.ns)
    w = np.empty(5 * m.ns * m.ns)
    g = np.empty(m.nt * 9)
    args = (_p(x), _p(Mi), _p(Rt0), _p(R0t), _p(w), _p(t), _p(kap), m.mu, _p(nnt), m.ns, 6, m.nt, _p(g), ld,
            C.byref(flags))
    gpu_lib.cc_correlator(*args)
    t0 = time.perf_counter()
    gpu_lib.cc_correlator(*args)
    dt = time.perf_counter() - t0
    err = float(np.max(np.abs(g - g_ref)) / np.max(np.abs(g_ref)))
    print(f"cc_correlator 32x32 Nt=64: {err:.2e} of the largest entry; {1e3 * dt:.1f} ms per call with host "
          f"buffers (R_t0 back to the host: {Rt0.nbytes / 1e6:.0f} MB)")
    assert err <= 1e-10


def test_trajectory_host_block_equals_device_block(gpu, restated):
    """trajectory() (simulation/organic_hmc.c:192-294) with the reference's
    state block in host memory (the library keeps a device block and moves
    only x, M_hat in and x, p, p_dot, x_old, M_hat, M_hat_old out) against
    the same call with the block in device memory, on the same random
    stream: same Metropolis decision, field, inverse and log det."""
    import torch

    import ephmc
    from oracle import Model
    lib = ephmc.load_library()
    lib.ephmc_rng_seed.argtypes = [C.c_ulonglong]
    lib.ephmc_rng_seed.restype = None
    lib.construct_M_hat.argtypes = [P, P, P, P, P, D, P, U, U, U, P]
    lib.construct_M_hat.restype = None
    lib.logDetM_and_inv_M_hat.argtypes = [P, P, P, U, U, P]
    lib.logDetM_and_inv_M_hat.restype = D
    lib.trajectory.argtypes = [P, P, P, P, P, D, D, U, P, P, U, U, U, U, D, P, P, I, U, P, P, P, P, P]
    lib.trajectory.restype = C.c_short
    m = Model.physical(6, 6, 16, 4.0, mu0=1.0)
    nnt = restated.lattice(m.l1, m.l2)
    t, kap = np.array(m.t), np.array(m.kappa)
    dim, VV = m.dim, m.ns * m.ns
    flags = OrganicFlags()
    block0 = np.zeros(4 * dim + (8 + m.nt) * VV)
    block0[:dim] = 0.3 * restated.random_x(21, dim)
    w = np.empty(5 * VV)
    perm = np.zeros(max(m.ns, 2 * m.nt), dtype=np.int32)
    M = block0[4 * dim: 4 * dim + VV]
    lib.construct_M_hat(_p(block0), _p(M), _p(w), _p(t), _p(kap), m.mu, _p(nnt), m.ns, 6, m.nt, C.byref(flags))
    ld0 = lib.logDetM_and_inv_M_hat(_p(M), _p(w), _p(perm), m.ns, 1, C.byref(flags))
    out = []
    for on_device in (False, True):
        for seed in (31, 32):
            lib.ephmc_rng_seed(seed)
            old = np.array([ld0])
            blk = block0.copy()
            bd = torch.from_numpy(blk).cuda() if on_device else None
            acc = lib.trajectory(bd.data_ptr() if on_device else _p(blk), None, None, _p(t), _p(kap), m.mu, m.omega,
                                 1, None, _p(nnt), m.ns, 6, m.nt, 3, np.pi / 2, None, None, 1, 1, None, _p(old), None, None,
                                 C.byref(flags))
            if on_device:
                blk = bd.cpu().numpy()
            out.append((acc, blk[:dim].copy(), blk[4 * dim: 4 * dim + VV].copy(), old[0]))
    for (a0, x0, m0, l0), (a1, x1, m1, l1) in zip(out[:2], out[2:]):
        assert a0 == a1
        assert np.max(np.abs(x0 - x1)) <= 1e-12 * np.max(np.abs(x1))
        assert np.max(np.abs(m0 - m1)) <= 1e-12 * np.max(np.abs(m1))
        assert abs(l0 - l1) <= 1e-12 * abs(l1)
