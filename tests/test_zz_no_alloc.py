"""GPU test of ephmc_logdet_inverse_noalloc, the entry point that allocates
nothing (its LU workspace is a static device array), for callers whose device
memory is owned by someone else or who must not allocate after start-up.

Called through the C ABI with a device matrix the caller owns; compared with
the context-based ephmc_logdet_inverse on the same matrix, on two calls in a
row (the static workspace keeps the previous call's data, which must not leak
into the next result).  Named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    import ephmc
    lib = ephmc.load_library()
    f = lib.ephmc_logdet_inverse_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_uint, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p, C.c_void_p]
    return lib


def _noalloc(lib, Md, n):
    ld, sg = C.c_double(0.0), C.c_int(0)
    ipiv = np.zeros(n, dtype=np.int32)
    st = lib.ephmc_logdet_inverse_noalloc(Md.data_ptr(), n, C.byref(ld), C.byref(sg), ipiv.ctypes.data, None)
    return st, ld.value, sg.value, ipiv


@pytest.mark.parametrize("n,l1,l2", [(36, 6, 6), (256, 16, 16)])
def test_noalloc_matches_context_entry_point_twice(gpu, n, l1, l2):
    import torch

    import ephmc
    lib = _lib()
    rng = np.random.default_rng(n)
    with ephmc.Context(l1, l2, 1, [0.1, 0.1, 0.1], [0.0, 0.0, 0.0], -1.0, 0.1) as ctx:
        for call in range(2):
            A = rng.standard_normal((n, n)) + (2.0 + call) * np.eye(n)
            ref = A.copy()
            ld_ref, sg_ref, ipiv_ref = ctx.logdet_inverse(ref)
            Md = torch.from_numpy(A.copy()).cuda()
            st, ld, sg, ipiv = _noalloc(lib, Md, n)
            assert st == 0, lib.ephmc_last_error_message()
            inv = Md.cpu().numpy()
            assert abs(ld - ld_ref) <= 1e-12 * abs(ld_ref) + 1e-13
            assert sg == sg_ref
            assert np.array_equal(ipiv, ipiv_ref)
            assert np.max(np.abs(inv - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_noalloc_rejects_oversize(gpu):
    import torch
    lib = _lib()
    Md = torch.zeros((257, 257), dtype=torch.float64, device="cuda")
    st, _, _, _ = _noalloc(lib, Md, 257)
    assert st == 2
    assert b"256" in lib.ephmc_last_error_message()


def test_noalloc_alternating_sizes(gpu):
    """Calls of different sizes share the static workspace: 256, 128, 256, 64,
    256 in a row, each against numpy.  The LU kernel's call counter sits at the
    same word for every size, so the panel flags and messages that a smaller
    call leaves behind never carry the epoch of a later, larger call."""
    import torch
    lib = _lib()
    rng = np.random.default_rng(7)
    for n in (256, 128, 256, 64, 256, 128):
        A = rng.standard_normal((n, n)) + 3.0 * np.eye(n)
        Md = torch.from_numpy(A.copy()).cuda()
        st, ld, sg, ipiv = _noalloc(lib, Md, n)
        assert st == 0, lib.ephmc_last_error_message()
        s_np, ld_np = np.linalg.slogdet(A.T)  # the LU sees the transpose (column-major)
        assert abs(ld - ld_np) <= 1e-11 * abs(ld_np), n
        assert sg == int(s_np), n
        inv = Md.cpu().numpy()
        ref = np.linalg.inv(A)
        assert np.max(np.abs(inv - ref)) <= 1e-10 * np.max(np.abs(ref)), n
