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


def test_noalloc_singular_then_regular(gpu):
    """The all-ones matrix has an exact zero pivot at the second step:
    EPHMC_ERR_SINGULAR, with *logdet and *sign left as they were; the next
    call, of another size, on the same static workspace is correct."""
    import torch
    lib = _lib()
    Md = torch.ones((64, 64), dtype=torch.float64, device="cuda")
    ld, sg = C.c_double(123.0), C.c_int(7)
    st = lib.ephmc_logdet_inverse_noalloc(Md.data_ptr(), 64, C.byref(ld), C.byref(sg), None, None)
    assert st == 4
    assert ld.value == 123.0 and sg.value == 7
    rng = np.random.default_rng(11)
    A = rng.standard_normal((100, 100)) + 3.0 * np.eye(100)
    Md = torch.from_numpy(A.copy()).cuda()
    st, ld2, sg2, _ = _noalloc(lib, Md, 100)
    assert st == 0, lib.ephmc_last_error_message()
    s_np, ld_np = np.linalg.slogdet(A.T)
    assert abs(ld2 - ld_np) <= 1e-11 * abs(ld_np) and sg2 == int(s_np)
    assert np.max(np.abs(Md.cpu().numpy() - np.linalg.inv(A.T).T)) <= 1e-10 * np.max(np.abs(np.linalg.inv(A)))


def test_noalloc_refuses_another_devices_matrix(gpu):
    """A matrix on another GPU than the current one is refused (the static
    workspace is per device); runs only where a second device exists."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device")
    lib = _lib()
    Md = torch.eye(16, dtype=torch.float64, device="cuda:1")
    torch.cuda.set_device(0)
    st, _, _, _ = _noalloc(lib, Md, 16)
    assert st == 2
