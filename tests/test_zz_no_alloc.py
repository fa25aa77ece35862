"""The allocation-free tri-diagonal solve (tcgpu_tdm_solve_noalloc).

It exists for callers that may not allocate device memory, or have a library
do so on their behalf: frameworks that own the whole device memory pool,
real-time hosts that reserve all device memory up front, or plugins whose
allocations belong to their host. Its factor table lives in a fixed static
device array instead of cudaMalloc'd memory. Here it is called through the C ABI and checked against the ordinary
tdm.solve() entry point on the same systems, for two calls in a row (the
second with a different system, so nothing may carry over from the first).
Both run the same arithmetic, so the answers must agree exactly, the same
bit-exact standard the other tdm tests apply.
"""
import ctypes as C

import numpy as np
import pytest

from simpletcsolver_b200 import abi

pytestmark = pytest.mark.gpu


def reference_solve(lib, l, c, u, q, periodic, cplx):
    """tdm.solve() with host right-hand sides."""
    tdm = abi.tdm_vtable(lib)
    n, nrhs = l.shape[0], q.shape[0]
    info = abi.TdmInfoP()
    assert tdm.construct(n, nrhs, periodic, cplx, C.byref(info)) == 0
    ptr = abi.c_double_p()
    for v, getter in ((l, tdm.get_l), (c, tdm.get_c), (u, tdm.get_u)):
        getter(info, C.byref(ptr))
        np.ctypeslib.as_array(ptr, shape=(n,))[:] = v
    data = np.ascontiguousarray(q.copy())
    assert tdm.solve(info, data.ctypes.data_as(C.c_void_p)) == 0
    assert tdm.destruct(info) == 0
    return data


def random_system(rng, n, nrhs, cplx):
    l = rng.uniform(-1.0, 1.0, n)
    u = rng.uniform(-1.0, 1.0, n)
    c = rng.uniform(2.5, 4.0, n) * rng.choice([-1.0, 1.0], n)
    q = rng.standard_normal((nrhs, n, 2) if cplx else (nrhs, n))
    return l, c, u, q


@pytest.mark.parametrize("periodic,cplx", [(False, False), (True, False), (False, True), (True, True)])
def test_noalloc_solve_matches_tdm_solve_twice(lib, periodic, cplx):
    import torch
    f = lib.tcgpu_tdm_solve_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_bool, C.c_bool, abi.c_double_p, abi.c_double_p, abi.c_double_p,
                  C.c_void_p]
    rng = np.random.default_rng(99 + 2 * periodic + cplx)
    for n, nrhs in ((257, 40), (33, 7)):
        l, c, u, q = random_system(rng, n, nrhs, cplx)
        expect = reference_solve(lib, l, c, u, q, periodic, cplx)
        dq = torch.from_numpy(np.ascontiguousarray(q.copy())).cuda()
        torch.cuda.synchronize()
        rc = f(n, nrhs, periodic, cplx, l.ctypes.data_as(abi.c_double_p), c.ctypes.data_as(abi.c_double_p),
               u.ctypes.data_as(abi.c_double_p), C.c_void_p(dq.data_ptr()))
        assert rc == 0, abi.last_error(lib)
        np.testing.assert_array_equal(dq.cpu().numpy(), expect)


def test_noalloc_solve_rejects_oversized_systems(lib):
    import torch
    f = lib.tcgpu_tdm_solve_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_bool, C.c_bool, abi.c_double_p, abi.c_double_p, abi.c_double_p,
                  C.c_void_p]
    n = 8193                                    # one past TCGPU_TDM_NOALLOC_MAX_SIZE
    l = np.zeros(n)
    dq = torch.zeros(n, dtype=torch.float64, device="cuda")
    rc = f(n, 1, False, False, l.ctypes.data_as(abi.c_double_p), l.ctypes.data_as(abi.c_double_p),
           l.ctypes.data_as(abi.c_double_p), C.c_void_p(dq.data_ptr()))
    assert rc != 0
    assert "size" in abi.last_error(lib)
    host = np.zeros(8)                          # host right-hand sides would need a device copy
    rc = f(8, 1, False, False, l.ctypes.data_as(abi.c_double_p), l.ctypes.data_as(abi.c_double_p),
           l.ctypes.data_as(abi.c_double_p), host.ctypes.data_as(C.c_void_p))
    assert rc != 0
    assert "device memory" in abi.last_error(lib)
