"""The allocation-free evaluator entry point, mbx_evaluate_noalloc (GPU).

It serves callers that must not allocate device memory while they run (an
allocator-free real-time loop, a fixed memory pool, a plugin that may not grow
the process's device memory).  This file is named so that pytest collects it
last.  Two calls in a row through the C ABI must agree with mbx_evaluate (the
entry point that allocates its staging buffers) within the tolerances of the
other GPU tests, and with each other bit for bit (the entry point sums the
energy in a fixed order and its scratch array must be cleared between calls).
"""
import ctypes

import numpy as np
import pytest

from mbx_b200 import capi, workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

E_REL = 1e-10
E_ABS_NMER = 1e-8
G_ABS = 1e-8


def _noalloc(name, xyz, grad, e_per, result, stream):
    L = capi.lib()
    f = L.mbx_evaluate_noalloc
    f.argtypes = [ctypes.c_char_p, ctypes.c_long] + [ctypes.c_void_p] * 5
    f.restype = ctypes.c_int
    ptr = (lambda t: None if t is None else t.data_ptr())
    n = xyz.shape[0]
    return f(name.encode(), n, ptr(xyz), ptr(grad), ptr(e_per), ptr(result), stream)


@pytest.mark.parametrize("name,maker", [("mbpol3b", workloads.gas_trimers), ("mbpol2b", workloads.gas_dimers)])
def test_noalloc_matches_evaluate_on_two_calls(name, maker):
    ctx = capi.Context(0)   # loads the fitted coefficients on the device
    xyz_np = np.ascontiguousarray(maker(3000, seed=21))
    n = len(xyz_np)
    # the existing entry point (allocates its own staging buffers)
    g_ref = np.zeros_like(xyz_np)
    v_ref = np.zeros(9)
    e_ref_per = np.zeros(n)
    e_ref = ctx.evaluate(name, xyz_np, g_ref, v_ref, e_ref_per)

    stream = torch.cuda.current_stream().cuda_stream
    xyz = torch.tensor(xyz_np, device="cuda")
    results = []
    for call in range(2):
        grad = torch.zeros_like(xyz)
        e_per = torch.full((n,), 7.0, dtype=torch.float64, device="cuda") if call == 0 else None
        result = torch.full((7,), 123.0, dtype=torch.float64, device="cuda")
        rc = _noalloc(name, xyz, grad, e_per, result, stream)
        torch.cuda.synchronize()
        assert rc == 0
        r = result.cpu().numpy()
        g = grad.cpu().numpy()
        assert abs(r[0] - e_ref) < E_REL * abs(e_ref) or abs(r[0] - e_ref) < E_ABS_NMER
        np.testing.assert_allclose(g, g_ref, rtol=0, atol=G_ABS)
        np.testing.assert_allclose(r[1:], v_ref[[0, 1, 2, 4, 5, 8]], rtol=1e-9, atol=1e-8)
        if e_per is not None:
            np.testing.assert_allclose(e_per.cpu().numpy(), e_ref_per, rtol=0, atol=E_ABS_NMER)
        results.append(r[0])
    # fixed-order sum: the two calls agree exactly
    assert results[0] == results[1]
    ctx.close()


def test_noalloc_rejects_oversize_and_unknown():
    capi.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    xyz = torch.zeros((1, 27), dtype=torch.float64, device="cuda")
    result = torch.zeros(7, dtype=torch.float64, device="cuda")
    f = capi.lib().mbx_evaluate_noalloc
    f.argtypes = [ctypes.c_char_p, ctypes.c_long] + [ctypes.c_void_p] * 5
    f.restype = ctypes.c_int
    too_many = 262144 + 1
    assert f(b"mbpol3b", too_many, xyz.data_ptr(), None, None, result.data_ptr(), stream) == 22
    assert f(b"ch4ch42b", 1, xyz.data_ptr(), None, None, result.data_ptr(), stream) == 95
