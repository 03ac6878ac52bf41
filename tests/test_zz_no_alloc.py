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


def _gas(name, n, seed):
    """Gas-phase n-mers of the evaluator's monomers, first atoms 2.6 A to
    just beyond the evaluator's cutoff from the first monomer's."""
    from mbx_b200.specs import SPECS
    s = SPECS[name]
    rng = np.random.default_rng(seed)
    bodies = {m: f() for m, f in workloads.BODIES.items()}
    out = []
    for _ in range(n):
        parts = []
        for k, m in enumerate(s.monomers):
            c = np.zeros(3) if k == 0 else workloads._random_directions(rng, 1)[0] * rng.uniform(2.6, s.rf + 0.5)
            parts.append(workloads.place(rng, bodies[m], c[None, :])[0].reshape(-1))
        out.append(np.concatenate(parts))
    return np.ascontiguousarray(np.array(out))


@pytest.mark.parametrize("grads", [True, False])
@pytest.mark.parametrize("name", ["mbpol3b", "mbpol2b", "ch4h2o2b", "ch4h2o3b"])
def test_noalloc_matches_evaluate_on_two_calls(name, grads):
    ctx = capi.Context(0)
    xyz_np = _gas(name, 3000, seed=21)
    n = len(xyz_np)
    # the existing entry point (allocates its own staging buffers)
    g_ref = np.zeros_like(xyz_np)
    v_ref = np.zeros(9)
    e_ref_per = np.zeros(n)
    e_ref = ctx.evaluate(name, xyz_np, g_ref if grads else None, v_ref, e_ref_per, grads=grads)

    stream = torch.cuda.current_stream().cuda_stream
    xyz = torch.tensor(xyz_np, device="cuda")
    results = []
    for call in range(2):
        grad = torch.zeros_like(xyz) if grads else None
        e_per = torch.full((n,), 7.0, dtype=torch.float64, device="cuda") if call == 0 else None
        result = torch.full((7,), 123.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = _noalloc(name, xyz, grad, e_per, result, stream)
        torch.cuda.synchronize()
        assert rc == 0
        r = result.cpu().numpy()
        assert abs(r[0] - e_ref) < E_REL * abs(e_ref) or abs(r[0] - e_ref) < E_ABS_NMER
        if grads:
            np.testing.assert_allclose(grad.cpu().numpy(), g_ref, rtol=0, atol=G_ABS)
            np.testing.assert_allclose(r[1:], v_ref[[0, 1, 2, 4, 5, 8]], rtol=1e-9, atol=1e-8)
        else:
            assert not r[1:].any()   # no virial without gradients
        if e_per is not None:
            np.testing.assert_allclose(e_per.cpu().numpy(), e_ref_per, rtol=0, atol=E_ABS_NMER)
        results.append(r[0])
    # fixed-order sum: the two calls agree exactly
    assert results[0] == results[1]
    ctx.close()


_FRESH = r"""
import ctypes, json, sys
sys.path.insert(0, %(root)r)
import numpy as np
import torch
from mbx_b200 import capi, workloads
L = capi.lib()          # the library only: no context exists in this process
f = L.mbx_evaluate_noalloc
f.argtypes = [ctypes.c_char_p, ctypes.c_long] + [ctypes.c_void_p] * 5
f.restype = ctypes.c_int
xyz = torch.tensor(workloads.gas_trimers(400, seed=5), device="cuda")
grad = torch.zeros_like(xyz)
result = torch.zeros(7, dtype=torch.float64, device="cuda")
s = torch.cuda.current_stream().cuda_stream
out = []
for _ in range(2):
    grad.zero_()
    torch.cuda.synchronize()
    rc = f(b"mbpol3b", xyz.shape[0], xyz.data_ptr(), grad.data_ptr(), None, result.data_ptr(), s)
    torch.cuda.synchronize()
    out.append({"rc": rc, "e": result[0].item(), "gmax": grad.abs().max().item()})
print(json.dumps(out))
"""


def test_noalloc_first_call_without_context():
    """In a fresh process with no context: the first call loads the models'
    fitted coefficients itself (no zero energies), and agrees with the
    context-based entry point."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH % {"root": root}], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    calls = json.loads(r.stdout.strip().splitlines()[-1])
    ctx = capi.Context(0)
    xyz_np = workloads.gas_trimers(400, seed=5)
    g = np.zeros_like(xyz_np)
    e_ref = ctx.evaluate("mbpol3b", xyz_np, g)
    ctx.close()
    for c in calls:
        assert c["rc"] == 0 and c["e"] != 0.0
        assert abs(c["e"] - e_ref) < E_REL * abs(e_ref) or abs(c["e"] - e_ref) < E_ABS_NMER
        assert abs(c["gmax"] - np.abs(g).max()) < G_ABS
    assert calls[0]["e"] == calls[1]["e"]


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
