"""The drop-in boundary from the reference's own C++ (GPU).

``oracle/_ref/libmbx_ref_gpu.so`` is the reference's ``bblock::System``
compiled with ``-DMBX_GPU_2B3B``: ``System::Get2B`` / ``Get3B``
(bblock/system.cpp:2425, 2769) forward to ``libmbx_b200.so`` through the C
ABI (oracle/ref_gpu_glue.cpp, built by oracle/build_ref_gpu.py), and
everything else, including the public ``TwoBodyEnergy(true)`` /
``ThreeBodyEnergy(true)`` entries (system.cpp:2403-2423, 2727-2745), is the
reference's code.  Its energies, ``grad_`` and ``virial_`` must equal the
unmodified reference's (the committed fixtures of tests/golden) within
1e-10 relative / 1e-8 kcal/mol/A.
"""
import os
import sys

import numpy as np
import pytest

import mbx_oracle as mo
from conftest import GOLDEN

pytestmark = pytest.mark.gpu
sys.path.insert(0, GOLDEN)


@pytest.mark.parametrize("name", ["water_256", "methane_water"])
def test_patched_reference_system_matches_reference(name):
    from make_ref_fixtures import WORKLOADS, xyz_hash
    if not mo.RefGpuSystem.available():
        pytest.fail("oracle/_ref/libmbx_ref_gpu.so is not built (python oracle/build_ref_gpu.py)")
    make_fn, c2, c3 = WORKLOADS[name]
    ids, xyz, box = make_fn()
    d = np.load(os.path.join(GOLDEN, "ref_%s.npz" % name))
    assert str(d["xyz_sha256"]) == xyz_hash(xyz)
    r = mo.RefGpuSystem(ids, xyz, box, c2, c3)
    for nb in (2, 3):
        e = r.energy(nb)
        er = float(d["e%d" % nb])
        assert abs(e - er) <= 1e-10 * abs(er), (nb, e, er)
        np.testing.assert_allclose(r.real_grads(), d["g%d" % nb], rtol=0, atol=1e-8)
        np.testing.assert_allclose(r.virial(), d["v%d" % nb], rtol=1e-10, atol=1e-7)
    # energy only (do_grads = false) through the same entry
    e3 = r.energy(3, do_grads=False)
    assert abs(e3 - float(d["e3"])) <= 1e-10 * abs(float(d["e3"]))
