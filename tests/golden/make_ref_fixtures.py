#!/usr/bin/env python3
"""Writes the reference's own results on the synthetic workloads as fixtures.

Test infrastructure.  Runs the compiled reference (oracle/_ref/libmbx_ref.so,
built by oracle/build_ref.py from the reference's sources) through
``bblock::System::TwoBodyEnergy(true)`` / ``ThreeBodyEnergy(true)``
(bblock/system.cpp:2403-2423, 2727-2745) on the seeded workloads of
``mbx_b200.workloads`` and stores, per workload, in
``tests/golden/ref_<workload>.npz``:

* ``xyz_sha256``: the input coordinates' hash (the workload recipe must not drift);
* ``e1`` (water workloads): the 1-body energy, ``g1``, ``v1`` its gradient
  and virial (``OneBodyEnergy(true)``, bblock/system.cpp:2140);
* ``e2``, ``e3``: the 2-body and 3-body energies (kcal/mol);
* ``g2``, ``g3``: the gradients of real atoms, input order (kcal/mol/A);
* ``v2``, ``v3``: the virials (9 each);
* ``n2``, ``n3``: the reference's dimer / trimer list lengths and
  ``l2_sha256``, ``l3_sha256``: the hash of each list in input monomer
  indices, every n-mer sorted and the rows sorted (the reference's sortEdge
  canonical form), as little-endian int64.

The GPU tests compare the CUDA path with these, so that the reference itself,
not a restatement of it, is the oracle on the full-size workloads, also where
the reference library cannot be built (the GPU machines hold no reference
sources).

Usage: ``python tests/golden/make_ref_fixtures.py`` (after oracle/build_ref.py).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mbx_oracle as mo  # noqa: E402
from mbx_b200 import workloads  # noqa: E402

WORKLOADS = {
    "water_256": (lambda: workloads.water_256(0), 9.0, 7.0),
    "water_2048": (lambda: workloads.water_2048(0), 9.0, 7.0),
    "methane_water": (lambda: workloads.methane_water_box(seed=0), 9.0, 7.0),
    "water_256_bead": (lambda: workloads.water_256_bead(0), 9.0, 7.0),
}


# workloads whose monomers all have a GPU 1-body term (water, CH4)
ONEBODY = ("water_256", "water_2048", "water_256_bead", "methane_water")


def list_hash(nm):
    nm = np.ascontiguousarray(np.asarray(nm, dtype="<i8"))
    return hashlib.sha256(nm.tobytes()).hexdigest()


def xyz_hash(xyz):
    return hashlib.sha256(np.ascontiguousarray(np.asarray(xyz, dtype="<f8")).tobytes()).hexdigest()


def make(name):
    make_fn, c2, c3 = WORKLOADS[name]
    ids, xyz, box = make_fn()
    r = mo.RefSystem(ids, xyz, box, c2, c3)
    out = {"xyz_sha256": xyz_hash(xyz)}
    if name in ONEBODY:
        # System::OneBodyEnergy(true) (bblock/system.cpp:2140)
        out["e1"] = r.energy(1)
        out["g1"] = r.real_grads()
        out["v1"] = r.virial()
    for nb, cut in ((2, c2), (3, c3)):
        out["e%d" % nb] = r.energy(nb)
        out["g%d" % nb] = r.real_grads()
        out["v%d" % nb] = r.virial()
        nm = r.pair_list(nb, cut)
        out["n%d" % nb] = len(nm)
        out["l%d_sha256" % nb] = list_hash(nm)
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)
    print("%s: E2B %.10f E3B %.10f, %d dimers, %d trimers" % (name, out["e2"], out["e3"], out["n2"], out["n3"]))


def main():
    if not mo.RefSystem.available():
        raise SystemExit("oracle/_ref/libmbx_ref.so is not built (python oracle/build_ref.py)")
    for name in WORKLOADS:
        make(name)


if __name__ == "__main__":
    main()
