"""``bblock::System``, reduced to its 2-body/3-body path, on the CUDA library.

Same names, argument meanings and error behaviour as the reference's
``bblock::System`` (bblock/system.h) for the calls this path needs:
``AddMonomer``, ``AddMolecule``, ``Initialize``, ``SetUpFromJson``,
``Set2bCutoff``, ``Set3bCutoff``, ``SetPBC``, ``SetRealXyz``,
``TwoBodyEnergy``, ``ThreeBodyEnergy``, ``GetRealGrads``, ``GetGrads``,
``GetVirial``, ``GetPairList``, ``GetXyz``, ``GetRealXyz``.  Energies are
computed by ``mbx_energy`` (include/mbx_b200.h) on the GPU; nothing here
computes them on the CPU.

``precision`` selects the FP64 kernels (default) or the mixed kernels (FP32
monomials with FP64 accumulation).
"""
import json

import numpy as np

from . import capi
from .specs import MONOMER_ATOM_NAMES, MONOMER_ATOMS
from .topology import Topology


class CUException(RuntimeError):
    """Mirrors the reference's CUException (tools/custom_exceptions.h)."""


class System:
    def __init__(self, device=0, context=None):
        self._ids = []
        self._xyz = []
        self._islocal = []
        self._molecules = []
        self.initialized = False
        self.cutoff2b = 100.0   # System::System defaults (bblock/system.cpp:63-133)
        self.cutoff3b = 5.0
        self.box = []
        self.ignore_1b = []
        self.ignore_2b = []
        self.ignore_3b = []
        self.precision = "fp64"
        self.device = device
        self._ctx = context
        self.grad = None
        self.virial = np.zeros(9)
        self.energy = 0.0

    # ------------------------------------------------------------ set-up
    def AddMonomer(self, xyz, atoms, id, islocal=1, tag=0):
        if self.initialized:
            raise CUException("The system has already been initialized. Adding a new monomer is not possible")
        if id not in MONOMER_ATOMS:
            raise CUException("Monomer %s is not supported on this path" % id)
        xyz = np.asarray(xyz, np.float64).reshape(-1)
        if len(xyz) != 3 * MONOMER_ATOMS[id] or len(atoms) != MONOMER_ATOMS[id]:
            raise CUException("monomer %s needs %d atoms" % (id, MONOMER_ATOMS[id]))
        self._ids.append(id)
        self._xyz.append(xyz)
        self._islocal.append(int(islocal))

    def AddMolecule(self, molec):
        self._molecules.append(list(molec))

    def Initialize(self):
        if self.initialized:
            raise CUException("The system has already been initialized. Reinitialization is not possible")
        if not self._ids:
            raise CUException("Monomer vector cannot be empty.")
        self.top = Topology(self._ids, self._islocal)
        self.sites = self.top.sites_from_input(np.concatenate(self._xyz))
        self.grad = np.zeros_like(self.sites)
        if self._ctx is None:
            self._ctx = capi.Context(self.device)
        t = self.top
        self._ctx.set_topology(t.ids, t.first_index, t.tag, t.is_local, t.numsites)
        self._ctx.set_real_order(t.site_of_input_atom)
        self.initialized = True
        self._push_config()

    def SetUpFromJson(self, json_text=None):
        """Reads the "MBX" block (bblock/system.cpp:1198-1580): box, cutoffs, ignore lists."""
        cfg = {}
        if json_text:
            cfg = json.loads(json_text) if isinstance(json_text, str) else dict(json_text)
        m = cfg.get("MBX", {})
        self.box = list(m.get("box", []))
        self.cutoff2b = float(m.get("twobody_cutoff", 100.0))
        self.cutoff3b = float(m.get("threebody_cutoff", 5.0))
        self.ignore_1b = [str(t) for t in m.get("ignore_1b_poly", [])]
        self.ignore_2b = [list(t) for t in m.get("ignore_2b_poly", [])]
        self.ignore_3b = [list(t) for t in m.get("ignore_3b_poly", [])]
        if not self.initialized:
            self.Initialize()
        else:
            self._push_config()

    def Set2bCutoff(self, c):
        self.cutoff2b = float(c)
        self._push_config()

    def Set3bCutoff(self, c):
        self.cutoff3b = float(c)
        self._push_config()

    def SetPBC(self, box=()):
        if len(box) not in (0, 9):
            raise CUException("Box size of %d is not acceptable." % len(box))
        self.box = list(box)
        self._push_config()

    def _push_config(self):
        if not self.initialized:
            return
        box = np.asarray(self.box, np.float64) if len(self.box) else None
        try:
            self._ctx.set_config(self.cutoff2b, self.cutoff3b, box, self.ignore_2b, self.ignore_3b)
            self._ctx.set_ignore_1b(self.ignore_1b)
        except capi.MBXError as e:
            raise CUException(str(e))

    def SetRealXyz(self, xyz):
        self.sites = self.top.sites_from_input(xyz)

    def SetXyz(self, sites):
        self.sites = np.asarray(sites, np.float64).reshape(-1).copy()

    # ------------------------------------------------------------ energies
    def _term(self, nbody, do_grads, use_ghost):
        if not self.initialized:
            raise CUException("System has not been initialized. %dB Energy calculation not possible." % nbody)
        self.grad[:] = 0.0
        self.virial[:] = 0.0
        self.energy = self._ctx.energy(nbody, self.sites, self.grad if do_grads else None, self.virial,
                                       use_ghost=use_ghost, mixed=self.precision == "mixed", grads=do_grads)
        return self.energy

    def OneBodyEnergy(self, do_grads):
        """System::OneBodyEnergy (bblock/system.cpp:2140): the 1-body term of
        the local monomers (water: Partridge-Schwenke) on the GPU."""
        return self._term(1, do_grads, False)

    def TwoBodyEnergy(self, do_grads, use_ghost=False):
        return self._term(2, do_grads, use_ghost)

    def ThreeBodyEnergy(self, do_grads, use_ghost=False):
        return self._term(3, do_grads, use_ghost)

    def EnergyFromRealXyz(self, nbody, xyz_real, grad_real=None, do_grads=True, use_ghost=False):
        """The nbody term (1, 2, 3) on real coordinates in input order -- a
        CUDA tensor for a GPU-resident caller (i-PI, LAMMPS) or a numpy
        array -- without copying them into the System (SetRealXyz followed
        by OneBody/TwoBody/ThreeBodyEnergy, with the gradient accumulated
        into grad_real in input order, GetRealGrads).  The System's own
        coordinates, gradient and virial are not touched; returns (energy,
        virial)."""
        if not self.initialized:
            raise CUException("System has not been initialized. %dB Energy calculation not possible." % nbody)
        vir = np.zeros(9)
        e = self._ctx.energy_real(nbody, xyz_real, grad_real if do_grads else None, vir, use_ghost=use_ghost,
                                  mixed=self.precision == "mixed", grads=do_grads)
        return e, vir

    def TwoAndThreeBodyEnergy(self, do_grads, use_ghost=False):
        """Both terms in one call (no counterpart in the reference, whose
        Energy() runs Get2B and Get3B one after the other): the 2b and 3b
        terms run side by side on the GPU.  Returns (E2B, E3B); the gradient
        and virial hold their sum."""
        if not self.initialized:
            raise CUException("System has not been initialized. 2B/3B Energy calculation not possible.")
        self.grad[:] = 0.0
        self.virial[:] = 0.0
        e2, e3 = self._ctx.energy_2b3b(self.sites, self.grad if do_grads else None, self.virial,
                                       use_ghost=use_ghost, mixed=self.precision == "mixed", grads=do_grads)
        self.energy = e2 + e3
        return e2, e3

    # ------------------------------------------------------------ getters
    def GetRealGrads(self):
        return self.top.input_from_sites(self.grad)

    def GetGrads(self):
        return self.grad.copy()

    def GetVirial(self):
        return self.virial.copy()

    def GetXyz(self):
        return self.sites.copy()

    def GetRealXyz(self):
        return self.top.input_from_sites(self.sites)

    def GetPairList(self, nmax, cutoff, istart=0, iend=None, use_ghost=False):
        """n-mers in input monomer indices, each sorted, rows sorted (system.cpp:313)."""
        if nmax not in (2, 3):
            raise CUException("nmax value of %d is not acceptable. Possible values are 2 or 3." % nmax)
        nm = self._ctx.nmers(nmax, cutoff, self.sites, use_ghost)
        return self.top.nmers_to_input(nm)

    def NmerCounts(self, nbody):
        """(listed, evaluated) n-mers of the last energy call."""
        return self._ctx.counts(nbody)


def from_arrays(ids, xyz, box=None, cutoff2b=9.0, cutoff3b=7.0, ignore_2b=(), ignore_3b=(), device=0,
                precision="fp64", context=None):
    """Builds an initialised System from monomer ids and input-order coordinates."""
    from .specs import MONOMER_ATOMS as NAT
    names = {m: list(v) for m, v in MONOMER_ATOM_NAMES.items()}
    s = System(device, context)
    xyz = np.asarray(xyz, np.float64).reshape(-1)
    off = 0
    for i, m in enumerate(ids):
        n = 3 * NAT[m]
        s.AddMonomer(xyz[off:off + n], names[m], m)
        s.AddMolecule([i])
        off += n
    s.Initialize()
    s.SetUpFromJson({"MBX": {"box": [] if box is None else list(np.asarray(box).reshape(-1)),
                             "twobody_cutoff": cutoff2b, "threebody_cutoff": cutoff3b,
                             "ignore_2b_poly": [list(t) for t in ignore_2b],
                             "ignore_3b_poly": [list(t) for t in ignore_3b]}})
    s.precision = precision
    return s
