"""Monomer bookkeeping of ``bblock::System``, restated for the 2-body/3-body path.

The reference stores monomers in an internal order: monomer types sorted by
ascending count (ties keep first appearance), input order within a type
(``systools::OrderMonomers``, bblock/sys_tools.cpp:44-131).  Coordinates live in
a site array that also holds each monomer's electrostatic virtual sites
(h2o: O H H M; ch4: C H H H H), ``first_index_`` giving the first site of each
monomer (``System::AddMonomerInfo``, bblock/system.cpp:1794-1969).  Every real
atom carries a tag equal to its position in the input (``System::AddMonomer``,
bblock/system.cpp:848-870); the n-mer search compares the tags of the monomers'
first atoms (bblock/sys_tools.cpp:562,585).
"""
import numpy as np

from .specs import MONOMER_ATOMS, MONOMER_SITES


class Topology:
    def __init__(self, mon_ids, is_local=None):
        mon_ids = list(mon_ids)
        if not mon_ids:
            raise ValueError("Monomer vector cannot be empty.")
        for m in mon_ids:
            if m not in MONOMER_ATOMS:
                raise ValueError("unknown monomer id %r (supported: %s)" % (m, sorted(MONOMER_ATOMS)))
        self.input_ids = mon_ids
        n = len(mon_ids)
        if is_local is None:
            is_local = [1] * n
        nat_in = [MONOMER_ATOMS[m] for m in mon_ids]
        atom_start_in = np.concatenate([[0], np.cumsum(nat_in)[:-1]]).astype(np.int64)
        # type order: ascending count, ties by first appearance (strict <)
        types = []
        for m in mon_ids:
            if m not in types:
                types.append(m)
        counts = [(t, mon_ids.count(t)) for t in types]
        order = []
        while counts:
            best = 0
            for i in range(1, len(counts)):
                if counts[i][1] < counts[best][1]:
                    best = i
            order.append(counts.pop(best)[0])
        internal = [i for t in order for i in range(n) if mon_ids[i] == t]
        self.type_order = order
        self.internal_to_input = np.array(internal, np.int64)
        self.input_to_internal = np.empty(n, np.int64)
        self.input_to_internal[self.internal_to_input] = np.arange(n)
        self.ids = [mon_ids[i] for i in internal]
        self.nat = np.array([MONOMER_ATOMS[m] for m in self.ids], np.int32)
        self.nsites = np.array([MONOMER_SITES[m] for m in self.ids], np.int32)
        self.first_index = np.concatenate([[0], np.cumsum(self.nsites)[:-1]]).astype(np.int64)
        self.numsites = int(self.nsites.sum())
        self.numat = int(self.nat.sum())
        self.tag = atom_start_in[self.internal_to_input].astype(np.int64)
        self.is_local = np.array([int(is_local[i]) for i in internal], np.int32)
        self.atom_start_in = atom_start_in
        self.type_code = np.array([order.index(m) for m in self.ids], np.int32)
        # site index (internal) of every real atom, listed in input atom order
        site_of_input_atom = np.empty(self.numat, np.int64)
        for pos, i in enumerate(internal):
            a0 = atom_start_in[i]
            for j in range(nat_in[i]):
                site_of_input_atom[a0 + j] = self.first_index[pos] + j
        self.site_of_input_atom = site_of_input_atom

    @property
    def nmon(self):
        return len(self.ids)

    def sites_from_input(self, xyz_in):
        """Real-atom coordinates (input order, 3 per atom) -> site array (internal)."""
        xyz_in = np.asarray(xyz_in, np.float64).reshape(-1, 3)
        if len(xyz_in) != self.numat:
            raise ValueError("expected %d atoms, got %d" % (self.numat, len(xyz_in)))
        sites = np.zeros((self.numsites, 3))
        sites[self.site_of_input_atom] = xyz_in
        return sites.reshape(-1)

    def input_from_sites(self, site_arr):
        """Site array (internal, 3 per site) -> real atoms in input order."""
        return np.asarray(site_arr).reshape(-1, 3)[self.site_of_input_atom].reshape(-1)

    def nmers_to_input(self, nmers):
        """Internal monomer indices -> input indices, each n-mer sorted, rows sorted."""
        nm = self.internal_to_input[np.asarray(nmers, np.int64)]
        if nm.size == 0:
            return nm.reshape(0, nm.shape[1] if nm.ndim == 2 else 0)
        nm = np.sort(nm, axis=1)
        return nm[np.lexsort(nm.T[::-1])]
