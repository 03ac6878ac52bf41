"""Batched configurations: many independent systems evaluated together.

No counterpart in the reference, which evaluates one ``bblock::System`` per
call; this is the batched form for path-integral beads, cluster sets and other
independent configurations (``mbx_set_batch`` / ``mbx_batch_energy`` in
``include/mbx_b200.h``).  Each configuration keeps the reference's semantics
(its own internal monomer order, tags, box and n-mer lists; n-mers never span
two configurations); the device work of a term is one n-mer build per
configuration and one evaluation launch per evaluator over all of them, and can
be captured once into a CUDA graph and replayed.
"""
import numpy as np

from . import capi
from .topology import Topology


class Batch:
    """configs: [(monomer ids, input-order coordinates, box[9] or None)]."""

    def __init__(self, configs, cutoff2b=9.0, cutoff3b=7.0, device=0, context=None):
        import torch
        self.topos = []
        ids, first, tags, sites = [], [], [], []
        conf_mon, boxes, has_box = [0], [], []
        site_off = atom_off = 0
        for mon_ids, xyz, box in configs:
            t = Topology(mon_ids)
            self.topos.append(t)
            ids += t.ids
            first += list(t.first_index + site_off)
            tags += list(t.tag + atom_off)
            sites.append(t.sites_from_input(xyz))
            conf_mon.append(conf_mon[-1] + t.nmon)
            boxes.append(np.zeros(9) if box is None else np.asarray(box, np.float64).reshape(9))
            has_box.append(0 if box is None else 1)
            site_off += t.numsites
            atom_off += t.numat
        self.site_offsets = np.concatenate([[0], np.cumsum([t.numsites for t in self.topos])])
        self.nconf = len(configs)
        self.ctx = context or capi.Context(device)
        self.ctx.set_topology(ids, first, tags, None, site_off)
        self.ctx.set_config(cutoff2b, cutoff3b, None)
        self.ctx.set_batch(conf_mon, np.array(boxes), np.array(has_box))
        self.sites = torch.tensor(np.concatenate(sites), dtype=torch.float64, device="cuda:%d" % device)
        self.grad = torch.zeros_like(self.sites)

    def energy(self, nbody, grads=True, mixed=False, graph=True, virials=False):
        """Term energies of every configuration (gradients += into self.grad)."""
        return self.ctx.batch_energy(nbody, self.sites, self.grad if grads else None, mixed=mixed, graph=graph,
                                     virials=virials)

    def energy_2b3b(self, grads=True, mixed=False, graph=True, virials=False):
        """Both terms of every configuration side by side: (e2[], e3[])."""
        return self.ctx.batch_energy_2b3b(self.sites, self.grad if grads else None, mixed=mixed, graph=graph,
                                          virials=virials)

    def tune(self, nbody, mixed=False):
        return self.ctx.tune(nbody, self.sites, self.grad, mixed=mixed)

    def real_grads(self, k):
        """Gradient of configuration k on its real atoms, input order (3 per atom)."""
        t = self.topos[k]
        g = self.grad[self.site_offsets[k] * 3:self.site_offsets[k + 1] * 3].cpu().numpy().reshape(-1, 3)
        return g[t.site_of_input_atom].reshape(-1)
