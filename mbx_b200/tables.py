"""Loader for the PIP term tables and fitted coefficients in ``mbx_b200/data``.

``<name>.pip.gz`` holds one line per term ``k coef deg v1 .. v_deg`` meaning
``P(a, x) = sum a[k] * coef * x[v1] * ... * x[v_deg]`` (produced from the
reference's generated programs by ``codegen/pip_extract.py``); ``<name>.fit``
holds the fitted linear coefficients ``a`` of the model, one per line.
"""
import functools
import gzip
import os

import numpy as np

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


class PipTable:
    def __init__(self, name, nvars, ncoef, degree, k, coef, deg, var):
        self.name = name
        self.nvars = nvars
        self.ncoef = ncoef
        self.degree = degree
        self.k = k          # int32 [nterms]
        self.coef = coef    # float64 [nterms]
        self.deg = deg      # int32 [nterms]
        self.var = var      # int32 [nterms, 4], -1 padded

    @property
    def nterms(self):
        return len(self.k)


@functools.lru_cache(maxsize=None)
def load_pip(name):
    """Term table of an evaluator (its shared table where it has one) or of a
    table name.  var[t, :deg[t]] are the variables of term t; the array is
    max(4, degree) wide."""
    from .specs import SPECS
    if name in SPECS:
        name = SPECS[name].pip_table
    path = os.path.join(DATA, name + ".pip.gz")
    with gzip.open(path, "rt") as f:
        f.readline()
        nvars, ncoef, degree, nterms = map(int, f.readline().split())
        k = np.empty(nterms, np.int32)
        coef = np.empty(nterms, np.float64)
        deg = np.empty(nterms, np.int32)
        var = np.full((nterms, max(4, degree)), -1, np.int32)
        for t, line in enumerate(f):
            p = line.split()
            k[t] = int(p[0])
            coef[t] = float(p[1])
            d = int(p[2])
            deg[t] = d
            for i in range(d):
                var[t, i] = int(p[3 + i])
    if t + 1 != nterms:
        raise ValueError("%s: expected %d terms, read %d" % (path, nterms, t + 1))
    return PipTable(name, nvars, ncoef, degree, k, coef, deg, var)


@functools.lru_cache(maxsize=None)
def load_fit(name):
    """Fitted linear coefficients of an evaluator (an alias evaluator of
    specs.KERNEL_ALIASES without a fit of its own has its target's)."""
    from mbx_b200.specs import KERNEL_ALIASES
    if name in KERNEL_ALIASES and not os.path.exists(os.path.join(DATA, name + ".fit")):
        name = KERNEL_ALIASES[name]
    with open(os.path.join(DATA, name + ".fit")) as f:
        return np.array([float(v) for v in f.read().split()], np.float64)
