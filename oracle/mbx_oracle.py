"""CPU oracle for the 2-body/3-body path (restatement of the reference).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker, never by the product.

The arithmetic lives in ``mbx_oracle.c`` (compiled to
``oracle/_build/libmbx_oracle.so``); this module restates the orchestration of
``System::TwoBodyEnergy/ThreeBodyEnergy`` -> ``Get2B/Get3B``
(bblock/system.cpp:2403-2725, 2727-3073):

1. ``SetPBC``: wrap every monomer with ``FixMonomerCoordinates``
   (bblock/system.cpp:741-744), in place, on every call;
2. ``AddClusters`` over the monomers' first atoms (bblock/sys_tools.cpp:472);
3. per n-mer: gather the real atoms, move monomers 2 (and 3) to the image
   closest to monomer 1 (``GetCloseDimerImage/GetCloseTrimerImage``,
   bblock/sys_tools.cpp:322-366,438-442), skip ignored type tuples
   (bblock/system.cpp:2606-2618, 2940-2952), sort the monomer ids as
   ``e2b::get_2b_energy`` / ``e3b::get_3b_energy`` do
   (potential/2b/energy2b.cpp:240-254, potential/3b/energy3b.cpp:185-216) and
   evaluate; unknown tuples contribute 0;
4. accumulate energy, ``grad_`` (real atoms only) and ``virial_``.
"""
import ctypes
import os
import subprocess

import numpy as np

from mbx_b200.specs import SPECS, DISPATCH_2B, DISPATCH_3B, LP_GAMMA_IN, LP_GAMMA_OUT
from mbx_b200.specs import dispatch as dispatch_nmer
from mbx_b200.tables import load_pip, load_fit
from mbx_b200.topology import Topology

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libmbx_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmbx_ref.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libmbx_ref_gpu.so")


def build(force=False):
    """Compile mbx_oracle.c (needs gcc).  Returns the library path."""
    src = os.path.join(HERE, "mbx_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-o", LIB, src,
                               "-lm"])
    return LIB


class _Spec(ctypes.Structure):
    _fields_ = [
        ("nbody", ctypes.c_int), ("nreal", ctypes.c_int), ("nsites", ctypes.c_int), ("nat", ctypes.c_int * 3),
        ("nlp", ctypes.c_int), ("lp", (ctypes.c_int * 4) * 3), ("nvars", ctypes.c_int),
        ("vkind", ctypes.c_int * 128), ("vs1", ctypes.c_int * 128), ("vs2", ctypes.c_int * 128),
        ("vk", ctypes.c_double * 128), ("vd", ctypes.c_double * 128), ("sw_triple", ctypes.c_int),
        ("ri", ctypes.c_double), ("rf", ctypes.c_double), ("skip", ctypes.c_int),
        ("gin", ctypes.c_double), ("gout", ctypes.c_double), ("virial_raw", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "mbx_oracle.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lp = ctypes.POINTER(ctypes.c_long)
        L.mbxo_invert_box.argtypes = [dp, dp]
        L.mbxo_fix_monomers.argtypes = [ctypes.c_int, lp, ip, dp, dp, dp]
        L.mbxo_close_image.argtypes = [dp, dp, dp, ctypes.c_int, dp]
        L.mbxo_add_clusters.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, dp, lp,
                                        ip, ctypes.c_int, lp, ctypes.c_long]
        L.mbxo_add_clusters.restype = ctypes.c_long
        L.mbxo_pip_eval.argtypes = [ctypes.c_int, ctypes.c_long, ip, dp, ip, ip, ctypes.c_int, dp, dp, dp]
        L.mbxo_pip_eval.restype = ctypes.c_double
        L.mbxo_holder_eval.argtypes = [ctypes.POINTER(_Spec), ctypes.c_long, ip, dp, ip, ip, ctypes.c_int, dp,
                                       ctypes.c_long, dp, dp, dp, dp]
        L.mbxo_holder_eval.restype = ctypes.c_double
        L.mbxo_holder_dcoef.argtypes = [ctypes.POINTER(_Spec), ctypes.c_int, ctypes.c_long, ip, dp, ip, ip, ctypes.c_int,
                                        dp, dp]
        L.mbxo_holder_dcoef.restype = ctypes.c_int
        L.mbxo_spec_size.restype = ctypes.c_long
        L.mbxo_holder_vars.argtypes = [ctypes.POINTER(_Spec), ctypes.c_long, dp, dp,
                                       ctypes.POINTER(ctypes.c_ubyte)]
        L.mbxo_holder_vars.restype = ctypes.c_long
        assert L.mbxo_spec_size() == ctypes.sizeof(_Spec)
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def _ip(a):
    return _p(a, ctypes.c_int)


def _lp(a):
    return _p(a, ctypes.c_long)


_spec_cache = {}


def c_spec(name):
    if name in _spec_cache:
        return _spec_cache[name]
    s = SPECS[name]
    cs = _Spec()
    cs.nbody = s.nbody
    cs.nreal = s.nreal
    cs.nsites = len(s.sites)
    for i, n in enumerate(s.nat):
        cs.nat[i] = n
    cs.nlp = len(s.lp)
    for i, l in enumerate(s.lp):
        for j in range(4):
            cs.lp[i][j] = l[j]
    cs.nvars = s.nvars
    for v, (kind, a, b, k, d0) in enumerate(s.variables):
        cs.vkind[v] = 0 if kind == "exp" else 1
        cs.vs1[v] = a
        cs.vs2[v] = b
        cs.vk[v] = k
        cs.vd[v] = d0
    cs.sw_triple = {"pair": 0, "triple": 1, "triple2": 2, "cos2": 3}[s.switch]
    cs.ri = s.ri
    cs.rf = s.rf
    cs.skip = {"pair_gt": 0, "two_of_three_gt": 1, "all_three_gt": 2}[s.skip]
    cs.virial_raw = 1 if s.virial == "raw" else 0
    cs.gin = LP_GAMMA_IN
    cs.gout = LP_GAMMA_OUT
    _spec_cache[name] = cs
    return cs


def pip_eval(name, a, x, want_grad=True):
    """Generated polynomial P(a, x) (and dP/dx) for one configuration."""
    t = load_pip(name)
    x = np.ascontiguousarray(x, np.float64)
    a = np.ascontiguousarray(a, np.float64)
    g = np.zeros(t.nvars) if want_grad else None
    e = lib().mbxo_pip_eval(t.nvars, t.nterms, _ip(t.k), _p(t.coef), _ip(t.deg), _ip(np.ascontiguousarray(t.var)),
                            t.var.shape[1], _p(a), _p(x), _p(g))
    return (e, g) if want_grad else e


def holder_eval(name, xyz, do_grads=True, a=None, per_nmer=False):
    """Evaluator (holder) for n n-mers; xyz: [n, nreal*3] in holder order, imaged.

    Returns (E_sum, grad [n, nreal*3] or None, virial[9], e_per or None)."""
    t = load_pip(name)
    s = SPECS[name]
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, s.nreal * 3)
    n = len(xyz)
    a = load_fit(name) if a is None else np.ascontiguousarray(a, np.float64)
    grad = np.zeros_like(xyz) if do_grads else None
    vir = np.zeros(9)
    eper = np.zeros(n) if per_nmer else None
    e = lib().mbxo_holder_eval(ctypes.byref(c_spec(name)), t.nterms, _ip(t.k), _p(t.coef), _ip(t.deg),
                               _ip(np.ascontiguousarray(t.var)), t.var.shape[1], _p(a), n, _p(xyz), _p(grad),
                               _p(vir) if do_grads else None, _p(eper))
    return e, grad, vir, eper


def holder_vars(name, xyz):
    """Polynomial variables of every n-mer (mbxo_holder_vars): (x[n][nvars],
    live[n]); x is 0 for n-mers beyond the evaluator's cutoff."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    spec = c_spec(name)
    n = xyz.shape[0]
    x = np.zeros((n, spec.nvars))
    live = np.zeros(n, dtype=np.uint8)
    lib().mbxo_holder_vars(ctypes.byref(spec), ctypes.c_long(n), _p(xyz), _p(x),
                           live.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
    return x, live.astype(bool)


def holder_dcoef(name, xyz):
    """dE/da for each n-mer: [n, ncoef] (switched monomial sums)."""
    t = load_pip(name)
    s = SPECS[name]
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, s.nreal * 3)
    out = np.zeros((len(xyz), s.ncoef))
    for i in range(len(xyz)):
        lib().mbxo_holder_dcoef(ctypes.byref(c_spec(name)), s.ncoef, t.nterms, _ip(t.k), _p(t.coef), _ip(t.deg),
                                _ip(np.ascontiguousarray(t.var)), t.var.shape[1], _p(xyz[i]), _p(out[i]))
    return out


def invert_box(box):
    box = np.ascontiguousarray(box, np.float64)
    inv = np.zeros(9)
    if lib().mbxo_invert_box(_p(box), _p(inv)) != 0:
        raise ValueError("Matrix has no inverse. Determinant is 0")
    return inv


def _frac(inv, p):
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return np.stack([inv[0] * x + inv[3] * y + inv[6] * z, inv[1] * x + inv[4] * y + inv[7] * z,
                     inv[2] * x + inv[5] * y + inv[8] * z], axis=-1)


def _cart(box, f):
    u, v, w = f[..., 0], f[..., 1], f[..., 2]
    return np.stack([box[0] * u + box[3] * v + box[6] * w, box[1] * u + box[4] * v + box[7] * w,
                     box[2] * u + box[5] * v + box[8] * w], axis=-1)


def close_image(box, inv, first1, xyz2):
    """GetCloseDimerImage (bblock/sys_tools.cpp:322-366), vectorised over n-mers.

    first1: [n, 3] first atom of monomer 1; xyz2: [n, 3*nat2].  numpy evaluates
    the same left-to-right products and sums as the reference (no FMA)."""
    n = len(xyz2)
    q = xyz2.reshape(n, -1, 3)
    f1 = _frac(inv, first1)
    f20 = _frac(inv, q[:, 0, :])
    d = np.floor(f20 - f1 + 0.5)
    f = _frac(inv, q) - d[:, None, :]
    return np.ascontiguousarray(_cart(box, f).reshape(n, -1))


def add_clusters(nmax, cutoff, first_atoms, tag, is_local, box=None, use_ghost=False):
    """n-mer list (internal monomer indices) exactly as AddClusters builds it."""
    first_atoms = np.ascontiguousarray(first_atoms, np.float64).reshape(-1)
    nmon = len(first_atoms) // 3
    use_pbc = box is not None
    boxa = np.ascontiguousarray(box if use_pbc else np.zeros(9), np.float64)
    inv = invert_box(boxa) if use_pbc else np.zeros(9)
    tag = np.ascontiguousarray(tag, np.int64)
    is_local = np.ascontiguousarray(is_local, np.int32)
    L = lib()
    cap = 1 << 16
    while True:
        out = np.zeros(cap * nmax, np.int64)
        n = L.mbxo_add_clusters(nmax, cutoff, nmon, int(use_pbc), _p(boxa), _p(inv), _p(first_atoms), _lp(tag),
                                _ip(is_local), int(use_ghost), _lp(out), cap)
        if n <= cap:
            return out[:n * nmax].reshape(n, nmax)
        cap = n


def get_nb_energy(ids, xyzs, nm, do_grads=True):
    """e2b::get_2b_energy / e3b::get_3b_energy (potential/2b/energy2b.cpp:206,
    potential/3b/energy3b.cpp:139): nm n-mers of monomers ids, coordinates per
    slot xyzs[s] ([nm * 3 * nat_s]), not imaged.  Returns (E, grads per slot,
    virial); unknown tuples give 0."""
    name, order = dispatch_nmer(list(ids))
    blocks = [np.asarray(x, np.float64).reshape(nm, -1) for x in xyzs]
    if name is None:
        return 0.0, [np.zeros_like(b) for b in blocks], np.zeros(9)
    xyz = np.concatenate([blocks[o] for o in order], axis=1)
    e, g, vir, _ = holder_eval(name, xyz, do_grads)
    grads = [None] * len(ids)
    off = 0
    for o in order:
        w = blocks[o].shape[1]
        grads[o] = g[:, off:off + w] if do_grads else np.zeros_like(blocks[o])
        off += w
    return e, grads, vir


class OracleSystem:
    """The reference's System, reduced to what TwoBodyEnergy/ThreeBodyEnergy use."""

    def __init__(self, mon_ids, xyz, box=None, cutoff2b=9.0, cutoff3b=7.0, ignore_2b=(), ignore_3b=(),
                 is_local=None):
        self.top = Topology(mon_ids, is_local)
        self.sites = self.top.sites_from_input(xyz)
        self.box = None if box is None or len(box) == 0 else np.asarray(box, np.float64).reshape(9).copy()
        self.cutoff2b = float(cutoff2b)
        self.cutoff3b = float(cutoff3b)
        self.ignore_2b = [sorted(t) for t in ignore_2b]
        self.ignore_3b = [sorted(t) for t in ignore_3b]
        self.grad = np.zeros(3 * self.top.numsites)
        self.virial = np.zeros(9)

    def set_real_xyz(self, xyz):
        self.sites = self.top.sites_from_input(xyz)

    def _set_pbc(self):
        if self.box is None:
            return
        inv = invert_box(self.box)
        t = self.top
        lib().mbxo_fix_monomers(t.nmon, _lp(np.ascontiguousarray(t.first_index)), _ip(np.ascontiguousarray(t.nat)),
                                _p(self.box), _p(inv), _p(self.sites))

    def first_atoms(self):
        return self.sites.reshape(-1, 3)[self.top.first_index].reshape(-1)

    def nmers(self, nmax, cutoff=None, use_ghost=False):
        cutoff = (self.cutoff2b if nmax == 2 else self.cutoff3b) if cutoff is None else cutoff
        return add_clusters(nmax, cutoff, self.first_atoms(), self.top.tag, self.top.is_local, self.box, use_ghost)

    def energy(self, nbody, do_grads=True, use_ghost=False, per_type=None):
        """TwoBodyEnergy / ThreeBodyEnergy: returns the energy; fills grad, virial."""
        self.grad[:] = 0.0
        self.virial[:] = 0.0
        self._set_pbc()
        nm = self.nmers(nbody, use_ghost=use_ghost)
        return self._evaluate(nbody, nm, do_grads, per_type)

    def _evaluate(self, nbody, nm, do_grads, per_type):
        t = self.top
        sites = self.sites.reshape(-1, 3)
        inv = invert_box(self.box) if self.box is not None else None
        ignore = self.ignore_2b if nbody == 2 else self.ignore_3b
        etot = 0.0
        if len(nm) == 0:
            return 0.0
        codes = t.type_code[nm]
        keys, inverse = np.unique(codes, axis=0, return_inverse=True)
        inverse = np.asarray(inverse).reshape(-1)
        for g, key in enumerate(keys):
            types = tuple(t.type_order[c] for c in key)
            if sorted(types) in ignore:
                continue
            name, slots = dispatch_nmer(list(types))
            if name is None:
                continue
            sel = nm[inverse == g]
            nats = [int(t.nat[sel[0, s]]) for s in range(nbody)]
            # gather in original slot order, image relative to slot 0
            blocks = []
            for s in range(nbody):
                idx = t.first_index[sel[:, s]][:, None] + np.arange(nats[s])[None, :]
                blocks.append(np.ascontiguousarray(sites[idx].reshape(len(sel), -1)))
            if self.box is not None:
                for s in range(1, nbody):
                    blocks[s] = close_image(self.box, inv, blocks[0][:, :3], blocks[s])
            xyz = np.concatenate([blocks[s] for s in slots], axis=1)
            e, grad, vir, _ = holder_eval(name, xyz, do_grads)
            etot += e
            if per_type is not None:
                per_type[name] = per_type.get(name, 0.0) + e
            if do_grads:
                self.virial += vir
                off = 0
                for s in slots:
                    n3 = 3 * nats[s]
                    idx = (3 * t.first_index[sel[:, s]])[:, None] + np.arange(n3)[None, :]
                    np.add.at(self.grad, idx, grad[:, off:off + n3])
                    off += n3
        return etot

    def real_grads(self):
        """Gradients of the real atoms in input order (GetRealGrads)."""
        return self.top.input_from_sites(self.grad)


class RefSystem:
    """bblock::System from the reference library (oracle/_ref), via ref_harness.cpp."""

    _L = None
    LIB = REF_LIB

    @classmethod
    def available(cls):
        return os.path.exists(cls.LIB)

    @classmethod
    def L(cls):
        if cls._L is None:
            L = ctypes.CDLL(cls.LIB)
            dp = ctypes.POINTER(ctypes.c_double)
            L.mbxref_new.argtypes = [ctypes.c_char_p, dp, ctypes.c_char_p]
            L.mbxref_new.restype = ctypes.c_void_p
            L.mbxref_free.argtypes = [ctypes.c_void_p]
            L.mbxref_last_error.restype = ctypes.c_char_p
            L.mbxref_energy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
            L.mbxref_real_grads.argtypes = [ctypes.c_void_p, dp]
            L.mbxref_virial.argtypes = [ctypes.c_void_p, dp]
            L.mbxref_set_real_xyz.argtypes = [ctypes.c_void_p, dp]
            L.mbxref_num_real_sites.argtypes = [ctypes.c_void_p]
            L.mbxref_pair_list.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                           ctypes.POINTER(ctypes.c_ulong), ctypes.c_long]
            L.mbxref_pair_list.restype = ctypes.c_long
            L.mbxref_set_threads.argtypes = [ctypes.c_int]
            L.mbxref_poly.argtypes = [ctypes.c_int, dp, dp, dp]
            L.mbxref_poly.restype = ctypes.c_double
            L.mbxref_get_2b.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long, dp, dp, ctypes.c_long,
                                        ctypes.c_long, dp, dp, dp]
            L.mbxref_get_2b.restype = ctypes.c_double
            L.mbxref_get_3b.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_long, dp, dp, dp] + [ctypes.c_long] * 3 + \
                                       [dp, dp, dp, dp]
            L.mbxref_get_3b.restype = ctypes.c_double
            cls._L = L
        return cls._L

    def __init__(self, mon_ids, xyz, box=None, cutoff2b=9.0, cutoff3b=7.0, ignore_2b=(), ignore_3b=()):
        import json
        cfg = {"twobody_cutoff": cutoff2b, "threebody_cutoff": cutoff3b,
               "ignore_2b_poly": [list(t) for t in ignore_2b], "ignore_3b_poly": [list(t) for t in ignore_3b],
               "max_n_eval_2b": 1024, "max_n_eval_3b": 1024}
        if box is not None and len(box):
            cfg["box"] = [float(v) for v in np.asarray(box).reshape(-1)]
        else:
            cfg["box"] = []
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        self.nat = len(xyz) // 3
        self.h = self.L().mbxref_new(" ".join(mon_ids).encode(), _p(xyz), json.dumps({"MBX": cfg}).encode())
        if not self.h:
            raise RuntimeError(self.L().mbxref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            self.L().mbxref_free(self.h)
            self.h = None

    def set_real_xyz(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        self.L().mbxref_set_real_xyz(self.h, _p(xyz))

    def energy(self, nbody, do_grads=True):
        e = ctypes.c_double()
        if self.L().mbxref_energy(self.h, nbody, int(do_grads), ctypes.byref(e)) != 0:
            raise RuntimeError(self.L().mbxref_last_error().decode())
        return e.value

    def real_grads(self):
        g = np.zeros(3 * self.nat)
        self.L().mbxref_real_grads(self.h, _p(g))
        return g

    def virial(self):
        v = np.zeros(9)
        self.L().mbxref_virial(self.h, _p(v))
        return v

    def pair_list(self, nmax, cutoff):
        """n-mers in input monomer indices, each sorted, rows sorted (sortEdge rule)."""
        n = self.L().mbxref_pair_list(self.h, nmax, cutoff, None, 0)
        out = np.zeros(max(n, 1), np.uint64)
        self.L().mbxref_pair_list(self.h, nmax, cutoff, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulong)), n)
        nm = out[:n].astype(np.int64).reshape(-1, nmax)
        nm = np.sort(nm, axis=1)
        return nm[np.lexsort(nm.T[::-1])] if len(nm) else nm

    @classmethod
    def poly(cls, kind, a, x, want_grad=True):
        a = np.ascontiguousarray(a, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        g = np.zeros(len(x)) if want_grad else None
        e = cls.L().mbxref_poly(kind, _p(a), _p(x), _p(g))
        return (e, g) if want_grad else e

    @classmethod
    def set_threads(cls, n):
        cls.L().mbxref_set_threads(n)


class RefGpuSystem(RefSystem):
    """The reference's bblock::System with Get2B/Get3B forwarded to the CUDA
    library over its C ABI (oracle/build_ref_gpu.py, oracle/ref_gpu_glue.cpp):
    the C++ caller of the drop-in boundary."""

    _L = None
    LIB = REF_GPU_LIB
