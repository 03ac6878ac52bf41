"""ctypes binding of the C ABI in ``include/mbx_b200.h`` (``libmbx_b200.so``).

This is the Python side of the drop-in boundary: every compute call goes to
the CUDA library.  There is no CPU fallback: when the library is missing it
is built on first use (``mbx_b200/build.py``, nvcc for sm_100a, a few
minutes), and loading fails loudly if that build fails or no CUDA device is
present.
"""
import ctypes
import os
import weakref

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmbx_b200.so")

MBX_DEVICE_PTRS = 1
MBX_MIXED = 2
MBX_NO_GRADS = 4
MBX_GRAPH = 8

EVALUATORS = ("mbpol2b", "mbpol3b", "ch4h2o2b", "ch4ch42b", "ch4h2o3b",
              "h2oli2b", "h2ona2b", "h2ok2b", "h2orb2b", "h2ocs2b",
              "h2oli3b", "h2ona3b", "h2ok3b", "h2orb3b", "h2ocs3b",
              "fh2o2b", "clh2o2b", "brh2o2b", "ih2o2b", "fh2o3b", "clh2o3b", "brh2o3b", "ih2o3b",
              "nana2b", "clcl2b", "arar2b", "nacl2b", "csar2b", "arh2o2b",
              "h2h22b", "h2oh22b", "csh22b", "nh3nh32b", "nh3pbe2b", "ch4co22b", "mbpbe2b", "co23b", "mbpbe3b",
              "co2co22b", "co2a2b", "h2oco22b", "hehe2b", "h2ohe2b", "n2o5h2o2b", "n2o5h2o3b",
              "cm5100co22b", "cm595co22b", "cm590co22b", "cm585co22b", "cm5875co22b", "cm580co22b",
              "h2ocm5100co22b", "h2ocm595co22b", "h2ocm590co22b", "h2ocm585co22b", "h2ocm5875co22b",
              "h2ocm580co22b", "h2oco2a2b")


class MBXError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("mbx_b200 error %d: %s" % (code, msg))
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from mbx_b200 import build
        try:
            build.build(quiet=True)
        except Exception as e:  # noqa: BLE001 -- re-raised with the library path
            raise RuntimeError("mbx_b200 CUDA library %s is missing and could not be built: %s" % (LIB_PATH, e))
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, lp, ip = ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_int)
    cpp = ctypes.POINTER(ctypes.c_char_p)
    L.mbx_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, vp]
    L.mbx_destroy.argtypes = [vp]
    L.mbx_last_error.argtypes = [vp]
    L.mbx_last_error.restype = ctypes.c_char_p
    L.mbx_version.restype = ctypes.c_char_p
    L.mbx_set_topology.argtypes = [vp, ctypes.c_int, cpp, ip, ip, ip, ctypes.c_int]
    L.mbx_set_ignore_1b.argtypes = [vp, ctypes.c_int, cpp]
    L.mbx_set_real_order.argtypes = [vp, ctypes.c_int, ip]
    L.mbx_energy_real.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), dp, dp,
                                  ctypes.c_int]
    L.mbx_set_config.argtypes = [vp, ctypes.c_double, ctypes.c_double, dp, ctypes.c_int, cpp, ctypes.c_int, cpp]
    L.mbx_energy.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), dp, dp,
                             ctypes.c_int]
    L.mbx_last_counts.argtypes = [vp, ctypes.c_int, lp, lp]
    L.mbx_energy_2b3b.argtypes = [vp, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), dp, dp, ctypes.c_int]
    L.mbx_nmers.argtypes = [vp, ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, lp, ctypes.c_long, lp]
    L.mbx_evaluate.argtypes = [vp, ctypes.c_char_p, ctypes.c_long, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_double),
                               ctypes.c_int]
    L.mbx_evaluate_noalloc.argtypes = [ctypes.c_char_p, ctypes.c_long, dp, dp, dp, dp, vp]
    L.mbx_evaluate_dcoef.argtypes = [vp, ctypes.c_char_p, ctypes.c_long, dp, dp, dp, ctypes.c_int]
    L.mbx_poly.argtypes = [vp, ctypes.c_char_p, ctypes.c_long, dp, dp, dp, ctypes.c_int]
    L.mbx_set_coefficients.argtypes = [vp, ctypes.c_char_p, dp, ctypes.c_int]
    L.mbx_evaluator_info.argtypes = [ctypes.c_char_p, ip, ip, ip, ip]
    L.mbx_last_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ip]
    L.mbx_fma_peaks.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.mbx_set_batch.argtypes = [vp, ctypes.c_int, ip, dp, ip]
    L.mbx_batch_energy.argtypes = [vp, ctypes.c_int, dp, dp, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.mbx_tune.argtypes = [vp, ctypes.c_int, dp, dp, ctypes.c_int, ip, ctypes.POINTER(ctypes.c_double)]
    L.mbx_batch_energy_2b3b.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    L.mbx_get_knobs.argtypes = [vp, ctypes.c_int, ip]
    L.mbx_set_knobs.argtypes = [vp, ctypes.c_int, ip]
    L.mbx_qf_image.argtypes = [ctypes.c_char_p, dp, lp, ip, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), dp]
    _lib = L
    return L


EXPORTED = ("mbx_create", "mbx_destroy", "mbx_last_error", "mbx_version", "mbx_set_topology", "mbx_set_config",
            "mbx_energy", "mbx_last_counts", "mbx_nmers", "mbx_evaluate", "mbx_evaluate_dcoef", "mbx_poly",
            "mbx_set_coefficients", "mbx_evaluator_info", "mbx_last_timing", "mbx_fma_peaks", "mbx_set_batch",
            "mbx_batch_energy", "mbx_tune", "mbx_get_knobs", "mbx_set_knobs", "mbx_energy_2b3b",
            "mbx_batch_energy_2b3b", "mbx_set_ignore_1b", "mbx_set_real_order", "mbx_energy_real", "mbx_qf_image")

KNOBS = ("nb_warps", "nb_unroll", "tri_threads", "dim_threads")


def evaluator_info(name):
    nb, nr, nv, nc = (ctypes.c_int() for _ in range(4))
    if lib().mbx_evaluator_info(name.encode(), ctypes.byref(nb), ctypes.byref(nr), ctypes.byref(nv),
                                ctypes.byref(nc)) != 0:
        raise MBXError(95, "unknown evaluator %s" % name)
    return nb.value, nr.value, nv.value, nc.value


def qf_image(name, coef=None):
    """Host-built operands of the tensor-core mixed kernel (mbx_qf_image): the
    B image (bytes), the per-column factors (float32) and the constant term,
    for coefficients coef (None: the fitted ones).  No device needed."""
    nbytes, nb = ctypes.c_long(), ctypes.c_int()
    r = lib().mbx_qf_image(name.encode(), None, ctypes.byref(nbytes), ctypes.byref(nb), None, None, None)
    if r:
        raise RuntimeError("mbx_qf_image(%s): %d" % (name, r))
    img = np.zeros(nbytes.value, np.uint8)
    colf = np.zeros(nb.value, np.float32)
    b0 = ctypes.c_double()
    c = None if coef is None else np.ascontiguousarray(coef, np.float64)
    r = lib().mbx_qf_image(name.encode(), None if c is None else c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           ctypes.byref(nbytes), ctypes.byref(nb), img.ctypes.data,
                           colf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(b0))
    if r:
        raise RuntimeError("mbx_qf_image(%s): %d" % (name, r))
    return img.tobytes(), colf, b0.value


def fma_peaks(device=0):
    r = (ctypes.c_double * 3)()
    code = lib().mbx_fma_peaks(device, r)
    if code:
        raise MBXError(code, "fma peak benchmark failed")
    return {"fp64_tflops": r[0], "fp32_tflops": r[1], "fp32x2_tflops": r[2]}


def _ptr(a):
    """(pointer, is_device) for a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None, None
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError("arrays must be contiguous float64")
        return a.ctypes.data, False
    # torch tensor
    if a.dtype.__repr__() != "torch.float64" or not a.is_contiguous():
        raise TypeError("tensors must be contiguous float64")
    return a.data_ptr(), a.is_cuda


# live contexts by handle (weak: a Context is closed when collected)
_LIVE = weakref.WeakValueDictionary()


class Context:
    """One CUDA stream and the device state of the 2b/3b path (mbx_ctx)."""

    def __init__(self, device=0, stream=None):
        L = lib()
        h = ctypes.c_void_p()
        code = L.mbx_create(ctypes.byref(h), device, ctypes.c_void_p(stream) if stream else None)
        if code:
            raise MBXError(code, "mbx_create failed (no CUDA device?)")
        self.h = h
        self.device = device
        self.stream = stream or 0   # 0: a stream of the context's own
        _LIVE[h.value] = self

    @staticmethod
    def from_handle(handle):
        """The live Context whose mbx_ctx* is handle (torch.ops.mbxgpu ops take
        the context by its handle)."""
        c = _LIVE.get(int(handle))
        if c is None or not getattr(c, "h", None):
            raise MBXError(22, "no live context with handle %#x" % int(handle))
        return c

    def _order(self, dev_ptrs):
        """Device arrays from torch: when the library runs on another stream
        than torch's current one, torch's work on them (allocation, zeroing)
        must be complete before the library's kernels start."""
        if not dev_ptrs:
            return
        import torch
        cur = torch.cuda.current_stream(self.device)
        mine = self.stream if self.stream != 1 else 0   # 1: cudaStreamLegacy, torch's default stream
        if self.stream in (0, None) or mine != cur.cuda_stream:
            cur.synchronize()

    def close(self):
        if getattr(self, "h", None):
            _LIVE.pop(self.h.value, None)
            lib().mbx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        if code:
            raise MBXError(code, lib().mbx_last_error(self.h).decode())

    def set_topology(self, ids, first_index, tag, is_local, numsites):
        n = len(ids)
        arr = (ctypes.c_char_p * n)(*[s.encode() for s in ids])
        fi = np.ascontiguousarray(first_index, np.int32)
        tg = np.ascontiguousarray(tag, np.int32)
        lo = None if is_local is None else np.ascontiguousarray(is_local, np.int32)
        self._check(lib().mbx_set_topology(self.h, n, arr, fi.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           tg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           None if lo is None else lo.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           int(numsites)))

    def set_config(self, cutoff2b, cutoff3b, box=None, ignore_2b=(), ignore_3b=()):
        b = None if box is None else np.ascontiguousarray(box, np.float64).reshape(9)
        i2 = [s.encode() for t in ignore_2b for s in t]
        i3 = [s.encode() for t in ignore_3b for s in t]
        a2 = (ctypes.c_char_p * max(len(i2), 1))(*i2)
        a3 = (ctypes.c_char_p * max(len(i3), 1))(*i3)
        self._box = b
        self._check(lib().mbx_set_config(self.h, cutoff2b, cutoff3b, None if b is None else b.ctypes.data,
                                         len(ignore_2b), a2, len(ignore_3b), a3))

    def set_real_order(self, site_of_atom):
        a = np.ascontiguousarray(site_of_atom, np.int32)
        self._check(lib().mbx_set_real_order(self.h, len(a), a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def energy_real(self, nbody, xyz_real, grad_real=None, virial=None, use_ghost=False, mixed=False, grads=True):
        """A term on real coordinates in input order (numpy or CUDA tensor,
        not modified); the gradient is accumulated in input order."""
        px, dx = _ptr(xyz_real)
        self._order(dx)
        pg, dg = _ptr(grad_real)
        pv, _ = _ptr(virial)
        if grad_real is not None and bool(dg) != bool(dx):
            raise TypeError("xyz_real and grad_real must both be host or both be device arrays")
        flags = (MBX_DEVICE_PTRS if dx else 0) | (MBX_MIXED if mixed else 0) | \
                (0 if (grads and grad_real is not None) else MBX_NO_GRADS)
        e = ctypes.c_double()
        self._check(lib().mbx_energy_real(self.h, nbody, px, int(use_ghost), ctypes.byref(e), pg, pv, flags))
        return e.value

    def set_ignore_1b(self, ids=()):
        a = (ctypes.c_char_p * max(len(ids), 1))(*[i.encode() for i in ids])
        self._check(lib().mbx_set_ignore_1b(self.h, len(ids), a))

    def energy(self, nbody, xyz, grad=None, virial=None, use_ghost=False, mixed=False, grads=True):
        """Get1B/Get2B/Get3B on site coordinates xyz (numpy or CUDA tensor, wrapped in place)."""
        px, dx = _ptr(xyz)
        self._order(dx)
        pg, dg = _ptr(grad)
        pv, _ = _ptr(virial)
        flags = (MBX_DEVICE_PTRS if dx else 0) | (MBX_MIXED if mixed else 0) | (0 if grads else MBX_NO_GRADS)
        if grad is not None and bool(dg) != bool(dx):
            raise TypeError("xyz and grad must both be host or both be device arrays")
        if virial is not None and not isinstance(virial, np.ndarray):
            raise TypeError("virial is a host numpy array")
        e = ctypes.c_double()
        self._check(lib().mbx_energy(self.h, nbody, px, int(use_ghost), ctypes.byref(e), pg, pv, flags))
        return e.value

    def energy_2b3b(self, xyz, grad=None, virial=None, use_ghost=False, mixed=False, grads=True):
        """Get2B and Get3B side by side on the GPU; returns (E2B, E3B)."""
        px, dx = _ptr(xyz)
        self._order(dx)
        pg, dg = _ptr(grad)
        pv, _ = _ptr(virial)
        flags = (MBX_DEVICE_PTRS if dx else 0) | (MBX_MIXED if mixed else 0) | (0 if grads else MBX_NO_GRADS)
        if grad is not None and bool(dg) != bool(dx):
            raise TypeError("xyz and grad must both be host or both be device arrays")
        if virial is not None and not isinstance(virial, np.ndarray):
            raise TypeError("virial is a host numpy array")
        e2, e3 = ctypes.c_double(), ctypes.c_double()
        self._check(lib().mbx_energy_2b3b(self.h, px, int(use_ghost), ctypes.byref(e2), ctypes.byref(e3), pg, pv,
                                          flags))
        return e2.value, e3.value

    def counts(self, nbody):
        a, b = ctypes.c_long(), ctypes.c_long()
        self._check(lib().mbx_last_counts(self.h, nbody, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def timing(self):
        a, b, k = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(lib().mbx_last_timing(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(k)))
        return a.value, b.value, k.value

    def nmers(self, nbody, cutoff, xyz, use_ghost=False):
        xyz = np.ascontiguousarray(xyz, np.float64)
        cnt = ctypes.c_long()
        self._check(lib().mbx_nmers(self.h, nbody, cutoff, xyz.ctypes.data, int(use_ghost), None, 0,
                                    ctypes.byref(cnt)))
        out = np.zeros(max(cnt.value, 1) * nbody, np.int64)
        self._check(lib().mbx_nmers(self.h, nbody, cutoff, xyz.ctypes.data, int(use_ghost),
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), cnt.value,
                                    ctypes.byref(cnt)))
        return out[:cnt.value * nbody].reshape(-1, nbody)

    def evaluate(self, name, xyz, grad=None, virial=None, e_per=None, mixed=False, grads=True):
        nb, nreal, nv, nc = evaluator_info(name)
        px, dx = _ptr(xyz)
        self._order(dx)
        n = (xyz.shape[0] if xyz.ndim > 1 else xyz.size // (3 * nreal))
        pg, _ = _ptr(grad)
        pv, _ = _ptr(virial)
        pe, _ = _ptr(e_per)
        flags = (MBX_DEVICE_PTRS if dx else 0) | (MBX_MIXED if mixed else 0) | \
                (0 if (grads and grad is not None) else MBX_NO_GRADS)
        e = ctypes.c_double()
        self._check(lib().mbx_evaluate(self.h, name.encode(), n, px, pg, pv, pe, ctypes.byref(e), flags))
        return e.value

    def evaluate_dcoef(self, name, xyz, w=None, out=None):
        nb, nreal, nv, nc = evaluator_info(name)
        px, dx = _ptr(xyz)
        self._order(dx)
        n = (xyz.shape[0] if xyz.ndim > 1 else xyz.size // (3 * nreal))
        if out is None:
            out = np.zeros(nc)
        po, _ = _ptr(out)
        pw, _ = _ptr(w)
        self._check(lib().mbx_evaluate_dcoef(self.h, name.encode(), n, px, pw, po,
                                             MBX_DEVICE_PTRS if dx else 0))
        return out

    def poly(self, name, x, g=None, e=None):
        """Generated polynomial, variable-major x[nvars][nd] (poly_*::eval(nd, a, x, t, g))."""
        nb, nreal, nv, nc = evaluator_info(name)
        px, dx = _ptr(x)
        self._order(dx)
        nd = x.shape[-1] if x.ndim > 1 else x.size // nv
        if e is None:
            e = np.zeros(nd) if not dx else None
        pg, _ = _ptr(g)
        pe, _ = _ptr(e)
        self._check(lib().mbx_poly(self.h, name.encode(), nd, px, pg, pe, MBX_DEVICE_PTRS if dx else 0))
        return e

    def set_coefficients(self, name, a=None):
        pa, da = _ptr(None if a is None else a)
        self._check(lib().mbx_set_coefficients(self.h, name.encode(), pa, MBX_DEVICE_PTRS if da else 0))

    # ------------------------------------------------------------ batches
    def set_batch(self, conf_mon, boxes=None, has_box=None):
        """Configuration k owns monomers conf_mon[k] .. conf_mon[k+1]-1 of the
        topology; boxes[k] (9) where has_box[k]."""
        cm = np.ascontiguousarray(conf_mon, np.int32)
        nconf = len(cm) - 1
        b = None if boxes is None else np.ascontiguousarray(boxes, np.float64).reshape(nconf, 9)
        hb = None if has_box is None else np.ascontiguousarray(has_box, np.int32)
        ipp = ctypes.POINTER(ctypes.c_int)
        self._check(lib().mbx_set_batch(self.h, nconf, cm.ctypes.data_as(ipp), None if b is None else b.ctypes.data,
                                        None if hb is None else hb.ctypes.data_as(ipp)))
        self._nconf = nconf
        self._keep = (cm, b, hb)

    def batch_energy(self, nbody, xyz, grad=None, mixed=False, graph=False, virials=False):
        """One term of every configuration (device xyz, device grad +=).
        Returns energies[nconf] (and virials[nconf, 9] when asked)."""
        px, dx = _ptr(xyz)
        self._order(dx)
        pg, dg = _ptr(grad)
        if not dx or (grad is not None and not dg):
            raise TypeError("batches take CUDA tensors")
        flags = MBX_DEVICE_PTRS | (MBX_MIXED if mixed else 0) | (MBX_GRAPH if graph else 0) | \
            (0 if grad is not None else MBX_NO_GRADS)
        e = np.zeros(self._nconf)
        v = np.zeros((self._nconf, 9)) if virials else None
        dpp = ctypes.POINTER(ctypes.c_double)
        self._check(lib().mbx_batch_energy(self.h, nbody, px, pg, e.ctypes.data_as(dpp),
                                           None if v is None else v.ctypes.data_as(dpp), flags))
        return (e, v) if virials else e

    def batch_energy_2b3b(self, xyz, grad=None, mixed=False, graph=False, virials=False):
        """Both terms of every configuration, side by side on the GPU.
        Returns (e2[nconf], e3[nconf]) (and virials[nconf, 9], summed)."""
        px, dx = _ptr(xyz)
        self._order(dx)
        pg, dg = _ptr(grad)
        if not dx or (grad is not None and not dg):
            raise TypeError("batches take CUDA tensors")
        flags = MBX_DEVICE_PTRS | (MBX_MIXED if mixed else 0) | (MBX_GRAPH if graph else 0) | \
            (0 if grad is not None else MBX_NO_GRADS)
        e2 = np.zeros(self._nconf)
        e3 = np.zeros(self._nconf)
        v = np.zeros((self._nconf, 9)) if virials else None
        dpp = ctypes.POINTER(ctypes.c_double)
        self._check(lib().mbx_batch_energy_2b3b(self.h, px, pg, e2.ctypes.data_as(dpp), e3.ctypes.data_as(dpp),
                                                None if v is None else v.ctypes.data_as(dpp), flags))
        return (e2, e3, v) if virials else (e2, e3)

    def tune(self, nbody, xyz, grad=None, mixed=False):
        """Autotunes the builder's launch shapes of a term on the current batch
        (or system); returns (knobs dict, best ms)."""
        px, dx = _ptr(xyz)
        self._order(dx)
        pg, _ = _ptr(grad)
        if not dx:
            raise TypeError("tuning takes CUDA tensors")
        flags = MBX_DEVICE_PTRS | (MBX_MIXED if mixed else 0) | (0 if grad is not None else MBX_NO_GRADS)
        out = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        self._check(lib().mbx_tune(self.h, nbody, px, pg, flags, out, ctypes.byref(ms)))
        return dict(zip(KNOBS, list(out))), ms.value

    def knobs(self, nbody):
        out = (ctypes.c_int * 4)()
        self._check(lib().mbx_get_knobs(self.h, nbody, out))
        return dict(zip(KNOBS, list(out)))

    def set_knobs(self, nbody, **kw):
        """Sets launch shapes of a term (keys of KNOBS; the others kept)."""
        k = self.knobs(nbody)
        k.update(kw)
        arr = (ctypes.c_int * 4)(*[int(k[n]) for n in KNOBS])
        self._check(lib().mbx_set_knobs(self.h, nbody, arr))
