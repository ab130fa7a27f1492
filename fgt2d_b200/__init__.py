"""B200 plane-wave fast Gauss transform (2D and 3D), Python front end.

Mirrors the reference's calling sequence
``fgt2d(nd, delta, eps, ns, sources, ifcharge, charge, ifdipole, rnormal,
dipstr, iper, ifpgh, pot, grad, hess, nt, targ, ifpghtarg, pottarg,
gradtarg, hesstarg)`` (2d/planewave/src/fgt2d.f:19-22; fgt3d identical with
d = 3) over the C ABI in ``include/fgt_b200.h``.  Arrays use the reference's
memory layout: ``sources`` is the Fortran ``sources(d, ns)``, i.e. a C-order
``(ns, d)`` array; ``charge(nd, ns)`` is ``(ns, nd)``; outputs likewise.

The compute path is the CUDA library ``fgt2d_b200/lib/libfgt_b200.so``; there
is no CPU fallback: importing works without it, but every call raises if the
library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = ["fgt2d", "fgt3d", "transform", "transform_pgh", "Context", "Plan", "HostTree", "lib",
           "FGTError", "PREC_FP64", "PREC_MIXED", "PREC_AUTO", "nhess"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfgt_b200.so")

PREC_FP64, PREC_MIXED, PREC_AUTO = 0, 1, 2
_PREC = {"fp64": PREC_FP64, "mixed": PREC_MIXED, "auto": PREC_AUTO}
STATUS = {0: "ok", 1: "bad argument", 2: "unsupported option", 3: "out of memory",
          4: "CUDA error", 5: "no CUDA device", 6: "problem exceeds the fixed scratch"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_lib = None


class FGTError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = int(status)
        msg = f"{where}: status {status} ({STATUS.get(int(status), 'unknown')})"
        if status == 4 and _lib is not None:
            msg += f", cuda error {_lib.fgt_last_cuda_error()}"
        super().__init__(msg)


class PlanInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ["dim", "nd", "ns", "nt", "npwlevel", "nlevels", "nboxes", "npw", "nexp", "nlmax",
                 "nform", "neval", "ndirect_tasks", "nmp", "nloc"]] + \
               [("direct_pairs", ctypes.c_longlong), ("form_sources", ctypes.c_longlong),
                ("eval_points", ctypes.c_longlong), ("device_bytes", ctypes.c_longlong),
                ("host_tree_s", ctypes.c_double), ("host_lists_s", ctypes.c_double),
                ("host_plan_s", ctypes.c_double), ("large_delta", ctypes.c_int),
                ("all_direct", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("shift_bytes", ctypes.c_longlong * 3), ("form_flops", ctypes.c_double),
                ("eval_flops", ctypes.c_double), ("form_route_flops", ctypes.c_double),
                ("eval_route_flops", ctypes.c_double)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["shift_bytes"] = list(self.shift_bytes)
        return d


class Request(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nd", ctypes.c_int), ("delta", ctypes.c_double),
                ("eps", ctypes.c_double), ("ns", ctypes.c_int), ("sources", _dp), ("charge", _dp),
                ("nt", ctypes.c_int), ("targ", _dp), ("ifpgh", ctypes.c_int),
                ("ifpghtarg", ctypes.c_int), ("pot", _dp), ("pottarg", _dp), ("grad", _dp),
                ("hess", _dp), ("gradtarg", _dp), ("hesstarg", _dp), ("ifdipole", ctypes.c_int),
                ("rnormal", _dp), ("dipstr", _dp)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("points", ctypes.c_longlong),
                ("peak_bytes", ctypes.c_longlong), ("budget_bytes", ctypes.c_longlong),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double), ("mean_s", ctypes.c_double),
                ("max_s", ctypes.c_double), ("span_s", ctypes.c_double),
                ("hi_priority", ctypes.c_longlong)]


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FGTError(5, f"fgt2d_b200: {LIB_PATH} is missing (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    i, d = ctypes.c_int, ctypes.c_double
    L.fgt_ctx_create.argtypes = [i, ctypes.POINTER(_vp)]
    L.fgt_ctx_destroy.argtypes = [_vp]
    L.fgt_ctx_set_precision.argtypes = [_vp, i]
    L.fgt_ctx_set_host_threads.argtypes = [_vp, i]
    L.fgt_ctx_set_tree.argtypes = [_vp, i]
    L.fgt_ctx_set_sm_budget.argtypes = [_vp, i]
    L.fgt_ctx_set_grid_yield.argtypes = [_vp, i]
    L.fgt_ctx_set_scheme.argtypes = [_vp, i]
    L.fgt_plan_expansion.argtypes = [_vp, i, i, ctypes.POINTER(ctypes.c_double)]
    L.fgt_server_create.argtypes = [i, ctypes.c_longlong, i, ctypes.POINTER(_vp)]
    L.fgt_server_set_precision.argtypes = [_vp, i]
    L.fgt_server_set_sm_budget.argtypes = [_vp, i]
    L.fgt_server_set_grid_yield.argtypes = [_vp, i]
    L.fgt_server_submit.argtypes = [_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_longlong)]
    L.fgt_server_wait.argtypes = [_vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double)]
    L.fgt_server_stats_get.argtypes = [_vp, ctypes.POINTER(ServerStats)]
    L.fgt_server_destroy.argtypes = [_vp]
    L.fgt_device_tree_create.argtypes = [_vp, i, d, d, i, _dp, i, _dp, ctypes.POINTER(_vp)]
    L.fgt_default_ctx.restype = _vp
    L.fgt_ctx_stream.restype = _vp
    L.fgt_ctx_stream.argtypes = [_vp]
    L.fgt_probe_fp64_mma_tflops.argtypes = [_vp, ctypes.POINTER(ctypes.c_double)]
    L.fgt_tc_selftest.argtypes = [i, i, ctypes.POINTER(ctypes.c_double)]
    llp = ctypes.POINTER(ctypes.c_longlong)
    L.fgt_plan_create_shard.argtypes = [_vp, i, i, d, d, i, _dp, i, _dp, i, i, i, i, ctypes.POINTER(_vp)]
    L.fgt_plan_shard_counts.argtypes = [_vp, i, llp, llp, llp]
    L.fgt_plan_shard_owned.argtypes = [_vp, llp, llp]
    L.fgt_plan_execute_device_phase.argtypes = [_vp, i, _vp, _vp, _vp, _vp]
    L.fgt_plan_mp_pack.argtypes = [_vp, i, _vp, _vp]
    L.fgt_plan_mp_unpack.argtypes = [_vp, i, _vp, _vp]
    L.fgt_host_shard_create.argtypes = [i, i, d, d, i, _dp, i, _dp, i, i, i, i, ctypes.POINTER(_vp)]
    L.fgt_host_shard_counts.argtypes = [_vp, i, llp, llp]
    L.fgt_host_shard_slots.argtypes = [_vp, i, i, ctypes.POINTER(ctypes.c_int)]
    L.fgt_host_shard_stats.argtypes = [_vp, llp]
    L.fgt_host_shard_destroy.argtypes = [_vp]
    L.fgt_tc_error.argtypes = [i, i, ctypes.POINTER(ctypes.c_int)]
    L.fgt_large_delta_noalloc.argtypes = [i, i, d, i, _vp, _vp, i, _dp, i, _vp, i, _vp, i, _vp, _vp]
    L.fgt_transform.argtypes = [_vp, i, i, d, d, i, _dp, i, _dp, i, _dp, _dp, i, _dp, _dp, _dp, i,
                                _dp, i, _dp, _dp, _dp]
    L.fgt_plan_create.argtypes = [_vp, i, i, d, d, i, _dp, i, _dp, i, i, ctypes.POINTER(_vp)]
    L.fgt_plan_execute_host.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp]
    L.fgt_plan_execute_device.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.fgt_plan_execute_host_pgh.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.fgt_plan_create_cd.argtypes = [_vp, i, i, d, d, i, _dp, i, _dp, i, i, i, i, ctypes.POINTER(_vp)]
    L.fgt_plan_execute_host_full.argtypes = [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.fgt_plan_execute_device_full.argtypes = [_vp] + [_vp] * 10
    L.fgt_plan_execute_device_pgh.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.fgt_plan_profile_device.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float)]
    L.fgt_plan_get_info.argtypes = [_vp, ctypes.POINTER(PlanInfo)]
    L.fgt_plan_profile_dominant.argtypes = [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, i]
    L.fgt_plan_destroy.argtypes = [_vp]
    L.fgt_status_string.restype = ctypes.c_char_p
    L.fgt_status_string.argtypes = [i]
    L.fgt_build_info.restype = ctypes.c_char_p
    L.fgt_host_tree_create.argtypes = [i, d, d, i, _dp, i, _dp, i, ctypes.POINTER(_vp)]
    L.fgt_host_tree_dims.argtypes = [_vp, _ip]
    L.fgt_host_tree_field.restype = ctypes.c_longlong
    L.fgt_host_tree_field.argtypes = [_vp, i, _vp]
    L.fgt_host_tree_destroy.argtypes = [_vp]
    _lib = L
    return L


def _check(st, where):
    if st != 0:
        raise FGTError(st, where)


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape)


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class Context:
    """One CUDA device, its stream and the precision mode."""

    def __init__(self, device=0, precision="auto", host_threads=0, tree="device", scheme="planewave"):
        L = lib()
        h = _vp()
        _check(L.fgt_ctx_create(int(device), ctypes.byref(h)), "fgt_ctx_create")
        self._h = h
        self.set_precision(precision)
        self.set_tree(tree)
        self.set_scheme(scheme)
        if host_threads:
            L.fgt_ctx_set_host_threads(self._h, int(host_threads))

    def set_tree(self, where):
        """Where plans build their tree: "device" (point work on the GPU) or "host"."""
        _check(lib().fgt_ctx_set_tree(self._h, {"device": 0, "host": 1}[where]), "fgt_ctx_set_tree")

    def set_scheme(self, scheme):
        """The algorithm of plans created afterwards: "planewave" (2d/planewave,
        3d/planewave) or "nufft" (2d/nufft, 3d/nufft: plane-wave expansions at
        the cut level only, their NUFFTs as the exact sums)."""
        _check(lib().fgt_ctx_set_scheme(self._h, {"planewave": 0, "nufft": 1}[scheme]), "fgt_ctx_set_scheme")

    def set_sm_budget(self, sms):
        """SMs the persistent kernels of plans created afterwards size their grids for (0: all)."""
        _check(lib().fgt_ctx_set_sm_budget(self._h, int(sms)), "fgt_ctx_set_sm_budget")

    def set_grid_yield(self, on):
        """One CTA per task instead of persistent CTAs (plans created afterwards)."""
        _check(lib().fgt_ctx_set_grid_yield(self._h, int(bool(on))), "fgt_ctx_set_grid_yield")

    def set_precision(self, precision):
        p = _PREC[precision] if isinstance(precision, str) else int(precision)
        _check(lib().fgt_ctx_set_precision(self._h, p), "fgt_ctx_set_precision")

    @property
    def handle(self):
        return self._h

    def fp64_mma_tflops(self):
        """Measured FP64 tensor-core throughput of this device (TFLOP/s)."""
        v = ctypes.c_double()
        _check(lib().fgt_probe_fp64_mma_tflops(self._h, ctypes.byref(v)), "fgt_probe_fp64_mma_tflops")
        return v.value

    @property
    def stream(self):
        """The context's cudaStream_t as an integer."""
        return lib().fgt_ctx_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _default_ctx():
    h = lib().fgt_default_ctx()
    if not h:
        raise FGTError(5, "fgt_default_ctx")
    return h


def nhess(dim):
    """Hessian components per density: 3 in 2D (xx, xy, yy), 6 in 3D
    (xx, yy, zz, xy, xz, yz), the reference's orders."""
    return 3 if dim == 2 else 6


def _outputs(dim, nd, ns, nt, ifpgh, ifpghtarg, out=None):
    """Output arrays of the flags; ``out`` (optional dict) supplies caller
    arrays (e.g. pinned host memory) of the right shapes, C-contiguous f64."""
    H = nhess(dim)
    shapes = {"pot": ((ns, nd), ifpgh >= 1), "grad": ((ns, dim, nd), ifpgh >= 2),
              "hess": ((ns, H, nd), ifpgh >= 3), "pottarg": ((nt, nd), ifpghtarg >= 1),
              "gradtarg": ((nt, dim, nd), ifpghtarg >= 2), "hesstarg": ((nt, H, nd), ifpghtarg >= 3)}
    o = {}
    for k, (shape, want) in shapes.items():
        a = out.get(k) if out else None
        if not want:
            o[k] = None
        elif a is not None:
            if a.shape != shape or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out[{k!r}] must be a C-contiguous float64 array of shape {shape}")
            o[k] = a
        else:
            o[k] = np.zeros(shape)
    return o


def transform_pgh(dim, nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, ctx=None,
                  ifcharge=1, ifdipole=0, rnormal=None, dipstr=None, out=None):
    """Whole transform with gradients (ifpgh / ifpghtarg = 2) and Hessians (3).

    Returns a dict with ``pot`` (ns, nd), ``grad`` (ns, dim, nd), ``hess``
    (ns, H, nd) and the same for the targets (``pottarg``, ``gradtarg``,
    ``hesstarg``), None where not requested: the reference's
    ``grad(nd, dim, ns)`` / ``hess(nd, H, ns)`` in C order.  Dipoles
    (ifdipole = 1) take ``rnormal`` (ns, dim) and ``dipstr`` (ns, nd);
    ifcharge = 0 ignores ``charge``.  ``out`` (optional) maps output names to
    caller arrays that receive the results (pinned host memory avoids a
    staged copy).
    """
    L = lib()
    src = _f64(sources, (-1, dim))
    ns = src.shape[0]
    q = _f64(charge, (ns, nd)) if ns and ifcharge else None
    rn = _f64(rnormal, (ns, dim)) if ifdipole else None
    ds = _f64(dipstr, (ns, nd)) if ifdipole else None
    trg = _f64(targ, (-1, dim)) if targ is not None else np.zeros((0, dim))
    nt = trg.shape[0]
    o = _outputs(dim, nd, ns, nt, ifpgh, ifpghtarg, out)
    h = ctx.handle if ctx is not None else _default_ctx()
    st = L.fgt_transform(h, dim, nd, float(delta), float(eps), ns, _p(src), ifcharge, _p(q),
                         ifdipole, _p(rn), _p(ds), ifpgh, _p(o["pot"]), _p(o["grad"]), _p(o["hess"]),
                         nt, _p(trg), ifpghtarg, _p(o["pottarg"]), _p(o["gradtarg"]),
                         _p(o["hesstarg"]))
    _check(st, "fgt_transform")
    return o


def transform(dim, nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, ctx=None,
              ifcharge=1, ifdipole=0, rnormal=None, dipstr=None, out=None):
    """Whole transform; returns ``(pot, pottarg)`` shaped ``(ns, nd)``, ``(nt, nd)``.
    With ifpgh or ifpghtarg >= 2 it returns the reference's six outputs
    ``(pot, grad, hess, pottarg, gradtarg, hesstarg)`` (see transform_pgh)."""
    o = transform_pgh(dim, nd, delta, eps, sources, charge, targ, ifpgh, ifpghtarg, ctx, ifcharge,
                      ifdipole, rnormal, dipstr, out)
    if max(ifpgh, ifpghtarg) >= 2:
        return o["pot"], o["grad"], o["hess"], o["pottarg"], o["gradtarg"], o["hesstarg"]
    return o["pot"], o["pottarg"]


def fgt2d(nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, ctx=None):
    """2D transform with the reference's argument meaning (fgt2d.f:19-61)."""
    return transform(2, nd, delta, eps, sources, charge, targ, ifpgh, ifpghtarg, ctx)


def fgt3d(nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0, ctx=None):
    """3D transform with the reference's argument meaning (fgt3d.f:19-64)."""
    return transform(3, nd, delta, eps, sources, charge, targ, ifpgh, ifpghtarg, ctx)


class Plan:
    """Tree, lists and device task arrays for fixed points; apply many times."""

    def __init__(self, ctx, dim, nd, delta, eps, sources, targ=None, ifpgh=1, ifpghtarg=0,
                 ifcharge=1, ifdipole=0):
        L = lib()
        self.ctx = ctx
        self.dim, self.nd = dim, nd
        src = _f64(sources, (-1, dim))
        trg = _f64(targ, (-1, dim)) if targ is not None else np.zeros((0, dim))
        self.ns, self.nt = src.shape[0], trg.shape[0]
        self.ifpgh, self.ifpghtarg = ifpgh, ifpghtarg
        self.ifcharge, self.ifdipole = ifcharge, ifdipole
        h = _vp()
        _check(L.fgt_plan_create_cd(ctx.handle, dim, nd, float(delta), float(eps), self.ns, _p(src),
                                    self.nt, _p(trg), ifcharge, ifdipole, ifpgh, ifpghtarg,
                                    ctypes.byref(h)), "fgt_plan_create_cd")
        self._h = h

    def execute_host_full(self, charge=None, rnormal=None, dipstr=None):
        """All outputs for the plan's source kinds and flags (dict as transform_pgh)."""
        q = _f64(charge, (self.ns, self.nd)) if self.ifcharge else None
        rn = _f64(rnormal, (self.ns, self.dim)) if self.ifdipole else None
        ds = _f64(dipstr, (self.ns, self.nd)) if self.ifdipole else None
        o = _outputs(self.dim, self.nd, self.ns, self.nt, self.ifpgh, self.ifpghtarg)
        _check(lib().fgt_plan_execute_host_full(self._h, _p(q), _p(rn), _p(ds), _p(o["pot"]),
                                                _p(o["grad"]), _p(o["hess"]), _p(o["pottarg"]),
                                                _p(o["gradtarg"]), _p(o["hesstarg"])),
               "fgt_plan_execute_host_full")
        return o

    def expansion(self, which, box):
        """The box's multipole ("mp") or local ("loc") plane-wave expansion
        after the last execute, complex (nd, nexp) in the reference's layout;
        None when the plan holds no such expansion for the box."""
        inf = self.info()
        out = np.zeros(2 * self.nd * inf["nexp"])
        st = lib().fgt_plan_expansion(self._h, {"mp": 0, "loc": 1}[which], int(box),
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if st == 1:
            return None
        _check(st, "fgt_plan_expansion")
        return (out[0::2] + 1j * out[1::2]).reshape(self.nd, inf["nexp"])

    def info(self):
        inf = PlanInfo()
        _check(lib().fgt_plan_get_info(self._h, ctypes.byref(inf)), "fgt_plan_get_info")
        return inf.as_dict()

    def execute_host(self, sources, charge, targ=None):
        src = _f64(sources, (self.ns, self.dim))
        q = _f64(charge, (self.ns, self.nd))
        trg = _f64(targ, (self.nt, self.dim)) if targ is not None else None
        pot = np.zeros((self.ns, self.nd))
        pt = np.zeros((self.nt, self.nd))
        _check(lib().fgt_plan_execute_host(self._h, _p(src), _p(q), _p(trg), _p(pot), _p(pt)),
               "fgt_plan_execute_host")
        return pot, pt

    def execute_host_pgh(self, charge):
        """All outputs of the plan's flags (dict as transform_pgh)."""
        q = _f64(charge, (self.ns, self.nd))
        o = _outputs(self.dim, self.nd, self.ns, self.nt, self.ifpgh, self.ifpghtarg)
        _check(lib().fgt_plan_execute_host_pgh(self._h, _p(q), _p(o["pot"]), _p(o["grad"]),
                                               _p(o["hess"]), _p(o["pottarg"]), _p(o["gradtarg"]),
                                               _p(o["hesstarg"])), "fgt_plan_execute_host_pgh")
        return o

    def execute_device_pgh(self, d_chg, d_pot, d_grad, d_hess, d_pottarg, d_gradtarg, d_hesstarg,
                           stream=None):
        """Device pointers (ints; 0 skips a gradient or Hessian); asynchronous."""
        _check(lib().fgt_plan_execute_device_pgh(self._h, d_chg, d_pot or None, d_grad or None,
                                                 d_hess or None, d_pottarg or None,
                                                 d_gradtarg or None, d_hesstarg or None, stream),
               "fgt_plan_execute_device_pgh")

    def execute_device(self, d_src, d_chg, d_trg, d_pot, d_pottarg, stream=None):
        """Device pointers (ints, e.g. ``tensor.data_ptr()``); asynchronous."""
        _check(lib().fgt_plan_execute_device(self._h, d_src, d_chg, d_trg or None, d_pot or None,
                                             d_pottarg or None, stream),
               "fgt_plan_execute_device")

    def profile_device(self, d_src, d_chg, d_trg, d_pot, d_pottarg):
        ms = (ctypes.c_float * 8)()
        _check(lib().fgt_plan_profile_device(self._h, d_src, d_chg, d_trg or None, d_pot or None,
                                             d_pottarg or None, ms), "fgt_plan_profile_device")
        names = ["gather", "form", "merge", "m2l", "split", "eval", "direct", "scatter"]
        return dict(zip(names, list(ms)))

    def profile_dominant(self, d_chg, d_pot, d_pottarg):
        """(ms, executed flops, name, algorithmic flops) of the plan's dominant
        tensor-core launch in one execute on the context's stream; None when
        the plan has none."""
        ms, fl, al = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        name = ctypes.create_string_buffer(64)
        st = lib().fgt_plan_profile_dominant(self._h, d_chg, d_pot or None, d_pottarg or None,
                                             ctypes.byref(ms), ctypes.byref(fl), ctypes.byref(al),
                                             name, 64)
        if st == 2:
            return None
        _check(st, "fgt_plan_profile_dominant")
        return ms.value, fl.value, name.value.decode(), al.value

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_TREE_INT = ["laddr", "ilevel", "iparent", "nchild", "ichild", "nnbors", "nbors", "isrc",
             "isrcse", "itarg", "itargse"]


def HostTree(dim, delta, eps, sources, targ, nthreads=0):
    """The host tree of the transform in the reference's conventions (1-based)."""
    L = lib()
    src = _f64(sources, (-1, dim))
    trg = src if targ is sources else _f64(targ, (-1, dim))
    h = _vp()
    _check(L.fgt_host_tree_create(dim, float(delta), float(eps), src.shape[0], _p(src),
                                  trg.shape[0], _p(trg), int(nthreads), ctypes.byref(h)),
           "fgt_host_tree_create")
    return _tree_dict(h)


def DeviceTree(ctx, dim, delta, eps, sources, targ):
    """The same tree built with its point work on the context's GPU."""
    L = lib()
    src = _f64(sources, (-1, dim))
    trg = src if targ is sources else _f64(targ, (-1, dim))
    h = _vp()
    _check(L.fgt_device_tree_create(ctx.handle, dim, float(delta), float(eps), src.shape[0], _p(src),
                                    trg.shape[0], _p(trg), ctypes.byref(h)),
           "fgt_device_tree_create")
    return _tree_dict(h)


def _tree_dict(h):
    L = lib()
    try:
        dims = np.zeros(4, dtype=np.int32)
        st = L.fgt_host_tree_dims(h, dims.ctypes.data_as(_ip))
        out = {"nlevels": int(dims[0]), "nboxes": int(dims[1]), "npwlevel": int(dims[2]),
               "nlmax": int(dims[3])}
        if st != 0:
            return out
        for k, name in enumerate(_TREE_INT):
            n = L.fgt_host_tree_field(h, k, None)
            a = np.zeros(n, dtype=np.int32)
            L.fgt_host_tree_field(h, k, a.ctypes.data_as(_vp))
            out[name] = a
        for k, name in ((11, "centers"), (12, "boxsize")):
            n = L.fgt_host_tree_field(h, k, None)
            a = np.zeros(n)
            L.fgt_host_tree_field(h, k, a.ctypes.data_as(_vp))
            out[name] = a
        return out
    finally:
        L.fgt_host_tree_destroy(h)


class Server:
    """Transform server on one device (continuous batching of independent
    requests over worker streams, admission by device-memory footprint)."""

    def __init__(self, device=0, max_bytes=0, workers=4, precision="auto", sm_budget=0, grid_yield=False):
        L = lib()
        h = _vp()
        _check(L.fgt_server_create(int(device), int(max_bytes), int(workers), ctypes.byref(h)),
               "fgt_server_create")
        self._h = h
        p = _PREC[precision] if isinstance(precision, str) else int(precision)
        _check(L.fgt_server_set_precision(h, p), "fgt_server_set_precision")
        _check(L.fgt_server_set_sm_budget(h, int(sm_budget)), "fgt_server_set_sm_budget")
        _check(L.fgt_server_set_grid_yield(h, int(bool(grid_yield))), "fgt_server_set_grid_yield")
        self._live = {}

    def submit(self, dim, nd, delta, eps, sources, charge, targ=None, ifpgh=1, ifpghtarg=0,
               rnormal=None, dipstr=None):
        """Queues one transform; returns its id.  The arrays are kept alive here.
        ``charge`` None: no charges; ``dipstr`` given: dipoles with ``rnormal``."""
        src = _f64(sources, (-1, dim))
        ns = src.shape[0]
        q = None if charge is None else (_f64(charge, (ns, nd)) if ns else np.zeros((0, nd)))
        ifd = int(dipstr is not None)
        rn = _f64(rnormal, (ns, dim)) if ifd else None
        ds = _f64(dipstr, (ns, nd)) if ifd else None
        trg = (src if targ is sources else _f64(targ, (-1, dim))) if targ is not None else None
        nt = trg.shape[0] if trg is not None else 0
        o = _outputs(dim, nd, ns, nt, ifpgh, ifpghtarg)
        r = Request(dim, nd, float(delta), float(eps), ns, _p(src), _p(q), nt, _p(trg), ifpgh,
                    ifpghtarg, _p(o["pot"]), _p(o["pottarg"]), _p(o["grad"]), _p(o["hess"]),
                    _p(o["gradtarg"]), _p(o["hesstarg"]), ifd, _p(rn), _p(ds))
        rid = ctypes.c_longlong()
        _check(lib().fgt_server_submit(self._h, ctypes.byref(r), ctypes.byref(rid)), "fgt_server_submit")
        self._live[rid.value] = (src, q, trg, o, rn, ds)
        return rid.value

    def wait_pgh(self, rid):
        """Blocks until request rid is done; returns (outputs dict, latency_s)."""
        lat = ctypes.c_double()
        st = lib().fgt_server_wait(self._h, int(rid), ctypes.byref(lat))
        o = self._live.pop(rid)[3]
        _check(st, "fgt_server_wait")
        return o, lat.value

    def wait(self, rid):
        """Blocks until request rid is done; returns (pot, pottarg, latency_s)."""
        o, lat = self.wait_pgh(rid)
        return o["pot"], o["pottarg"], lat

    def stats(self):
        s = ServerStats()
        _check(lib().fgt_server_stats_get(self._h, ctypes.byref(s)), "fgt_server_stats_get")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().fgt_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
