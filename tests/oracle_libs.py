"""ctypes front-ends for the two CPU checkers used by the tests.

- ``Oracle``: oracle/liboracle.so, the plain-C restatement of the reference step (built by
  oracle/Makefile; it travels with the repository).
- ``Reference``: oracle/_ref/libmpcdref.so, the unmodified reference sources compiled with a
  thin C wrapper (oracle/ref_capi.cpp). Built only where the reference sources exist.

Both expose the same methods on numpy arrays so a test can run either as the checker.
"""
import ctypes as C
import os

import numpy as np

from src_incompressible_openmp_b200 import _abi
from src_incompressible_openmp_b200.cases import to_c

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libmpcdref.so")

_d = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_P = C.POINTER(_abi.ParamsC)


def _fields_struct(Nc, with_fields=True):
    N = np.zeros(Nc, np.int32)
    arrs = {k: np.zeros(Nc) for k in _abi.FIELD_NAMES}
    s = _abi.CellFieldsC()
    s.N = N.ctypes.data_as(C.POINTER(C.c_int32))
    for k, a in arrs.items():
        setattr(s, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    arrs["N"] = N
    return s, arrs


def closure_detail(n, Nc):
    """Allocates every output array of mpcd_closure_detail_c; returns (struct, dict of arrays)."""
    d = _abi.ClosureDetailC()
    out = {}
    for k in ("repairedX", "repairedV"):
        out[k] = np.zeros(2 * n)
        setattr(d, k, out[k].ctypes.data_as(C.POINTER(C.c_double)))
    for k in ("refFields", "redFields", "repairedFields", "outFields"):
        s, arrs = _fields_struct(Nc)
        setattr(d, k, s)
        out[k] = arrs
    for k in ("pdriveRaw", "pdrive", "duRepairX", "duRepairY", "duEOSX", "duEOSY"):
        out[k] = np.zeros(Nc)
        setattr(d, k, out[k].ctypes.data_as(C.POINTER(C.c_double)))
    out["interzoneMask"] = np.zeros(Nc, np.int32)
    d.interzoneMask = out["interzoneMask"].ctypes.data_as(C.POINTER(C.c_int32))
    return d, out


_DPA = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

class _Checker:
    prefix = ""
    threads_arg = False

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L, pre = self.lib, self.prefix
        f = getattr(L, pre + "apply_bc")
        f.argtypes = [_P, _d, _d, C.c_uint64, C.POINTER(_abi.WallInfoC)]
        f.restype = C.c_int
        f = getattr(L, pre + "stream")
        f.argtypes = [_P, _d, _d]
        f = getattr(L, pre + "srd_shift_cells")
        f.argtypes = [_P, _d, C.c_uint64, _i]
        f = getattr(L, pre + "srd_collide")
        f.argtypes = [_P, _d, _i, C.c_uint64]
        f.restype = C.c_int
        f = getattr(L, pre + "cell_fields")
        f.argtypes = [_P, _d, _d, C.c_double, C.POINTER(_abi.CellFieldsC)]
        f = getattr(L, pre + "zone_owner_map")
        f.argtypes = [_P, C.c_int32, _i]
        extra = [C.c_int32] if self.threads_arg else []
        f = getattr(L, pre + "zone_pass")
        f.argtypes = [_P, _d, _d, _d, _d, C.c_int32, C.c_uint64] + extra + [C.POINTER(_abi.PassMetricsC)]
        f.restype = C.c_int
        f = getattr(L, pre + "liquid_closure")
        f.argtypes = [_P, _d, _d, _d, _d, _d, _d, C.POINTER(_abi.ClosureMetricsC), C.POINTER(_abi.ClosureDetailC)]
        f.restype = C.c_int
        f = getattr(L, pre + "step")
        f.argtypes = [_P, _d, _d, C.c_int64] + extra + [C.POINTER(_abi.StepMetricsC)]
        f.restype = C.c_int
        getattr(L, pre + "last_error").restype = C.c_char_p

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(getattr(self.lib, self.prefix + "last_error")().decode())

    def _t(self):
        return [self.nthreads] if self.threads_arg else []

    def stream(self, p, x, v):
        x, v = x.copy(), v.copy()
        getattr(self.lib, self.prefix + "stream")(C.byref(to_c(p)), x, v)
        return x, v

    def apply_bc(self, p, x, v, seed):
        x, v = x.copy(), v.copy()
        w = _abi.WallInfoC()
        self._chk(getattr(self.lib, self.prefix + "apply_bc")(C.byref(to_c(p)), x, v, seed, C.byref(w)))
        return x, v, _abi.struct_to_dict(w)

    def srd_shift_cells(self, p, x, seed):
        cid = np.zeros(p["n"], np.int32)
        getattr(self.lib, self.prefix + "srd_shift_cells")(C.byref(to_c(p)), np.ascontiguousarray(x), seed, cid)
        return cid

    def srd_collide(self, p, v, cid, seed):
        v = v.copy()
        self._chk(getattr(self.lib, self.prefix + "srd_collide")(C.byref(to_c(p)), v, np.ascontiguousarray(cid, np.int32), seed))
        return v

    def cell_fields(self, p, x, v, rho_target):
        s, arrs = _fields_struct(p["Nc"])
        getattr(self.lib, self.prefix + "cell_fields")(C.byref(to_c(p)), np.ascontiguousarray(x), np.ascontiguousarray(v), rho_target, C.byref(s))
        return arrs

    def zone_owner_map(self, p, mode):
        o = np.zeros(p["Nc"], np.int32)
        getattr(self.lib, self.prefix + "zone_owner_map")(C.byref(to_c(p)), _abi.LAYOUT_MODES[mode], o)
        return o

    def zone_pass(self, p, x, v, mode, seed_base):
        xo, vo = np.zeros_like(x), np.zeros_like(v)
        m = _abi.PassMetricsC()
        self._chk(getattr(self.lib, self.prefix + "zone_pass")(
            C.byref(to_c(p)), np.ascontiguousarray(x), np.ascontiguousarray(v), xo, vo,
            _abi.LAYOUT_MODES[mode], seed_base, *self._t(), C.byref(m)))
        return xo, vo, _abi.struct_to_dict(m)

    def zone_pass_serial(self, p, x, v, mode, seed_base):
        f = getattr(self.lib, self.prefix + "zone_pass_serial")
        f.argtypes = [C.POINTER(_abi.ParamsC), _DPA, _DPA, _DPA, _DPA, C.c_int32, C.c_uint64, C.POINTER(_abi.PassMetricsC)]
        f.restype = C.c_int
        xo, vo = np.zeros_like(x), np.zeros_like(v)
        m = _abi.PassMetricsC()
        self._chk(f(C.byref(to_c(p)), np.ascontiguousarray(x), np.ascontiguousarray(v), xo, vo, _abi.LAYOUT_MODES[mode],
                    seed_base, C.byref(m)))
        return xo, vo, _abi.struct_to_dict(m)

    def liquid_closure(self, p, refx, refv, redx, redv, detail=True):
        xo, vo = np.zeros_like(redx), np.zeros_like(redv)
        m = _abi.ClosureMetricsC()
        d, darr = closure_detail(p["n"], p["Nc"]) if detail else (None, None)
        self._chk(getattr(self.lib, self.prefix + "liquid_closure")(
            C.byref(to_c(p)), refx, refv, redx, redv, xo, vo, C.byref(m), C.byref(d) if d is not None else None))
        return xo, vo, _abi.struct_to_dict(m), darr

    def step(self, p, x, v, step):
        x, v = x.copy(), v.copy()
        m = _abi.StepMetricsC()
        self._chk(getattr(self.lib, self.prefix + "step")(C.byref(to_c(p)), x, v, step, *self._t(), C.byref(m)))
        return x, v, _abi.struct_to_dict(m)


class Oracle(_Checker):
    prefix = "oracle_"

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)


class Reference(_Checker):
    prefix = "ref_"
    threads_arg = True
    nthreads = 4

    def __init__(self, path=REF_SO):
        super().__init__(path)


def reference_available():
    return os.path.exists(REF_SO)
