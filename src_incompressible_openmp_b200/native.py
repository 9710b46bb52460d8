"""Python binding of the C-ABI (include/mpcd_c.h) in libmpcd_b200.so.

There is no CPU fallback: if the CUDA library is not built, or no sm_100 device is present,
every entry point raises. ``Context`` mirrors the reference's phase functions on a
device-resident state:

    reference (namespace mpcd)                       Context method
    main_...shifted_profiled.cpp:242-247 (stream)    stream()
    apply_bc_general                                 apply_bc(seed)
    srd_cell_id_with_random_shift                    srd_shift_cells(seed)
    srd_collision_step                               srd_collide(seed) / srd_collide_cells(cid, seed)
    compute_cell_fields                              cell_fields(rho_target)
    run_zone_pass_openmp                             zone_pass(mode, seed_base)
    run_liquid_closure(stateRef, stateRed)           save_ref() before the passes, then liquid_closure()
    the benchmark loop body                          step(step0, nsteps)
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from .cases import to_c

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpcd_b200.so")

_lib = None
_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_fp = C.POINTER(C.c_float)


class MpcdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads libmpcd_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    sig = {
        "mpcd_last_error": ([], C.c_char_p),
        "mpcd_io_last_error": ([], C.c_char_p),
        "mpcd_device_available": ([], C.c_int),
        "mpcd_read_params_kv": ([C.c_char_p, P(_abi.ParamsC)], C.c_int),
        "mpcd_read_kv_string": ([C.c_char_p, C.c_char_p, C.c_char_p, C.c_int], C.c_int),
        "mpcd_ctx_create": ([P(_abi.ParamsC), C.c_int, P(C.c_void_p)], C.c_int),
        "mpcd_ctx_create_form": ([P(_abi.ParamsC), C.c_int, C.c_int32, P(C.c_void_p)], C.c_int),
        "mpcd_ctx_destroy": ([C.c_void_p], C.c_int),
        "mpcd_ctx_stream": ([C.c_void_p], C.c_void_p),
        "mpcd_set_state": ([C.c_void_p, _dp, _dp, C.c_int64], C.c_int),
        "mpcd_get_state": ([C.c_void_p, _dp, _dp], C.c_int),
        "mpcd_set_state_device": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
        "mpcd_get_state_device": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
        "mpcd_stream": ([C.c_void_p], C.c_int),
        "mpcd_apply_bc": ([C.c_void_p, C.c_uint64, P(_abi.WallInfoC)], C.c_int),
        "mpcd_srd_shift_cells": ([C.c_void_p, C.c_uint64, C.c_void_p], C.c_int),
        "mpcd_srd_collide": ([C.c_void_p, C.c_uint64], C.c_int),
        "mpcd_srd_collide_cells": ([C.c_void_p, _ip, C.c_uint64], C.c_int),
        "mpcd_cell_fields": ([C.c_void_p, C.c_double, P(_abi.CellFieldsC)], C.c_int),
        "mpcd_save_ref": ([C.c_void_p], C.c_int),
        "mpcd_zone_pass": ([C.c_void_p, C.c_int32, C.c_uint64, P(_abi.PassMetricsC)], C.c_int),
        "mpcd_zone_pass_serial": ([C.c_void_p, C.c_int32, C.c_uint64, P(_abi.PassMetricsC)], C.c_int),
        "mpcd_liquid_closure": ([C.c_void_p, P(_abi.ClosureMetricsC), P(_abi.ClosureDetailC)], C.c_int),
        "mpcd_zone_owner_map": ([C.c_void_p, C.c_int32, _ip], C.c_int),
        "mpcd_step": ([C.c_void_p, C.c_int64, C.c_int64, P(_abi.StepMetricsC)], C.c_int),
        "mpcd_step_metrics": ([C.c_void_p, P(_abi.StepMetricsC)], C.c_int),
        "mpcd_run_jobs": ([C.c_void_p, C.c_int64, P(C.c_void_p), P(C.c_void_p), C.c_int64, C.c_int64,
                           P(C.c_void_p), P(C.c_void_p)], C.c_int),
        "mpcd_step_timed": ([C.c_void_p, C.c_int64, C.c_int64, P(C.c_double)], C.c_int),
        "mpcd_step_profile": ([C.c_void_p, C.c_int64, C.c_int64, P(C.c_double), C.c_int], C.c_int),
        "mpcd_launch_count": ([C.c_void_p], C.c_int64),
        "mpcd_ctx_set_graphs": ([C.c_void_p, C.c_int], C.c_int),
        "mpcd_ctx_collide_shape": ([C.c_void_p, C.c_int32, P(C.c_int32)], C.c_int),
        "mpcd_batch_create": ([P(_abi.ParamsC), C.c_int, C.c_int, P(C.c_void_p)], C.c_int),
        "mpcd_batch_create_form": ([P(_abi.ParamsC), C.c_int, C.c_int, C.c_int32, P(C.c_void_p)], C.c_int),
        "mpcd_batch_destroy": ([C.c_void_p], C.c_int),
        "mpcd_batch_size": ([C.c_void_p], C.c_int),
        "mpcd_batch_member": ([C.c_void_p, C.c_int], C.c_void_p),
        "mpcd_batch_step": ([C.c_void_p, C.c_int64, C.c_int64, P(C.c_double)], C.c_int),
        "mpcd_cell_fields_static": ([P(_abi.ParamsC), C.c_void_p, C.c_void_p, C.c_int64, C.c_double,
                                     P(_abi.CellFieldsC), C.c_void_p], C.c_int),
        "mpcd_learned_param_count": ([], C.c_int),
        "mpcd_learned_init": ([C.c_uint64, _fp], C.c_int),
        "mpcd_learned_samples": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int32, _fp, _fp, C.c_int64, P(C.c_int64)],
                                 C.c_int),
        "mpcd_learned_train": ([_fp, _fp, C.c_int64, _fp, C.c_int32, C.c_int32, C.c_float, C.c_uint64, C.c_int, _fp],
                               C.c_int),
        "mpcd_learned_grad": ([_fp, _fp, C.c_int64, _fp, C.c_int, _fp, _fp], C.c_int),
        "mpcd_learned_predict": ([_fp, C.c_int64, _fp, C.c_int, _fp], C.c_int),
        "mpcd_learned_set": ([C.c_void_p, _fp, C.c_double], C.c_int),
        "mpcd_learned_stats": ([C.c_void_p, P(C.c_int64), P(C.c_int64), P(C.c_int32)], C.c_int),
        "mpcd_learned_options": ([C.c_void_p, C.c_int32], C.c_int),
        "mpcd_profile_reset": ([C.c_void_p, C.c_int32], C.c_int),
        "mpcd_profile_read": ([C.c_void_p, _dp, P(C.c_int64)], C.c_int),
        "mpcd_zone_layout": ([P(_abi.ParamsC), C.c_int32, P(C.c_int32), C.c_void_p, C.c_int32], C.c_int),
        "mpcd_host_alloc": ([C.c_size_t], C.c_void_p),
        "mpcd_host_free": ([C.c_void_p], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


class PinnedArray:
    """A float64 numpy view of page-locked host memory (freed with close())."""

    def __init__(self, count):
        self.ptr = lib().mpcd_host_alloc(8 * count)
        if not self.ptr:
            raise MpcdError(2, lib().mpcd_last_error().decode())
        self.array = np.ctypeslib.as_array((C.c_double * count).from_address(self.ptr))

    def close(self):
        if self.ptr:
            lib().mpcd_host_free(self.ptr)
            self.ptr = None


def device_available():
    return bool(lib().mpcd_device_available())


def _check(rc):
    if rc != 0:
        raise MpcdError(rc, lib().mpcd_last_error().decode())


def read_params_kv(path):
    p = _abi.ParamsC()
    rc = lib().mpcd_read_params_kv(path.encode(), C.byref(p))
    if rc != 0:
        raise MpcdError(rc, lib().mpcd_io_last_error().decode())
    return p


def _fields_struct(Nc):
    arrs = {k: np.zeros(Nc) for k in _abi.FIELD_NAMES}
    arrs["N"] = np.zeros(Nc, np.int32)
    s = _abi.CellFieldsC()
    s.N = arrs["N"].ctypes.data_as(C.POINTER(C.c_int32))
    for k in _abi.FIELD_NAMES:
        setattr(s, k, arrs[k].ctypes.data_as(C.POINTER(C.c_double)))
    return s, arrs


def cell_fields_static(params, x_ptr, v_ptr, n, rho_target, out_ptrs, stream=0):
    """mpcd_cell_fields_static: cell fields of a caller-owned device state (device pointers
    x_ptr, v_ptr of 2n doubles) into caller-owned device arrays out_ptrs {field: pointer}
    (fields of mpcd_cellfields_c; missing ones are skipped), enqueued on `stream`."""
    s = _abi.CellFieldsC()
    for k, ptr in out_ptrs.items():
        t = C.c_int32 if k == "N" else C.c_double
        setattr(s, k, C.cast(C.c_void_p(ptr), C.POINTER(t)))
    pc = to_c(params)
    _check(lib().mpcd_cell_fields_static(C.byref(pc), C.c_void_p(x_ptr), C.c_void_p(v_ptr), n, rho_target,
                                         C.byref(s), C.c_void_p(stream)))


FORMS = {"f64": 0, "f32": 1, "fast": 2}  # mpcd_state_form
COLLIDE_SHAPES = 7  # MPCD_COLLIDE_SHAPES


class Context:
    """A device-resident MPCD state for one parameter set (one GPU). form "f64" is the plain
    form; "f32" the FP32 precision form; "fast" the fast form (FP32 bins, draws from hashes,
    order-free); the last two run whole steps and state I/O only."""

    def __init__(self, params, device=0, form="f64"):
        self.params = dict(params)
        self.n = int(params["n"])
        self.Nc = int(params["Nc"])
        self.form = form
        self._pc = to_c(params)
        h = C.c_void_p()
        _check(lib().mpcd_ctx_create_form(C.byref(self._pc), device, FORMS[form], C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().mpcd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state -------------------------------------------------------------------------
    def set_state(self, x, v):
        x = np.ascontiguousarray(x, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        _check(lib().mpcd_set_state(self.h, x, v, self.n))

    def get_state(self, x=None, v=None):
        """Particle-id-ordered copies of x and v (into the given float64 arrays if any)."""
        x = np.empty(2 * self.n) if x is None else x
        v = np.empty(2 * self.n) if v is None else v
        _check(lib().mpcd_get_state(self.h, x, v))
        return x, v

    def run_jobs(self, xs, vs, step0, nsteps, xo=None, vo=None):
        """Independent jobs with host buffers (mpcd_run_jobs): job j loads (xs[j], vs[j]), runs
        steps step0 + j*nsteps + 1 .. step0 + (j+1)*nsteps and stores its result in (xo[j], vo[j])
        (new arrays when not given); the copies of neighbouring jobs overlap each job's steps.
        Returns (xo, vo)."""
        k = len(xs)
        if len(vs) != k:
            raise ValueError("xs and vs differ in length")
        for a in list(xs) + list(vs):
            if a.dtype != np.float64 or a.size != 2 * self.n or not a.flags.c_contiguous:
                raise ValueError("job buffers must be contiguous float64 arrays of 2n values")
        xo = [np.empty(2 * self.n) for _ in range(k)] if xo is None else xo
        vo = [np.empty(2 * self.n) for _ in range(k)] if vo is None else vo
        for a in list(xo) + list(vo):
            if a.dtype != np.float64 or a.size != 2 * self.n or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError("job outputs must be writeable contiguous float64 arrays of 2n values")
        ptrs = lambda arrs: (C.c_void_p * max(k, 1))(*[a.ctypes.data for a in arrs])
        _check(lib().mpcd_run_jobs(self.h, k, ptrs(xs), ptrs(vs), step0, nsteps, ptrs(xo), ptrs(vo)))
        return xo, vo

    def set_state_device(self, x_ptr, v_ptr):
        _check(lib().mpcd_set_state_device(self.h, C.c_void_p(x_ptr), C.c_void_p(v_ptr), self.n))

    def get_state_device(self, x_ptr, v_ptr):
        _check(lib().mpcd_get_state_device(self.h, C.c_void_p(x_ptr), C.c_void_p(v_ptr)))

    @property
    def stream_handle(self):
        return lib().mpcd_ctx_stream(self.h)

    # phases ------------------------------------------------------------------------
    def stream(self):
        _check(lib().mpcd_stream(self.h))

    def apply_bc(self, seed):
        w = _abi.WallInfoC()
        _check(lib().mpcd_apply_bc(self.h, seed, C.byref(w)))
        return _abi.struct_to_dict(w)

    def srd_shift_cells(self, seed, want_cells=True):
        cid = np.empty(self.n, np.int32) if want_cells else None
        _check(lib().mpcd_srd_shift_cells(self.h, seed, cid.ctypes.data if want_cells else None))
        return cid

    def srd_collide(self, seed):
        _check(lib().mpcd_srd_collide(self.h, seed))

    def srd_collide_cells(self, cid, seed):
        _check(lib().mpcd_srd_collide_cells(self.h, np.ascontiguousarray(cid, np.int32), seed))

    def cell_fields(self, rho_target):
        s, arrs = _fields_struct(self.Nc)
        _check(lib().mpcd_cell_fields(self.h, rho_target, C.byref(s)))
        return arrs

    def save_ref(self):
        _check(lib().mpcd_save_ref(self.h))

    def zone_pass(self, mode, seed_base):
        m = _abi.PassMetricsC()
        _check(lib().mpcd_zone_pass(self.h, _abi.LAYOUT_MODES[mode] if isinstance(mode, str) else mode, seed_base, C.byref(m)))
        return _abi.struct_to_dict(m)

    def zone_pass_serial(self, mode, seed_base):
        """mpcd_zone_pass_serial: zones one after another on the live state (in place)."""
        m = _abi.PassMetricsC()
        _check(lib().mpcd_zone_pass_serial(self.h, _abi.LAYOUT_MODES[mode] if isinstance(mode, str) else mode, seed_base,
                                           C.byref(m)))
        return _abi.struct_to_dict(m)

    def liquid_closure(self, detail=False):
        m = _abi.ClosureMetricsC()
        d = None
        out = None
        if detail:
            d = _abi.ClosureDetailC()
            out = {}
            for k in ("repairedX", "repairedV"):
                out[k] = np.zeros(2 * self.n)
                setattr(d, k, out[k].ctypes.data_as(C.POINTER(C.c_double)))
            for k in ("refFields", "redFields", "repairedFields", "outFields"):
                s, arrs = _fields_struct(self.Nc)
                setattr(d, k, s)
                out[k] = arrs
            for k in ("pdriveRaw", "pdrive", "duRepairX", "duRepairY", "duEOSX", "duEOSY"):
                out[k] = np.zeros(self.Nc)
                setattr(d, k, out[k].ctypes.data_as(C.POINTER(C.c_double)))
            out["interzoneMask"] = np.zeros(self.Nc, np.int32)
            d.interzoneMask = out["interzoneMask"].ctypes.data_as(C.POINTER(C.c_int32))
        _check(lib().mpcd_liquid_closure(self.h, C.byref(m), C.byref(d) if d is not None else None))
        return (_abi.struct_to_dict(m), out) if detail else _abi.struct_to_dict(m)

    def zone_owner_map(self, mode):
        o = np.zeros(self.Nc, np.int32)
        _check(lib().mpcd_zone_owner_map(self.h, _abi.LAYOUT_MODES[mode], o))
        return o

    PHASES = ("stream_bc", "walls", "srd_index", "srd_signs", "collide", "cell_index", "ref_fields",
              "zone_seeds", "zone_pass", "closure_cells", "kick_resort")

    def step_timed(self, step0, nsteps):
        """Runs the steps; returns device seconds (CUDA events on the context's stream)."""
        t = C.c_double()
        _check(lib().mpcd_step_timed(self.h, step0, nsteps, C.byref(t)))
        return t.value

    def step_profile(self, step0, nsteps):
        """Runs the steps with phase-boundary events; returns {phase: device seconds}."""
        arr = (C.c_double * len(self.PHASES))()
        _check(lib().mpcd_step_profile(self.h, step0, nsteps, arr, len(self.PHASES)))
        return dict(zip(self.PHASES, list(arr)))

    def launch_count(self):
        return int(lib().mpcd_launch_count(self.h))

    def collide_shape(self, shape=-1):
        """mpcd_ctx_collide_shape: set the collision tile shape (0 .. COLLIDE_SHAPES-1) or, with -1, only query;
        returns the shape in use (-1 before the autotuner has run)."""
        r = C.c_int32()
        _check(lib().mpcd_ctx_collide_shape(self.h, shape, C.byref(r)))
        return r.value

    def set_graphs(self, enable):
        """Step replay from CUDA graphs (on by default)."""
        _check(lib().mpcd_ctx_set_graphs(self.h, 1 if enable else 0))

    def profile_reset(self, enable=True):
        """Clears the velocity-profile accumulators; with enable, every following step adds to them."""
        _check(lib().mpcd_profile_reset(self.h, 1 if enable else 0))

    def profile_read(self):
        """(time-averaged mean vx per row iy, steps accumulated)."""
        ux = np.zeros(int(self.params["Ny"]))
        k = C.c_int64()
        _check(lib().mpcd_profile_read(self.h, ux, C.byref(k)))
        return ux, k.value

    def step(self, step0, nsteps, metrics=False):
        m = _abi.StepMetricsC() if metrics else None
        _check(lib().mpcd_step(self.h, step0, nsteps, C.byref(m) if m is not None else None))
        return _abi.struct_to_dict(m) if metrics else None

    def learned_samples(self, step0, nsteps, stride, capacity=None):
        """mpcd_learned_samples: runs plain steps and returns (features [rows, 75], targets
        [rows, 2]) of every stride-th cell after each step's closure."""
        if capacity is None:
            capacity = nsteps * ((self.params["Nc"] + stride - 1) // stride)
        X = np.empty((max(capacity, 1), LEARNED_FEATURES), np.float32)
        Y = np.empty((max(capacity, 1), LEARNED_OUTPUTS), np.float32)
        n = C.c_int64()
        _check(lib().mpcd_learned_samples(self.h, step0, nsteps, stride, _f32p(X), _f32p(Y), capacity, C.byref(n)))
        return X[:n.value].copy(), Y[:n.value].copy()

    def learned_set(self, params, occ_limit=0.0):
        """mpcd_learned_set: the network in the step's closure (None: the plain closure), with
        the plain closure as the fallback of steps after one whose occStd exceeded occ_limit."""
        if params is None:
            _check(lib().mpcd_learned_set(self.h, None, 0.0))
            return
        p = _params32(params)
        _check(lib().mpcd_learned_set(self.h, _f32p(p), float(occ_limit)))

    def learned_options(self, bulk_only=True):
        """mpcd_learned_options: bulk_only -> no learned kick where the stencil crosses a wall."""
        _check(lib().mpcd_learned_options(self.h, 1 if bulk_only else 0))

    def learned_stats(self):
        """(plain steps, learned steps, next step's mode) since learned_set."""
        a, b, m = C.c_int64(), C.c_int64(), C.c_int32()
        _check(lib().mpcd_learned_stats(self.h, C.byref(a), C.byref(b), C.byref(m)))
        return a.value, b.value, m.value


LEARNED_FEATURES, LEARNED_OUTPUTS, LEARNED_PARAMS = 75, 2, 9155


def _f32p(a):
    return a.ctypes.data_as(_fp)


def _params32(params):
    p = np.ascontiguousarray(params, np.float32)
    if p.shape != (LEARNED_PARAMS,):
        raise ValueError(f"network parameters: {LEARNED_PARAMS} floats expected, got {p.shape}")
    return p


def _rows32(X, cols):
    X = np.ascontiguousarray(X, np.float32)
    if X.ndim != 2 or X.shape[1] != cols:
        raise ValueError(f"rows of {cols} floats expected, got {X.shape}")
    return X


def learned_init(seed):
    """mpcd_learned_init: Glorot-uniform weights, zero biases, unset output scale."""
    p = np.empty(LEARNED_PARAMS, np.float32)
    _check(lib().mpcd_learned_init(seed, _f32p(p)))
    return p


def learned_train(X, Y, params, epochs, batch=256, lr=1e-3, seed=0, device=0):
    """mpcd_learned_train: Adam on the device; returns (trained params, mean loss per epoch)."""
    X, Y = _rows32(X, LEARNED_FEATURES), _rows32(Y, LEARNED_OUTPUTS)
    if len(X) != len(Y):
        raise ValueError("features and targets differ in rows")
    p = _params32(params).copy()
    losses = np.zeros(max(epochs, 1), np.float32)
    _check(lib().mpcd_learned_train(_f32p(X), _f32p(Y), len(X), _f32p(p), epochs, batch, lr, seed, device,
                                    _f32p(losses)))
    return p, losses[:epochs]


def learned_grad(X, Y, params, device=0):
    """mpcd_learned_grad: (gradient, loss) of the mean squared error over all rows."""
    X, Y = _rows32(X, LEARNED_FEATURES), _rows32(Y, LEARNED_OUTPUTS)
    p = _params32(params)
    g = np.empty(LEARNED_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    _check(lib().mpcd_learned_grad(_f32p(X), _f32p(Y), len(X), _f32p(p), device, _f32p(g), _f32p(loss)))
    return g, float(loss[0])


def learned_predict(X, params, device=0):
    """mpcd_learned_predict: the network's kick for feature rows, [rows, 2]."""
    X = _rows32(X, LEARNED_FEATURES)
    p = _params32(params)
    out = np.empty((len(X), LEARNED_OUTPUTS), np.float32)
    _check(lib().mpcd_learned_predict(_f32p(X), len(X), _f32p(p), device, _f32p(out)))
    return out


class _Member(Context):
    """A replica of a Batch: a context the batch owns (not destroyed on its own)."""

    def __init__(self, params, handle):
        self.params = dict(params)
        self.n = int(params["n"])
        self.Nc = int(params["Nc"])
        self.h = handle

    def close(self):
        self.h = None


class Batch:
    """Independent replicas advanced together (mpcd_batch_*): each keeps its own parameters,
    size, state and zone layout; member(i) is the i-th replica's context. form "f64" (the plain
    form) or "fast" (every phase of a step one launch for all replicas)."""

    def __init__(self, params_list, device=0, form="f64"):
        self.params = [dict(p) for p in params_list]
        self.form = form
        arr = (_abi.ParamsC * len(self.params))(*[to_c(p) for p in self.params])
        h = C.c_void_p()
        _check(lib().mpcd_batch_create_form(arr, len(self.params), device, FORMS[form], C.byref(h)))
        self.h = h
        self.members = [_Member(p, lib().mpcd_batch_member(self.h, i)) for i, p in enumerate(self.params)]

    def member(self, i):
        return self.members[i]

    def step(self, step0, nsteps):
        """Advances every replica; returns the device seconds of the whole batch."""
        t = C.c_double()
        _check(lib().mpcd_batch_step(self.h, step0, nsteps, C.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.close()
            lib().mpcd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
