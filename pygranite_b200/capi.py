"""ctypes view of the C ABI in include/granite_b200.h (libgranite_b200.so).

The pybind11 module is the pygranite-compatible surface; this module is for callers that
bind the C ABI directly (the benchmark's device-resident path, ABI tests).
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgranite_b200.so")

GR_OK, GR_ERR_USER, GR_ERR_RUNTIME, GR_ERR_CALLBACK = 0, -1, -2, -3

# Every entry point declared in include/granite_b200.h.
EXPORTS = [
    "gr_settings_default", "gr_create", "gr_destroy", "gr_last_error", "gr_load_windfield",
    "gr_load_volume", "gr_load_constant", "gr_load_uplift", "gr_set_topography",
    "gr_compile_expression", "gr_expression_evaluate", "gr_set_seeds", "gr_run",
    "gr_result_info_get", "gr_stats_get", "gr_fetch_positions", "gr_fetch_status",
    "gr_fetch_lengths", "gr_fetch_total_curvature", "gr_fetch_curvatures",
    "gr_fetch_volume_info", "gr_fetch_compute_info", "gr_load_windfield_device",
    "gr_set_seeds_device", "gr_plan", "gr_advance_noalloc", "gr_update_settings", "gr_settings_get",
    "gr_set_lifetimes", "gr_batch_create", "gr_batch_destroy", "gr_batch_run", "gr_batch_stats_get", "gr_tune",
    "gr_fetch_final_positions", "gr_server_create", "gr_server_set_snapshot", "gr_server_start",
    "gr_server_submit", "gr_server_wait", "gr_server_result", "gr_server_release", "gr_server_cancel",
    "gr_server_stats_get", "gr_server_destroy", "gr_field_double_gyre", "gr_field_fourier", "gr_field_load",
    "gr_field_loader", "gr_field_snapshot", "gr_field_destroy", "gr_host_alloc", "gr_host_free",
    "gr_host_cache_limit", "gr_host_cache_trim", "gr_host_cache_stats_get", "gr_host_is_pinned",
    "gr_device_cache_stats_get", "gr_device_cache_trim", "gr_set_result_destinations",
]

GR_REQ_PENDING, GR_REQ_ACTIVE, GR_REQ_DONE, GR_REQ_CANCELLED, GR_REQ_FAILED = 0, 1, 2, 3, 4


class Settings(ctypes.Structure):
    _fields_ = [
        ("space", ctypes.c_int32), ("integrator", ctypes.c_int32), ("windfield_mode", ctypes.c_int32),
        ("constants_mode", ctypes.c_int32), ("volume_mode", ctypes.c_int32), ("uplift_mode", ctypes.c_int32),
        ("border_mode", ctypes.c_int32), ("curvature_mode", ctypes.c_int32), ("abort_mode", ctypes.c_int32),
        ("reverse", ctypes.c_int32), ("minimum_alive", ctypes.c_int32), ("grid_scale_len", ctypes.c_int32),
        ("offset_len", ctypes.c_int32), ("sphere_radius", ctypes.c_float), ("delta_t", ctypes.c_float),
        ("data_time_distance", ctypes.c_float), ("maximum_length", ctypes.c_float),
        ("maximum_simulation_time", ctypes.c_float), ("grid_scale", ctypes.c_float * 3),
        ("offset", ctypes.c_float * 3), ("save_interval", ctypes.c_int64), ("storage", ctypes.c_int32),
        ("time_mode", ctypes.c_int32), ("compensated", ctypes.c_int32), ("ring_slots", ctypes.c_int32),
        ("steps_per_launch", ctypes.c_int32), ("sort_interval", ctypes.c_int32), ("block_size", ctypes.c_int32),
        ("device", ctypes.c_int32), ("layout", ctypes.c_int32), ("grid_waves", ctypes.c_int32),
        ("filter_weights", ctypes.c_int32),
    ]


class ResultInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dim", ctypes.c_int32), ("records", ctypes.c_int64),
                ("curvature_records", ctypes.c_int64), ("info_records", ctypes.c_int64),
                ("steps", ctypes.c_int64), ("windows", ctypes.c_int64), ("particle_steps", ctypes.c_int64),
                ("n_volumes", ctypes.c_int32), ("n_expressions", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("run_ms", ctypes.c_double), ("launches", ctypes.c_int64),
                ("aux_launches", ctypes.c_int64), ("particle_steps", ctypes.c_int64),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64), ("jit_launches", ctypes.c_int64)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("windows", ctypes.c_int64), ("records", ctypes.c_int64),
                ("curvature_records", ctypes.c_int64), ("info_records", ctypes.c_int64)]


class BatchStats(ctypes.Structure):
    _fields_ = [("graph_ms", ctypes.c_double), ("nodes", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("aux_launches", ctypes.c_int64), ("particle_steps", ctypes.c_int64), ("captures", ctypes.c_int64),
                ("replays", ctypes.c_int64)]


class TuneResult(ctypes.Structure):
    _fields_ = [("layout", ctypes.c_int32), ("block_size", ctypes.c_int32), ("sort_interval", ctypes.c_int32),
                ("grid_waves", ctypes.c_int32), ("particle_steps_per_s", ctypes.c_double), ("trials", ctypes.c_int32)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dim", ctypes.c_int32), ("integrator", ctypes.c_int32),
                ("start_step", ctypes.c_int64), ("steps", ctypes.c_int64), ("submit_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double), ("state", ctypes.c_int32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "submitted", "admitted", "completed", "cancelled", "deferred", "windows", "sweeps", "jumps",
        "particle_steps", "capacity_particles", "peak_particles", "h2d_bytes", "d2h_bytes", "pending", "active",
        "clock_steps", "windows_per_sweep", "staged_later")]


class ResultDestinations(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("records_capacity", ctypes.c_int64),
                ("volume_info", ctypes.c_void_p * 8), ("compute_info", ctypes.c_void_p * 4),
                ("info_capacity", ctypes.c_int64)]


class HostCacheStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("live_bytes", "cached_bytes", "limit_bytes", "allocations", "reuses")]


LOADER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build with `make -C pygranite_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH)
        P, I32, I64, FP = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)
        CP = ctypes.POINTER(ctypes.c_char_p)
        sig = {
            "gr_settings_default": (None, [ctypes.POINTER(Settings)]),
            "gr_create": (ctypes.c_int, [ctypes.POINTER(Settings), ctypes.POINTER(P)]),
            "gr_destroy": (None, [P]),
            "gr_last_error": (ctypes.c_char_p, []),
            "gr_load_windfield": (ctypes.c_int, [P, I64, ctypes.POINTER(FP), I32, I64, I64, I64]),
            "gr_load_windfield_device": (ctypes.c_int, [P, I64, ctypes.POINTER(P), I32, I64, I64, I64]),
            "gr_load_volume": (ctypes.c_int, [P, I64, I32, FP, I64, I64, I64]),
            "gr_load_constant": (ctypes.c_int, [P, I64, I32, FP, I64]),
            "gr_load_uplift": (ctypes.c_int, [P, I64, FP, I64, I32]),
            "gr_set_topography": (ctypes.c_int, [P, FP, I64, I64]),
            "gr_compile_expression": (ctypes.c_int, [P, I32, ctypes.c_char_p, CP, I32, CP, I32]),
            "gr_expression_evaluate": (ctypes.c_int, [ctypes.c_char_p, CP, I32, CP, I32, I32, I32, FP, FP]),
            "gr_set_seeds": (ctypes.c_int, [P, FP, I64, I32]),
            "gr_set_seeds_device": (ctypes.c_int, [P, P, I64, I32]),
            "gr_run": (ctypes.c_int, [P, LOADER_FN, P]),
            "gr_result_info_get": (ctypes.c_int, [P, ctypes.POINTER(ResultInfo)]),
            "gr_stats_get": (ctypes.c_int, [P, ctypes.POINTER(Stats)]),
            "gr_fetch_positions": (ctypes.c_int, [P, FP, I64]),
            "gr_fetch_status": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int32), I64]),
            "gr_fetch_lengths": (ctypes.c_int, [P, FP, I64]),
            "gr_fetch_total_curvature": (ctypes.c_int, [P, FP, I64]),
            "gr_fetch_curvatures": (ctypes.c_int, [P, FP, I64]),
            "gr_fetch_volume_info": (ctypes.c_int, [P, I32, FP, I64]),
            "gr_fetch_compute_info": (ctypes.c_int, [P, I32, FP, I64]),
            "gr_plan": (ctypes.c_int, [ctypes.POINTER(Settings), ctypes.POINTER(PlanInfo), I64,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32), FP]),
            "gr_advance_noalloc": (ctypes.c_int, [ctypes.POINTER(Settings), I64, I64, I64, P, P, ctypes.c_float,
                                                  ctypes.c_float, ctypes.c_float, I32, P, P, P, P, I64, P,
                                                  ctypes.POINTER(ctypes.c_int64)]),
            "gr_update_settings": (ctypes.c_int, [P, ctypes.POINTER(Settings)]),
            "gr_settings_get": (ctypes.c_int, [P, ctypes.POINTER(Settings)]),
            "gr_set_lifetimes": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int32), I64]),
            "gr_batch_create": (ctypes.c_int, [ctypes.POINTER(P), I32, ctypes.POINTER(P)]),
            "gr_batch_destroy": (None, [P]),
            "gr_batch_run": (ctypes.c_int, [P]),
            "gr_batch_stats_get": (ctypes.c_int, [P, ctypes.POINTER(BatchStats)]),
            "gr_tune": (ctypes.c_int, [P, I32, ctypes.POINTER(TuneResult)]),
            "gr_fetch_final_positions": (ctypes.c_int, [P, FP, I64]),
            "gr_server_create": (ctypes.c_int, [ctypes.POINTER(Settings), I64, I64, I64, I64, I64, ctypes.POINTER(P)]),
            "gr_server_set_snapshot": (ctypes.c_int, [P, I64, ctypes.POINTER(P), I32, I32]),
            "gr_server_start": (ctypes.c_int, [P]),
            "gr_server_submit": (ctypes.c_int, [P, FP, I64, I32, ctypes.c_double, I32, I32,
                                                ctypes.POINTER(ctypes.c_int64)]),
            "gr_server_wait": (ctypes.c_int, [P, I64, ctypes.c_double, ctypes.POINTER(ctypes.c_int32)]),
            "gr_server_result": (ctypes.c_int, [P, I64, ctypes.POINTER(RequestInfo), FP,
                                                ctypes.POINTER(ctypes.c_int32), I64]),
            "gr_server_release": (ctypes.c_int, [P, I64]),
            "gr_server_cancel": (ctypes.c_int, [P, I64]),
            "gr_server_stats_get": (ctypes.c_int, [P, ctypes.POINTER(ServerStats)]),
            "gr_server_destroy": (None, [P]),
            "gr_field_double_gyre": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_double, I64, I64, ctypes.c_double, ctypes.c_double, ctypes.c_double, I64, I32,
                                                    ctypes.POINTER(P)]),
            "gr_field_fourier": (ctypes.c_int, [I32, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double), I32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_double, I64,
                                                I32, ctypes.POINTER(P)]),
            "gr_field_load": (ctypes.c_int, [P, P, I64]),
            "gr_field_loader": (ctypes.c_int, [P, P, I64]),
            "gr_field_snapshot": (ctypes.c_int, [P, I64, FP, I64]),
            "gr_field_destroy": (None, [P]),
            "gr_host_alloc": (ctypes.c_int, [I64, ctypes.POINTER(P)]),
            "gr_host_free": (ctypes.c_int, [P]),
            "gr_host_cache_limit": (ctypes.c_int, [I64]),
            "gr_host_cache_trim": (ctypes.c_int, []),
            "gr_host_cache_stats_get": (ctypes.c_int, [ctypes.POINTER(HostCacheStats)]),
            "gr_host_is_pinned": (ctypes.c_int, [P]),
            "gr_device_cache_stats_get": (ctypes.c_int, [I32, ctypes.POINTER(ctypes.c_int64),
                                                         ctypes.POINTER(ctypes.c_int64)]),
            "gr_device_cache_trim": (ctypes.c_int, []),
            "gr_set_result_destinations": (ctypes.c_int, [P, ctypes.POINTER(ResultDestinations)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class GraniteError(RuntimeError):
    pass


def _check(rc):
    if rc != GR_OK:
        raise GraniteError(lib().gr_last_error().decode())


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _names(names):
    arr = (ctypes.c_char_p * max(1, len(names)))(*[n.encode() for n in names])
    return ctypes.cast(arr, ctypes.POINTER(ctypes.c_char_p)), arr


def default_settings(**kw) -> Settings:
    s = Settings()
    lib().gr_settings_default(ctypes.byref(s))
    for k, v in kw.items():
        if k in ("grid_scale", "offset"):
            arr = getattr(s, k)
            for i, x in enumerate(v):
                arr[i] = x
            setattr(s, k + "_len", len(v))
        else:
            setattr(s, k, v)
    return s


def settings_from_reference(d: dict, **extra) -> Settings:
    """gr_settings from a dict of reference IntegratorSettings field names (int enums)."""
    m = dict(space=d.get("Space", 0), integrator=d.get("Integrator", 1), windfield_mode=d.get("WindfieldMode", 1),
             constants_mode=d.get("ConstantsMode", 0), volume_mode=d.get("AdditionalVolumeMode", 0),
             uplift_mode=d.get("UpLiftMode", 0), border_mode=d.get("BorderMode", 0),
             curvature_mode=d.get("CurvatureMode", 0), abort_mode=d.get("AbortMode", 0),
             reverse=int(bool(d.get("Reverse", False))), minimum_alive=d.get("MinimumAliveParticles", 0),
             sphere_radius=d.get("SphereRadius", 0.0), delta_t=d.get("DeltaT", 1.0),
             data_time_distance=d.get("DataTimeDistance", 60.0), maximum_length=d.get("MaximumLength", 0.0),
             maximum_simulation_time=d.get("MaximumSimulationTime", 100.0),
             grid_scale=d.get("GridScale", [25.0, 25.0, 25.0]), offset=d.get("Offset", [0.0, 0.0, 0.0]),
             save_interval=d.get("SaveInterval", 1))
    m.update(extra)
    return default_settings(**m)


def plan(settings: Settings, with_steps=True):
    """gr_plan: counts and (optionally) per-step window, flags and float32 time weights."""
    info = PlanInfo()
    _check(lib().gr_plan(ctypes.byref(settings), ctypes.byref(info), 0, None, None, None))
    if not with_steps:
        return info, None
    n = info.steps
    win = np.zeros(max(1, n), np.int64)
    flags = np.zeros(max(1, n), np.int32)
    w = np.zeros((max(1, n), 3), np.float32)
    _check(lib().gr_plan(ctypes.byref(settings), ctypes.byref(info), n,
                         win.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _fp(w)))
    return info, dict(window=win[:n], flags=flags[:n], weights=w[:n])


def advance_noalloc(settings: Settings, shape, wind_back_ptr, wind_front_ptr, time_back, time_front, time_start,
                    steps, px_ptr, py_ptr, pz_ptr, status_ptr, n, stream_ptr=None):
    """gr_advance_noalloc on caller-owned device buffers (raw pointers); returns particle-steps."""
    nz, ny, nx = shape if len(shape) == 3 else (1,) + tuple(shape)
    ps = ctypes.c_int64(0)
    _check(lib().gr_advance_noalloc(ctypes.byref(settings), nz, ny, nx, wind_back_ptr, wind_front_ptr, time_back,
                                    time_front, time_start, steps, px_ptr, py_ptr, pz_ptr, status_ptr, n,
                                    stream_ptr, ctypes.byref(ps)))
    return ps.value


def evaluate_expression(code, ref, volume_names=(), constant_names=(), dim=3, curvature_mode=0):
    """Host evaluation through gr_expression_evaluate (no GPU needed)."""
    vn, _k1 = _names(list(volume_names))
    cn, _k2 = _names(list(constant_names))
    r = np.ascontiguousarray(ref, np.float32)
    out = ctypes.c_float(0.0)
    _check(lib().gr_expression_evaluate(code.encode(), vn, len(volume_names), cn, len(constant_names), dim,
                                        curvature_mode, _fp(r), ctypes.byref(out)))
    return out.value


def pinned_empty(shape, dtype=np.float32):
    """Uninitialised array in page-locked host memory from gr_host_alloc; the block returns to the
    library's cache when the array is released.  Loads from and fetches into such arrays are
    single DMAs."""
    dtype = np.dtype(dtype)
    shape = tuple(int(d) for d in (shape if isinstance(shape, (tuple, list)) else (shape,)))
    nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
    if nbytes == 0:
        return np.empty(shape, dtype)
    p = ctypes.c_void_p()
    _check(lib().gr_host_alloc(nbytes, ctypes.byref(p)))
    buf = (ctypes.c_char * nbytes).from_address(p.value)
    weakref.finalize(buf, lib().gr_host_free, ctypes.c_void_p(p.value))
    return np.frombuffer(buf, dtype=dtype).reshape(shape)


def is_pinned(a) -> bool:
    """True when the array's data lies in page-locked host memory known to CUDA."""
    a = np.asarray(a)
    return a.nbytes > 0 and bool(lib().gr_host_is_pinned(ctypes.c_void_p(a.ctypes.data))) and \
        bool(lib().gr_host_is_pinned(ctypes.c_void_p(a.ctypes.data + a.nbytes - 1)))


def host_cache_stats() -> HostCacheStats:
    out = HostCacheStats()
    _check(lib().gr_host_cache_stats_get(ctypes.byref(out)))
    return out


def host_cache_limit(nbytes: int):
    _check(lib().gr_host_cache_limit(int(nbytes)))


def host_cache_trim():
    _check(lib().gr_host_cache_trim())


def device_cache_stats(device=0):
    """(reserved, used) bytes of the library's device memory pool on `device`."""
    r, u = ctypes.c_int64(), ctypes.c_int64()
    _check(lib().gr_device_cache_stats_get(device, ctypes.byref(r), ctypes.byref(u)))
    return r.value, u.value


def device_cache_trim():
    _check(lib().gr_device_cache_trim())


class Engine:
    """Thin owner of a gr_engine*."""

    def __init__(self, settings: Settings):
        self.h = ctypes.c_void_p()
        _check(lib().gr_create(ctypes.byref(settings), ctypes.byref(self.h)))
        self.dim = 3 if settings.space == 0 else 2
        self._keep = []

    def close(self):
        if self.h:
            lib().gr_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_windfield(self, snapshot, planes):
        planes = [np.ascontiguousarray(p, np.float32) for p in planes]
        arr = (ctypes.POINTER(ctypes.c_float) * len(planes))(*[_fp(p) for p in planes])
        shp = planes[0].shape
        nz, ny, nx = (shp if len(shp) == 3 else (1,) + tuple(shp))
        _check(lib().gr_load_windfield(self.h, snapshot, arr, len(planes), nz, ny, nx))

    def load_windfield_device(self, snapshot, ptrs, shape):
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        nz, ny, nx = (shape if len(shape) == 3 else (1,) + tuple(shape))
        _check(lib().gr_load_windfield_device(self.h, snapshot, arr, len(ptrs), nz, ny, nx))

    def load_volume(self, snapshot, index, plane):
        p = np.ascontiguousarray(plane, np.float32)
        shp = p.shape
        nz, ny, nx = (shp if len(shp) == 3 else (1,) + tuple(shp))
        _check(lib().gr_load_volume(self.h, snapshot, index, _fp(p), nz, ny, nx))

    def load_constant(self, snapshot, index, values):
        v = np.ascontiguousarray(values, np.float32)
        _check(lib().gr_load_constant(self.h, snapshot, index, _fp(v), v.size))

    def load_uplift(self, snapshot, values):
        v = np.ascontiguousarray(values, np.float32)
        _check(lib().gr_load_uplift(self.h, snapshot, _fp(v), v.shape[0], v.shape[1]))

    def set_topography(self, topo):
        t = np.ascontiguousarray(topo, np.float32)
        _check(lib().gr_set_topography(self.h, _fp(t), t.shape[0], t.shape[1]))

    def compile_expression(self, index, code, volume_names=(), constant_names=()):
        vn, k1 = _names(list(volume_names))
        cn, k2 = _names(list(constant_names))
        _check(lib().gr_compile_expression(self.h, index, code.encode(), vn, len(volume_names), cn,
                                           len(constant_names)))

    def set_seeds(self, seeds):
        s = np.ascontiguousarray(seeds, np.float32)
        _check(lib().gr_set_seeds(self.h, _fp(s), s.shape[0], s.shape[1]))

    def set_seeds_device(self, ptr, n, dim):
        _check(lib().gr_set_seeds_device(self.h, ptr, n, dim))

    def set_lifetimes(self, steps):
        """Per-particle lifetimes in steps (None clears them)."""
        if steps is None:
            _check(lib().gr_set_lifetimes(self.h, None, 0))
            return
        a = np.ascontiguousarray(steps, np.int32)
        _check(lib().gr_set_lifetimes(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), a.size))

    def settings(self) -> Settings:
        s = Settings()
        _check(lib().gr_settings_get(self.h, ctypes.byref(s)))
        return s

    def update_settings(self, **kw):
        """Changes run options (gr_update_settings) by field name."""
        s = self.settings()
        for k, v in kw.items():
            setattr(s, k, v)
        _check(lib().gr_update_settings(self.h, ctypes.byref(s)))

    def tune(self, trial_steps=40) -> TuneResult:
        r = TuneResult()
        _check(lib().gr_tune(self.h, trial_steps, ctypes.byref(r)))
        return r

    def status(self):
        n = self.info().n
        st = np.empty(n, np.int32)
        _check(lib().gr_fetch_status(self.h, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n))
        return st

    def final_positions(self):
        info = self.info()
        out = np.empty((info.n, info.dim), np.float32)
        _check(lib().gr_fetch_final_positions(self.h, _fp(out), out.size))
        return out

    def run(self, loader=None):
        """loader(snapshot) -> 1 / 0 / negative; None = the ring already holds every snapshot."""
        def cb(user, eng, snapshot):
            try:
                return int(loader(snapshot)) if loader is not None else 0
            except Exception:  # the error is reported through the status code
                return -1
        fn = LOADER_FN(cb)
        self._keep.append(fn)
        _check(lib().gr_run(self.h, fn, None))

    def run_native(self, field):
        """gr_run fed by a native device loader (gr_field_loader): no Python in the loop."""
        fn = LOADER_FN(ctypes.cast(lib().gr_field_loader, ctypes.c_void_p).value)
        _check(lib().gr_run(self.h, fn, field.h))

    def info(self) -> ResultInfo:
        r = ResultInfo()
        _check(lib().gr_result_info_get(self.h, ctypes.byref(r)))
        return r

    def stats(self) -> Stats:
        s = Stats()
        _check(lib().gr_stats_get(self.h, ctypes.byref(s)))
        return s

    def stream_results(self, positions=None, volume_info=(), compute_info=()):
        """Page-locked arrays that later runs fill while they go (gr_set_result_destinations):
        positions (n, records_capacity, dim), volume / compute info (n, info_capacity) each.
        No arguments turns streaming off."""
        if positions is None and not volume_info and not compute_info:
            self._streamed = None
            _check(lib().gr_set_result_destinations(self.h, None))
            return
        d = ResultDestinations()
        if positions is not None:
            d.positions = positions.ctypes.data
            d.records_capacity = positions.shape[1]
        caps = [a.shape[1] for a in list(volume_info) + list(compute_info) if a is not None]
        d.info_capacity = caps[0] if caps else 0
        for k, a in enumerate(volume_info):
            d.volume_info[k] = a.ctypes.data if a is not None and a.size else None
        for k, a in enumerate(compute_info):
            d.compute_info[k] = a.ctypes.data if a is not None and a.size else None
        self._streamed = (positions, list(volume_info), list(compute_info))   # kept alive
        _check(lib().gr_set_result_destinations(self.h, ctypes.byref(d)))

    def results(self, volumes=True, compute=True, pinned=False):
        """Every result array; pinned=True places the record arrays in page-locked memory
        (pinned_empty), which the engine fills by one DMA each."""
        info = self.info()
        n, L, D = info.n, info.records, info.dim
        alloc = pinned_empty if pinned else np.empty
        pos = alloc((n, L, D), np.float32)
        _check(lib().gr_fetch_positions(self.h, _fp(pos), pos.size))
        st = np.empty(n, np.int32)
        _check(lib().gr_fetch_status(self.h, st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n))
        out = dict(trajectories=pos, status=st, info=info)
        ln = np.zeros(n, np.float32)
        _check(lib().gr_fetch_lengths(self.h, _fp(ln), n))
        tc = np.zeros(n, np.float32)
        _check(lib().gr_fetch_total_curvature(self.h, _fp(tc), n))
        cv = np.zeros((n, info.curvature_records), np.float32)
        if info.curvature_records:
            _check(lib().gr_fetch_curvatures(self.h, _fp(cv), cv.size))
        out.update(lengths=ln, total_curvature=tc, curvatures=cv)
        if volumes:
            vols = []
            for k in range(info.n_volumes):
                a = alloc((n, info.info_records), np.float32)
                _check(lib().gr_fetch_volume_info(self.h, k, _fp(a), a.size))
                vols.append(a)
            out["volume_info"] = vols
        if compute:
            cmps = []
            for k in range(info.n_expressions):
                a = alloc((n, info.info_records), np.float32)
                _check(lib().gr_fetch_compute_info(self.h, k, _fp(a), a.size))
                cmps.append(a)
            out["compute_info"] = cmps
        return out


class Batch:
    """gr_batch: the runs of several engines as one CUDA graph (captured on the first run)."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        self.h = ctypes.c_void_p()
        _check(lib().gr_batch_create(arr, len(self.engines), ctypes.byref(self.h)))

    def run(self):
        _check(lib().gr_batch_run(self.h))

    def stats(self) -> BatchStats:
        s = BatchStats()
        _check(lib().gr_batch_stats_get(self.h, ctypes.byref(s)))
        return s

    def close(self):
        if self.h:
            lib().gr_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """gr_server: trajectory requests served with continuous batching over one field."""

    def __init__(self, settings: Settings, n_snapshots, shape, hbm_budget=0):
        nz, ny, nx = shape if len(shape) == 3 else (1,) + tuple(shape)
        self.dim = 3 if settings.space == 0 else 2
        self.h = ctypes.c_void_p()
        _check(lib().gr_server_create(ctypes.byref(settings), n_snapshots, nz, ny, nx, hbm_budget,
                                      ctypes.byref(self.h)))

    def set_snapshot(self, k, planes):
        """Host float32 planes (numpy)."""
        planes = [np.ascontiguousarray(p, np.float32) for p in planes]
        arr = (ctypes.c_void_p * len(planes))(*[p.ctypes.data for p in planes])
        _check(lib().gr_server_set_snapshot(self.h, k, arr, len(planes), 0))

    def set_snapshot_device(self, k, ptrs):
        """Device float32 planes (raw pointers)."""
        arr = (ctypes.c_void_p * len(ptrs))(*ptrs)
        _check(lib().gr_server_set_snapshot(self.h, k, arr, len(ptrs), 1))

    def start(self):
        _check(lib().gr_server_start(self.h))

    def submit(self, seeds, start_time, steps, integrator=1):
        s = np.ascontiguousarray(seeds, np.float32)
        rid = ctypes.c_int64(0)
        _check(lib().gr_server_submit(self.h, _fp(s), s.shape[0], s.shape[1], float(start_time), int(steps),
                                      int(integrator), ctypes.byref(rid)))
        return rid.value

    def wait(self, rid, timeout=-1.0):
        st = ctypes.c_int32(0)
        _check(lib().gr_server_wait(self.h, rid, float(timeout), ctypes.byref(st)))
        return st.value

    def info(self, rid) -> RequestInfo:
        r = RequestInfo()
        _check(lib().gr_server_result(self.h, rid, ctypes.byref(r), None, None, 0))
        return r

    def result(self, rid):
        info = self.info(rid)
        pos = np.empty((info.n, info.dim), np.float32)
        st = np.empty(info.n, np.int32)
        _check(lib().gr_server_result(self.h, rid, None, _fp(pos), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                      info.n))
        return pos, st, info

    def cancel(self, rid):
        _check(lib().gr_server_cancel(self.h, rid))

    def release(self, rid):
        _check(lib().gr_server_release(self.h, rid))

    def stats(self) -> ServerStats:
        s = ServerStats()
        _check(lib().gr_server_stats_get(self.h, ctypes.byref(s)))
        return s

    def close(self):
        if self.h:
            lib().gr_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Field:
    """gr_field: an analytic windfield evaluated on the device, snapshot by snapshot."""

    def __init__(self, handle, shape):
        self.h, self.shape = handle, tuple(shape)

    @classmethod
    def double_gyre(cls, A=0.1, eps=0.25, omega=2 * np.pi / 10, ny=128, nx=256, lx=2.0, ly=1.0, dt=1.0,
                    n_snapshots=16, device=0):
        h = ctypes.c_void_p()
        _check(lib().gr_field_double_gyre(A, eps, omega, ny, nx, lx, ly, dt, n_snapshots, device, ctypes.byref(h)))
        return cls(h, (ny, nx))

    @classmethod
    def fourier(cls, field, dt, n_snapshots, device=0):
        """From a workloads.FourierField: the same wave vectors, amplitudes, phases and scaling."""
        dim, m = field.dim, len(field.comps[0]["amp"])
        k = np.ascontiguousarray(np.stack([c["kvec"] for c in field.comps]), np.float64)      # (dim, m, dim)
        amp = np.ascontiguousarray(np.stack([c["amp"] for c in field.comps]), np.float64)
        ph = np.ascontiguousarray(np.stack([c["phase0"] for c in field.comps]), np.float64)
        om = np.ascontiguousarray(np.stack([c["omega"] for c in field.comps]), np.float64)
        sc = np.ascontiguousarray([c["scale"] for c in field.comps], np.float64)
        shape = np.ascontiguousarray(field.shape, np.int64)
        sp = np.ascontiguousarray(field.spacing, np.float64)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        h = ctypes.c_void_p()
        _check(lib().gr_field_fourier(dim, shape.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), dp(sp), m, dp(k),
                                      dp(amp), dp(ph), dp(om), dp(sc), dt, n_snapshots, device, ctypes.byref(h)))
        return cls(h, field.shape)

    def load(self, engine, snapshot):
        _check(lib().gr_field_load(self.h, engine.h, snapshot))

    def snapshot(self, k):
        """Snapshot k as float32 planes, (dim, *shape)."""
        out = np.empty((len(self.shape),) + self.shape, np.float32)
        _check(lib().gr_field_snapshot(self.h, k, _fp(out), out.size))
        return out

    def close(self):
        if self.h:
            lib().gr_field_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
