"""Python driver of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads oracle/_build/liboracle.so (built by oracle/Makefile) and runs the restated
reference algorithm on in-memory snapshots.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import this module; the engine never does.

Settings use the reference's IntegratorSettings field names and enum values
(source/granite/IntegratorSettings.hpp:16-181).  Results use the reference's accessor
shapes (source/granite/TrajectorySet.cpp:110-253): trajectories (N, L, D), info (N, L').
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

from . import expr_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


class _Node(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("value", ctypes.c_float),
                ("left", ctypes.c_int32), ("right", ctypes.c_int32)]


_FP = ctypes.POINTER(ctypes.c_float)


class OrInput(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("rk4", ctypes.c_int32), ("border_mode", ctypes.c_int32),
        ("curvature_mode", ctypes.c_int32), ("abort_mode", ctypes.c_int32),
        ("uplift_mode", ctypes.c_int32), ("windfield_mode", ctypes.c_int32),
        ("constants_mode", ctypes.c_int32), ("volume_mode", ctypes.c_int32),
        ("use_topography", ctypes.c_int32), ("reverse", ctypes.c_int32),
        ("use_sphere", ctypes.c_int32), ("time_mode", ctypes.c_int32),
        ("minimum_alive", ctypes.c_int32), ("compensated", ctypes.c_int32), ("save_interval", ctypes.c_int64),
        ("sphere_radius", ctypes.c_float), ("delta_t", ctypes.c_float),
        ("data_time_distance", ctypes.c_float), ("maximum_length", ctypes.c_float),
        ("maximum_simulation_time", ctypes.c_float),
        ("scale", ctypes.c_float * 3), ("offset", ctypes.c_float * 3), ("domain", ctypes.c_float * 3),
        ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
        ("n_volumes", ctypes.c_int32), ("n_constants", ctypes.c_int32),
        ("n_expr", ctypes.c_int32), ("n_snapshots", ctypes.c_int32),
        ("wind", ctypes.POINTER(_FP)), ("volumes", ctypes.POINTER(_FP)),
        ("constants", ctypes.POINTER(_FP)), ("uplift", ctypes.POINTER(_FP)),
        ("topography", _FP),
        ("expr", ctypes.POINTER(ctypes.POINTER(_Node))), ("expr_len", ctypes.POINTER(ctypes.c_int32)),
        ("n", ctypes.c_int64), ("seeds", _FP), ("threads", ctypes.c_int32),
        ("step_limit", ctypes.c_int64), ("filter_weights", ctypes.c_int32),
        ("start_step", ctypes.c_int64),
    ]


class OrOutput(ctypes.Structure):
    _fields_ = [
        ("max_records", ctypes.c_int64), ("positions", _FP), ("status", ctypes.POINTER(ctypes.c_int32)),
        ("lengths", _FP), ("total_curvature", _FP), ("curvature", _FP), ("volume_info", _FP),
        ("compute_info", _FP), ("step_of_abort", ctypes.POINTER(ctypes.c_int64)),
        ("records", ctypes.c_int64), ("curvature_records", ctypes.c_int64),
        ("info_records", ctypes.c_int64), ("steps", ctypes.c_int64),
        ("particle_steps", ctypes.c_int64), ("windows", ctypes.c_int64),
        ("seconds", ctypes.c_double), ("error", ctypes.c_int32), ("message", ctypes.c_char * 256),
    ]


class OrStep(ctypes.Structure):
    _fields_ = [("window", ctypes.c_int64), ("save", ctypes.c_int32), ("time_pos", ctypes.c_int32),
                ("t0", ctypes.c_double), ("t1", ctypes.c_double), ("t2", ctypes.c_double),
                ("t0f", ctypes.c_float), ("t1f", ctypes.c_float), ("t2f", ctypes.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        for name in ("oracle_run_f64", "oracle_run_f32"):
            fn = getattr(_lib, name)
            fn.argtypes = [ctypes.POINTER(OrInput), ctypes.POINTER(OrOutput)]
            fn.restype = ctypes.c_int
        _lib.oracle_schedule.argtypes = [ctypes.POINTER(OrInput), ctypes.POINTER(OrStep),
                                         ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        _lib.oracle_schedule.restype = ctypes.c_int64
    return _lib


# ---------------------------------------------------------------- settings

DEFAULTS = dict(
    SphereRadius=0.0, Space=0, Integrator=1, WindfieldMode=1, ConstantsMode=0,
    AdditionalVolumeMode=0, UpLiftMode=0, DeltaT=1.0, DataTimeDistance=60.0,
    GridScale=[25.0, 25.0, 25.0], Offset=[0.0, 0.0, 0.0], SaveInterval=1, Reverse=False,
    BorderMode=0, CurvatureMode=0, MaximumLength=0.0, MaximumSimulationTime=100.0,
    AbortMode=0, MinimumAliveParticles=0, Topography=None, AdditionalCompute=[],
)


def settings(**kw) -> dict:
    s = dict(DEFAULTS)
    s["GridScale"] = list(DEFAULTS["GridScale"])
    s["Offset"] = list(DEFAULTS["Offset"])
    s["AdditionalCompute"] = []
    for k, v in kw.items():
        if k not in s:
            raise KeyError(k)
        s[k] = v
    return s


def resolve_geometry(s: dict, grid):
    """GridScale / Offset / Domain resolution, TrajectoryIntegrator.tpp:521-574."""
    nx, ny, nz = grid
    gs = [np.float32(v) for v in s["GridScale"]]
    off = [np.float32(v) for v in s["Offset"]]
    if len(gs) == 1:
        scale = [gs[0]] * 3
    elif len(gs) == 2:
        scale = [gs[0], gs[1], gs[0]]
    elif len(gs) == 3:
        scale = list(gs)
    else:
        raise RuntimeError("ERROR < USER INPUT | Invalid GridScale dimension. >")
    if len(off) == 1:
        offset = [off[0]] * 3
    elif len(gs) == 2 and len(off) >= 2:
        offset = [off[0], off[1], off[0]]
    elif len(gs) == 3 and len(off) >= 3:
        offset = list(off)
    else:
        raise RuntimeError("ERROR < USER INPUT | Invalid Offset dimension. >")
    domain = [np.float32(np.float32(nx) * scale[0]), np.float32(np.float32(ny) * scale[1]),
              np.float32(np.float32(nz) * scale[2])]
    return scale, offset, domain


@dataclass
class Inputs:
    """All snapshots in memory: wind[s] is a list of component planes (numpy float32)."""
    wind: list
    seeds: np.ndarray
    volumes: list = field(default_factory=list)      # volumes[s] = {name: plane}
    constants: list = field(default_factory=list)    # constants[s] = {name: (N,)}
    uplift: list = field(default_factory=list)       # uplift[s] = (N, D)
    topography: np.ndarray | None = None


def _ptr(a):
    return a.ctypes.data_as(_FP)


def _build_input(s: dict, data: Inputs, time_mode=0, threads=0, step_limit=-1, compensated=False, filter_weights=0,
                 start_step=0):
    keep = []
    dim = 3 if s["Space"] == 0 else 2
    seeds = np.ascontiguousarray(data.seeds, dtype=np.float32)
    if seeds.ndim != 2 or seeds.shape[1] != dim:
        raise RuntimeError("ERROR < USER INPUT | Dimensions of IntegratorSettings and provided TrajectorySet do not match. >")
    n = seeds.shape[0]
    planes0 = [np.ascontiguousarray(p, dtype=np.float32) for p in data.wind[0]]
    if dim == 3:
        nz, ny, nx = planes0[0].shape
    else:
        (ny, nx), nz = planes0[0].shape, 1
    scale, offset, domain = resolve_geometry(s, (nx, ny, nz))
    ns = len(data.wind)

    def ptr_array(arrs):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in arrs]
        keep.extend(arrs)
        arr = (_FP * max(1, len(arrs)))(*[_ptr(a) for a in arrs])
        keep.append(arr)
        return ctypes.cast(arr, ctypes.POINTER(_FP))

    wind = ptr_array([p for snap in data.wind for p in snap[:dim]])
    vol_names = list(data.volumes[0].keys())[:8] if (data.volumes and s["AdditionalVolumeMode"] != 0) else []
    con_names = list(data.constants[0].keys())[:4] if (data.constants and s["ConstantsMode"] != 0) else []
    volumes = ptr_array([snap[k] for snap in (data.volumes or [{}]) for k in vol_names]) if vol_names else None
    constants = ptr_array([snap[k] for snap in (data.constants or [{}]) for k in con_names]) if con_names else None
    uplift = ptr_array([u.reshape(-1) for u in data.uplift]) if (data.uplift and s["UpLiftMode"] != 0) else None
    topo = None
    if data.topography is not None and dim == 3 and np.asarray(data.topography).size > 0:
        t = np.ascontiguousarray(data.topography, dtype=np.float32)
        keep.append(t)
        topo = _ptr(t)

    exprs = []
    if s["AdditionalCompute"]:
        for code in s["AdditionalCompute"][:4]:
            exprs.append(expr_oracle.compile_expression(
                code, vol_names, con_names, dim, s["CurvatureMode"]))
    nodes_arrs = []
    for e in exprs:
        a = (_Node * len(e))()
        for i, row in enumerate(e):
            a[i] = _Node(int(row["type"]), float(row["value"]), int(row["left"]), int(row["right"]))
        nodes_arrs.append(a)
    keep.extend(nodes_arrs)
    expr_ptrs = (ctypes.POINTER(_Node) * max(1, len(exprs)))(
        *[ctypes.cast(a, ctypes.POINTER(_Node)) for a in nodes_arrs])
    expr_len = (ctypes.c_int32 * max(1, len(exprs)))(*[len(e) for e in exprs])
    keep.extend([expr_ptrs, expr_len, seeds])

    inp = OrInput()
    inp.dim = dim
    inp.rk4 = int(s["Integrator"] == 1)
    inp.border_mode = int(s["BorderMode"]) if dim == 2 else 0
    inp.curvature_mode = int(s["CurvatureMode"])
    inp.abort_mode = int(s["AbortMode"])
    inp.uplift_mode = int(s["UpLiftMode"]) if dim == 3 else 0
    inp.windfield_mode = int(s["WindfieldMode"])
    inp.constants_mode = int(s["ConstantsMode"])
    inp.volume_mode = int(s["AdditionalVolumeMode"])
    inp.use_topography = int(topo is not None)
    inp.reverse = int(bool(s["Reverse"]))
    inp.use_sphere = int(dim == 2 and s["SphereRadius"] > 0)
    inp.time_mode = time_mode
    inp.minimum_alive = int(s["MinimumAliveParticles"])
    inp.compensated = int(bool(compensated))
    inp.save_interval = int(s["SaveInterval"])
    inp.sphere_radius = s["SphereRadius"]
    inp.delta_t = s["DeltaT"]
    inp.data_time_distance = s["DataTimeDistance"]
    inp.maximum_length = s["MaximumLength"]
    inp.maximum_simulation_time = s["MaximumSimulationTime"]
    for d in range(3):
        inp.scale[d] = scale[d]
        inp.offset[d] = offset[d]
        inp.domain[d] = domain[d]
    inp.nx, inp.ny, inp.nz = nx, ny, nz
    inp.n_volumes = len(vol_names)
    inp.n_constants = len(con_names)
    inp.n_expr = len(exprs)
    inp.n_snapshots = ns
    inp.wind = wind
    inp.volumes = volumes
    inp.constants = constants
    inp.uplift = uplift
    inp.topography = topo
    inp.expr = ctypes.cast(expr_ptrs, ctypes.POINTER(ctypes.POINTER(_Node)))
    inp.expr_len = ctypes.cast(expr_len, ctypes.POINTER(ctypes.c_int32))
    inp.n = n
    inp.seeds = _ptr(seeds)
    inp.threads = threads
    inp.step_limit = step_limit
    inp.filter_weights = filter_weights
    inp.start_step = start_step
    meta = dict(dim=dim, n=n, vol_names=vol_names, n_expr=len(exprs), grid=(nx, ny, nz),
                scale=scale, offset=offset, domain=domain)
    return inp, keep, meta


def schedule(s: dict, data: Inputs, time_mode=0):
    """Step schedule without alive checks: list of dicts (window, save, time_pos, t0.. t2f)."""
    inp, keep, _ = _build_input(s, data, time_mode)
    windows = ctypes.c_int64(0)
    k = lib().oracle_schedule(ctypes.byref(inp), None, 0, ctypes.byref(windows))
    if k < 0:
        raise RuntimeError("ERROR < USER INPUT | Cannot increment loader. >")
    steps = (OrStep * max(1, k))()
    lib().oracle_schedule(ctypes.byref(inp), steps, k, ctypes.byref(windows))
    return [dict(window=st.window, save=st.save, time_pos=st.time_pos, t0=st.t0, t1=st.t1, t2=st.t2,
                 t0f=st.t0f, t1f=st.t1f, t2f=st.t2f) for st in steps[:k]], windows.value


def run(s: dict, data: Inputs, precision="f64", time_mode=0, threads=0, step_limit=-1, compensated=False,
        filter_weights=0, start_step=0) -> dict:
    """Runs the oracle; returns outputs in the reference's accessor shapes.  filter_weights: 0 exact
    filter fractions, 1 / 2 fractions rounded / truncated to 1/256 (texture-hardware readings).
    start_step > 0: the particles stay put until that step of the clock, then integrate (a request
    that joins a running clock; the reference has no such form)."""
    inp, keep, meta = _build_input(s, data, time_mode, threads, step_limit, compensated, filter_weights,
                                   start_step)
    n, dim = meta["n"], meta["dim"]
    windows = ctypes.c_int64(0)
    k = lib().oracle_schedule(ctypes.byref(inp), None, 0, ctypes.byref(windows))
    if k < 0:
        raise RuntimeError("ERROR < USER INPUT | Cannot increment loader. >")
    if step_limit >= 0:
        k = min(k, step_limit)
    si = int(s["SaveInterval"])
    max_rec = (1 + (k + si - 1) // si + 1) if si > 0 else 2
    pos = np.zeros((max_rec, n, dim), np.float32)
    status = np.zeros(n, np.int32)
    lengths = np.zeros(n, np.float32)
    tc = np.zeros(n, np.float32)
    curv = np.zeros((max_rec, n), np.float32)
    nv, ne = max(1, len(meta["vol_names"])), max(1, meta["n_expr"])
    vol = np.zeros((nv, max_rec, n), np.float32)
    cmp_ = np.zeros((ne, max_rec, n), np.float32)
    abort_step = np.zeros(n, np.int64)
    out = OrOutput()
    out.max_records = max_rec
    out.positions = _ptr(pos)
    out.status = status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    out.lengths = _ptr(lengths)
    out.total_curvature = _ptr(tc)
    out.curvature = _ptr(curv)
    out.volume_info = _ptr(vol)
    out.compute_info = _ptr(cmp_)
    out.step_of_abort = abort_step.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    fn = lib().oracle_run_f64 if precision == "f64" else lib().oracle_run_f32
    rc = fn(ctypes.byref(inp), ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(out.message.decode())
    L, Lc, Li = out.records, out.curvature_records, out.info_records
    res = dict(
        trajectories=np.ascontiguousarray(pos[:L].transpose(1, 0, 2)),
        status=status, step_of_abort=abort_step,
        lengths=lengths if s["AbortMode"] != 0 else np.zeros(0, np.float32),
        total_curvature=tc if s["CurvatureMode"] != 0 else np.zeros(0, np.float32),
        curvatures=np.ascontiguousarray(curv[:Lc].T) if s["CurvatureMode"] == 3 else np.zeros((n, 0), np.float32),
        volume_info={name: np.ascontiguousarray(vol[i, :Li].T) for i, name in enumerate(meta["vol_names"])},
        compute_info=[np.ascontiguousarray(cmp_[e, :Li].T) for e in range(meta["n_expr"])],
        steps=out.steps, particle_steps=out.particle_steps, windows=out.windows,
        seconds=out.seconds, meta=meta,
    )
    return res
