"""ctypes driver of oracle/_ref/libref_integrate.so (TEST INFRASTRUCTURE ONLY).

Runs the reference's own `integrate` kernel (built from its sources by
oracle/ref_harness/Makefile) on a GPU; used by tests/golden/make_golden.py to write golden
fixtures and by the GPU tests to time the reference kernel as shipped.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import expr_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "_ref", "libref_integrate.so")

_FP = ctypes.POINTER(ctypes.c_float)


class ASTANode(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("value", ctypes.c_float), ("left", ctypes.c_int32),
                ("right", ctypes.c_int32)]


class RefArgs(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int32), ("blocks_fixed", ctypes.c_int32),
        ("delta_t", ctypes.c_float), ("data_time_distance", ctypes.c_float),
        ("maximum_simulation_time", ctypes.c_float), ("save_interval", ctypes.c_int64),
        ("scale", ctypes.c_float * 3), ("offset", ctypes.c_float * 3),
        ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
        ("n_snapshots", ctypes.c_int32), ("wind", ctypes.POINTER(_FP)), ("volume", _FP),
        ("ast", ctypes.POINTER(ASTANode)), ("ast_len", ctypes.c_int32),
        ("n", ctypes.c_int64), ("seeds", _FP), ("step_limit", ctypes.c_int64),
        ("max_records", ctypes.c_int64), ("positions", _FP), ("status", ctypes.POINTER(ctypes.c_int32)),
        ("total_curvature", _FP), ("volume_info", _FP), ("compute_info", _FP),
        ("records", ctypes.c_int64), ("info_records", ctypes.c_int64), ("steps", ctypes.c_int64),
        ("windows", ctypes.c_int64), ("loop_ms", ctypes.c_double), ("threads", ctypes.c_int32),
        ("blocks", ctypes.c_int32), ("message", ctypes.c_char * 256),
        ("count_steps", ctypes.c_int32), ("particle_steps", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
    ]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def run(settings: dict, wind, seeds, volume=None, blocks_fixed=False, step_limit=-1, count_steps=False):
    """settings: reference IntegratorSettings fields (as in oracle.oracle.settings).  The
    variant is chosen from them: 2D Euler plain, 3D RK4 + TotalCurvature + one constant
    volume + one expression, 3D RK4 plain, or 3D Euler plain."""
    lib = ctypes.CDLL(LIB_PATH)
    lib.ref_run.argtypes = [ctypes.POINTER(RefArgs)]
    lib.ref_run.restype = ctypes.c_int
    dim = 3 if settings["Space"] == 0 else 2
    a = RefArgs()
    if dim == 2:
        a.variant = 0
    elif settings.get("AdditionalCompute"):
        a.variant = 1
    elif settings.get("Integrator", 1) == 0:
        a.variant = 3
    else:
        a.variant = 2
    a.blocks_fixed = int(blocks_fixed)
    a.count_steps = int(count_steps)
    a.delta_t = settings["DeltaT"]
    a.data_time_distance = settings["DataTimeDistance"]
    a.maximum_simulation_time = settings["MaximumSimulationTime"]
    a.save_interval = settings["SaveInterval"]
    gs = list(settings["GridScale"]) + [settings["GridScale"][0]] * (3 - len(settings["GridScale"]))
    of = list(settings["Offset"]) + [settings["Offset"][0]] * (3 - len(settings["Offset"]))
    for d in range(3):
        a.scale[d] = gs[d]
        a.offset[d] = of[d]
    planes = [np.ascontiguousarray(p, np.float32) for snap in wind for p in snap[:dim]]
    shp = planes[0].shape
    if dim == 3:
        a.nz, a.ny, a.nx = shp
    else:
        a.nz, (a.ny, a.nx) = 1, shp
    a.n_snapshots = len(wind)
    arr = (_FP * len(planes))(*[p.ctypes.data_as(_FP) for p in planes])
    a.wind = ctypes.cast(arr, ctypes.POINTER(_FP))
    keep = [planes, arr]
    if a.variant == 1:
        vol = np.ascontiguousarray(volume, np.float32)
        keep.append(vol)
        a.volume = vol.ctypes.data_as(_FP)
        flat = expr_oracle.compile_expression(settings["AdditionalCompute"][0], ["T"], [], 3,
                                              settings.get("CurvatureMode", 0))
        nodes = (ASTANode * len(flat))(*[ASTANode(int(r["type"]), float(r["value"]), int(r["left"]),
                                                  int(r["right"])) for r in flat])
        keep.append(nodes)
        a.ast = ctypes.cast(nodes, ctypes.POINTER(ASTANode))
        a.ast_len = len(flat)
    sd = np.ascontiguousarray(seeds, np.float32)
    n = sd.shape[0]
    a.n = n
    a.seeds = sd.ctypes.data_as(_FP)
    a.step_limit = step_limit
    steps_max = int(a.maximum_simulation_time / a.delta_t) + 2
    if step_limit >= 0:
        steps_max = min(steps_max, step_limit + 1)
    si = int(a.save_interval)
    max_rec = (1 + steps_max // si + 1) if si > 0 else 2
    pos = np.zeros((max_rec, n, dim), np.float32)
    st = np.zeros(n, np.int32)
    tc = np.zeros(n, np.float32)
    vi = np.zeros((max_rec, n), np.float32)
    ci = np.zeros((max_rec, n), np.float32)
    a.max_records = max_rec
    a.positions = pos.ctypes.data_as(_FP)
    a.status = st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    a.total_curvature = tc.ctypes.data_as(_FP)
    a.volume_info = vi.ctypes.data_as(_FP)
    a.compute_info = ci.ctypes.data_as(_FP)
    rc = lib.ref_run(ctypes.byref(a))
    if rc != 0:
        raise RuntimeError("reference harness: " + a.message.decode())
    L, Li = a.records, a.info_records
    return dict(trajectories=np.ascontiguousarray(pos[:L].transpose(1, 0, 2)), status=st,
                total_curvature=tc, volume_info=np.ascontiguousarray(vi[:Li].T),
                compute_info=np.ascontiguousarray(ci[:Li].T), steps=a.steps, windows=a.windows,
                loop_ms=a.loop_ms, threads=a.threads, blocks=a.blocks, particle_steps=a.particle_steps,
                h2d_bytes=a.h2d_bytes, d2h_bytes=a.d2h_bytes)


class RefOptArgs(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("integrator", ctypes.c_int32), ("border_mode", ctypes.c_int32),
        ("curvature_mode", ctypes.c_int32), ("abort_mode", ctypes.c_int32), ("uplift_mode", ctypes.c_int32),
        ("windfield_mode", ctypes.c_int32), ("constants_mode", ctypes.c_int32), ("volume_mode", ctypes.c_int32),
        ("use_topography", ctypes.c_int32), ("reverse", ctypes.c_int32), ("use_sphere", ctypes.c_int32),
        ("comp_additional", ctypes.c_int32), ("blocks_fixed", ctypes.c_int32),
        ("delta_t", ctypes.c_float), ("data_time_distance", ctypes.c_float),
        ("maximum_simulation_time", ctypes.c_float), ("maximum_length", ctypes.c_float),
        ("sphere_radius", ctypes.c_float), ("save_interval", ctypes.c_int64),
        ("scale", ctypes.c_float * 3), ("offset", ctypes.c_float * 3),
        ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
        ("n_snapshots", ctypes.c_int32), ("wind", ctypes.POINTER(_FP)),
        ("n_volumes", ctypes.c_int32), ("volumes", ctypes.POINTER(_FP)),
        ("n_constants", ctypes.c_int32), ("constants", ctypes.POINTER(_FP)),
        ("uplift", ctypes.POINTER(_FP)), ("topography", _FP),
        ("ast", ctypes.POINTER(ASTANode)), ("ast_len", ctypes.c_int32),
        ("n", ctypes.c_int64), ("seeds", _FP),
        ("max_records", ctypes.c_int64), ("positions", _FP), ("status", ctypes.POINTER(ctypes.c_int32)),
        ("total_curvature", _FP), ("lengths", _FP), ("curvature", _FP), ("volume_info", _FP),
        ("compute_info", _FP),
        ("records", ctypes.c_int64), ("curvature_records", ctypes.c_int64), ("info_records", ctypes.c_int64),
        ("steps", ctypes.c_int64), ("windows", ctypes.c_int64), ("message", ctypes.c_char * 256),
    ]


def run_options(settings: dict, wind, seeds, volumes=None, constants=None, uplift=None, topography=None,
                blocks_fixed=True):
    """The reference's kernel for an option combination of oracle/ref_harness's OPT_VARIANTS
    (settings: reference IntegratorSettings field names, int enums).  volumes: [{name: plane}]
    (one constant volume at most); constants: [{name: (n,)}] per snapshot; uplift: [(n, 3)] per
    snapshot; topography: (ny, nx).  Returns the oracle's result layout."""
    lib = ctypes.CDLL(LIB_PATH)
    lib.ref_run_opt.argtypes = [ctypes.POINTER(RefOptArgs)]
    lib.ref_run_opt.restype = ctypes.c_int
    dim = 3 if settings.get("Space", 0) == 0 else 2
    a = RefOptArgs()
    a.dim = dim
    a.integrator = settings.get("Integrator", 1)
    a.border_mode = settings.get("BorderMode", 0) if dim == 2 else 0
    a.curvature_mode = settings.get("CurvatureMode", 0)
    a.abort_mode = settings.get("AbortMode", 0)
    a.uplift_mode = settings.get("UpLiftMode", 0) if dim == 3 else 0
    a.windfield_mode = settings.get("WindfieldMode", 1)
    a.constants_mode = settings.get("ConstantsMode", 0)
    a.volume_mode = settings.get("AdditionalVolumeMode", 0)
    a.use_topography = int(topography is not None and dim == 3)
    a.reverse = int(bool(settings.get("Reverse", False)))
    a.use_sphere = int(dim == 2 and settings.get("SphereRadius", 0.0) > 0)
    exprs = settings.get("AdditionalCompute", [])
    a.comp_additional = int(bool(exprs))
    a.blocks_fixed = int(blocks_fixed)
    a.delta_t = settings["DeltaT"]
    a.data_time_distance = settings["DataTimeDistance"]
    a.maximum_simulation_time = settings["MaximumSimulationTime"]
    a.maximum_length = settings.get("MaximumLength", 0.0)
    a.sphere_radius = settings.get("SphereRadius", 0.0)
    a.save_interval = settings["SaveInterval"]
    gs = list(settings["GridScale"]) + [settings["GridScale"][0]] * (3 - len(settings["GridScale"]))
    of = list(settings["Offset"]) + [settings["Offset"][0]] * (3 - len(settings["Offset"]))
    for d in range(3):
        a.scale[d] = gs[d]
        a.offset[d] = of[d]
    keep = []

    def ptrs(arrs):
        arrs = [np.ascontiguousarray(x, np.float32) for x in arrs]
        arr = (_FP * max(1, len(arrs)))(*[x.ctypes.data_as(_FP) for x in arrs])
        keep.extend([arrs, arr])
        return ctypes.cast(arr, ctypes.POINTER(_FP))

    a.wind = ptrs([p for snap in wind for p in snap[:dim]])
    shp = np.asarray(wind[0][0]).shape
    if dim == 3:
        a.nz, a.ny, a.nx = shp
    else:
        a.nz, (a.ny, a.nx) = 1, shp
    a.n_snapshots = len(wind)
    vol_names = list(volumes[0].keys())[:1] if (volumes and a.volume_mode) else []
    a.n_volumes = len(vol_names)
    if vol_names:
        a.volumes = ptrs([volumes[0][vol_names[0]]])
    con_names = list(constants[0].keys())[:4] if (constants and a.constants_mode) else []
    a.n_constants = len(con_names)
    if con_names:
        a.constants = ptrs([c[k] for c in constants for k in con_names])
    if uplift and a.uplift_mode:
        a.uplift = ptrs([u.reshape(-1) for u in uplift])
    if a.use_topography:
        t = np.ascontiguousarray(topography, np.float32)
        keep.append(t)
        a.topography = t.ctypes.data_as(_FP)
    if exprs:
        flat = expr_oracle.compile_expression(exprs[0], vol_names, con_names, dim, a.curvature_mode)
        nodes = (ASTANode * len(flat))(*[ASTANode(int(r["type"]), float(r["value"]), int(r["left"]),
                                                  int(r["right"])) for r in flat])
        keep.append(nodes)
        a.ast = ctypes.cast(nodes, ctypes.POINTER(ASTANode))
        a.ast_len = len(flat)
    sd = np.ascontiguousarray(seeds, np.float32)
    n = sd.shape[0]
    a.n = n
    a.seeds = sd.ctypes.data_as(_FP)
    steps_max = int(a.maximum_simulation_time / a.delta_t) + 2
    si = int(a.save_interval)
    max_rec = (1 + steps_max // si + 1) if si > 0 else 2
    pos = np.zeros((max_rec, n, dim), np.float32)
    st = np.zeros(n, np.int32)
    tc = np.zeros(n, np.float32)
    ln = np.zeros(n, np.float32)
    cv = np.zeros((max_rec, n), np.float32)
    vi = np.zeros((max_rec, n), np.float32)
    ci = np.zeros((max_rec, n), np.float32)
    a.max_records = max_rec
    a.positions = pos.ctypes.data_as(_FP)
    a.status = st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    a.total_curvature = tc.ctypes.data_as(_FP)
    a.lengths = ln.ctypes.data_as(_FP)
    a.curvature = cv.ctypes.data_as(_FP)
    a.volume_info = vi.ctypes.data_as(_FP)
    a.compute_info = ci.ctypes.data_as(_FP)
    rc = lib.ref_run_opt(ctypes.byref(a))
    if rc != 0:
        raise RuntimeError("reference harness: " + a.message.decode())
    L, Lc, Li = a.records, a.curvature_records, a.info_records
    return dict(trajectories=np.ascontiguousarray(pos[:L].transpose(1, 0, 2)), status=st,
                total_curvature=tc, lengths=ln, curvatures=np.ascontiguousarray(cv[:Lc].T),
                volume_info={k: np.ascontiguousarray(vi[:Li].T) for k in vol_names},
                compute_info=[np.ascontiguousarray(ci[:Li].T)] if exprs else [],
                steps=a.steps, windows=a.windows)
