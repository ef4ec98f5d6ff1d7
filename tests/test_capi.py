"""The C ABI (no GPU): exports, host-only entry points, and the step bookkeeping.

gr_plan restates the reference's host loop (TrajectoryIntegrator.tpp:778-995); its per-step
windows, record flags and float32 time weights must equal the oracle's schedule exactly.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc
from pygranite_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:int|void|const char \*)\s*(gr_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol():
    declared = declared_functions()
    assert len(declared) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    missing = declared - exported
    assert not missing, missing
    assert declared == set(capi.EXPORTS), declared ^ set(capi.EXPORTS)
    lib = capi.lib()
    for name in declared:
        assert getattr(lib, name) is not None


def test_settings_defaults_match_reference():
    s = capi.default_settings()
    # IntegratorSettings.hpp:89-181
    assert (s.space, s.integrator, s.windfield_mode, s.constants_mode, s.volume_mode, s.uplift_mode) == (0, 1, 1, 0, 0, 0)
    assert (s.delta_t, s.data_time_distance, s.maximum_simulation_time) == (1.0, 60.0, 100.0)
    assert list(s.grid_scale) == [25.0, 25.0, 25.0] and s.grid_scale_len == 3
    assert list(s.offset) == [0.0, 0.0, 0.0] and s.save_interval == 1
    assert (s.border_mode, s.curvature_mode, s.abort_mode, s.minimum_alive, s.reverse) == (0, 0, 0, 0, 0)


def test_invalid_settings_are_rejected_without_gpu():
    for bad in (dict(delta_t=0.0), dict(data_time_distance=-1.0), dict(maximum_simulation_time=1e12, delta_t=1e-3)):
        with pytest.raises(capi.GraniteError, match="ERROR < USER INPUT"):
            capi.plan(capi.default_settings(**bad))
    # engine options are checked before any CUDA call
    L = capi.lib()
    for bad, msg in ((dict(storage=3), b"storage"), (dict(filter_weights=2), b"filter weights"),
                     (dict(filter_weights=-1), b"filter weights")):
        h = ctypes.c_void_p()
        assert L.gr_create(ctypes.byref(capi.default_settings(**bad)), ctypes.byref(h)) == -1
        assert msg in L.gr_last_error() and not h.value


PLANS = [
    dict(Space=1, DeltaT=0.01, DataTimeDistance=1.0, MaximumSimulationTime=10.0, SaveInterval=1),
    dict(Space=0, DeltaT=60.0, DataTimeDistance=600.0, MaximumSimulationTime=120000.0, SaveInterval=10),
    dict(Space=0, DeltaT=0.3, DataTimeDistance=1.0, MaximumSimulationTime=7.0, SaveInterval=3),
    dict(Space=0, DeltaT=2.5, DataTimeDistance=1.0, MaximumSimulationTime=20.0, SaveInterval=0),   # steps over windows
    dict(Space=1, DeltaT=0.1, DataTimeDistance=0.7, MaximumSimulationTime=5.0, SaveInterval=4, WindfieldMode=0),
    dict(Space=1, DeltaT=0.1, DataTimeDistance=0.7, MaximumSimulationTime=5.0, SaveInterval=2, WindfieldMode=0,
         AdditionalVolumeMode=2),
    dict(Space=0, DeltaT=1.0 / 3, DataTimeDistance=1.0, MaximumSimulationTime=9.0, SaveInterval=1, UpLiftMode=2),
    dict(Space=0, DeltaT=0.7, DataTimeDistance=60.0, MaximumSimulationTime=100.0, SaveInterval=7),
]


@pytest.mark.parametrize("k", range(len(PLANS)))
@pytest.mark.parametrize("time_mode", [0, 1])
def test_plan_matches_oracle_schedule(k, time_mode):
    st = PLANS[k]
    dim = 3 if st["Space"] == 0 else 2
    shape = (2, 4, 4) if dim == 3 else (4, 4)
    info, plan = capi.plan(capi.settings_from_reference(st, time_mode=time_mode))
    wind = [[np.zeros(shape, np.float32)] * dim] * (info.windows + 2)   # a loader that never runs dry
    steps, windows = orc.schedule(orc.settings(**st), orc.Inputs(wind=wind, seeds=np.zeros((1, dim), np.float32)),
                                  time_mode=time_mode)
    assert info.steps == len(steps) and info.windows == windows
    assert np.array_equal(plan["window"], [s["window"] for s in steps])
    assert np.array_equal(plan["flags"] & 1, [s["save"] for s in steps])
    assert np.array_equal((plan["flags"] >> 1) & 1, [s["time_pos"] for s in steps])
    w = np.array([[s["t0f"], s["t1f"], s["t2f"]] for s in steps], np.float32)
    assert np.array_equal(plan["weights"].view(np.uint32), w.view(np.uint32))
    saves = sum(s["save"] for s in steps)
    assert info.records == 1 + saves + (1 if st["SaveInterval"] == 0 else 0)
