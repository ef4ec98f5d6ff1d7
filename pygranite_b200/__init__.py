"""B200-native drop-in for pygranite's trajectory step path.

`import pygranite_b200 as pygranite` exposes the reference's module surface
(Space, Integrator, BorderMode, CurvatureMode, AbortMode, UpLiftMode, WindfieldMode,
ConstantsMode, AdditionalVolumeMode, AbortReason, IntegratorSettings, DataLoader,
TrajectorySet, TrajectoryIntegrator; source/pygranite.cpp:41-152).  The classes live in
the compiled extension `_pygranite`, which drives libgranite_b200.so (sm_100a kernels behind
the C ABI in include/granite_b200.h).  There is no CPU fallback: importing fails if the
extension has not been built (`python -c "import __graft_entry__ as g; g.build()"`).
"""
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIBRARY_PATH = _os.path.join(_HERE, "libgranite_b200.so")

try:
    from . import _pygranite as _ext
except ImportError as exc:  # pragma: no cover - exercised only on an unbuilt tree
    raise ImportError(
        "pygranite_b200: the compiled extension is missing; build it with "
        "`make -C pygranite_b200/csrc` (sm_100a, nvcc)") from exc

from ._pygranite import *  # noqa: F401,F403  (enums, export_values names and classes)
from ._pygranite import (AbortMode, AbortReason, AdditionalVolumeMode, BorderMode,  # noqa: F401
                         ConstantsMode, CurvatureMode, DataLoader, IntegratorSettings, Integrator,
                         Space, TrajectoryIntegrator, TrajectorySet, UpLiftMode, WindfieldMode,
                         WindStorage)

__all__ = [n for n in dir(_ext) if not n.startswith("_")]
