"""B200-native drop-in for pygranite's trajectory step path.

`import pygranite_b200 as pygranite` exposes the reference's module surface
(Space, Integrator, BorderMode, CurvatureMode, AbortMode, UpLiftMode, WindfieldMode,
ConstantsMode, AdditionalVolumeMode, AbortReason, IntegratorSettings, DataLoader,
TrajectorySet, TrajectoryIntegrator; source/pygranite.cpp:41-152).  The classes live in
the compiled extension `_pygranite`, which drives libgranite_b200.so (sm_100a kernels behind
the C ABI in include/granite_b200.h).  The extension is loaded on the first use of any of
those names, so the pure-Python submodules (`workloads`) import without it.  There is no CPU
fallback: that first use raises ImportError if the extension has not been built
(`python -c "import __graft_entry__ as g; g.build()"`).
"""
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIBRARY_PATH = _os.path.join(_HERE, "libgranite_b200.so")

_ext = None


def _load():
    global _ext
    if _ext is None:
        try:
            from . import _pygranite
        except ImportError as exc:  # pragma: no cover - exercised only on an unbuilt tree
            raise ImportError(
                "pygranite_b200: the compiled extension is missing; build it with "
                "`make -C pygranite_b200/csrc` (sm_100a, nvcc)") from exc
        _ext = _pygranite
    return _ext


def __getattr__(name):
    # enums, their export_values names and the classes of the extension
    if name == "__all__":
        return [n for n in dir(_load()) if not n.startswith("_")]
    if name.startswith("_") or _os.path.exists(_os.path.join(_HERE, name + ".py")):
        # private names, and the import system's lookup of a submodule not yet imported
        raise AttributeError(name)
    ext = _load()
    try:
        return getattr(ext, name)
    except AttributeError:
        raise AttributeError(f"module 'pygranite_b200' has no attribute '{name}'") from None


def __dir__():
    return sorted(set(globals()) | set(__getattr__("__all__")))
