"""Writes the golden fixtures of tests/golden/ from the reference's own CUDA kernel.

Run on a machine with a B200 after `make -C oracle/ref_harness` (which needs the reference
sources) has produced oracle/_ref/libref_integrate.so:

    python tests/golden/make_golden.py [out_dir]

The inputs are regenerated from seeds by pygranite_b200.workloads, so the fixtures hold only
the reference's outputs: positions every 10 steps, abort codes and, for the 3D case, total
curvature, the temperature samples and the expression values; and, in filter_reference.npz,
one Euler step through a field equal to its own grid coordinates (2D and 3D), which exposes
the texture filter's interpolation weights; in options_reference.npz, the option combinations
of OPTION_CASES (loop borders, sphere coordinates, FastTotal / Individual curvature, length and
fit-length aborts, uplift, topography, constants, constant wind, reverse).  The reference filters through
texture hardware with 8-bit interpolation weights, so its outputs are matched within a
tolerance, not bit for bit.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.ref_harness import refrun  # noqa: E402
from pygranite_b200 import workloads as W  # noqa: E402

GYRE = dict(n=256, save_interval=10)
FOURIER = dict(n=512, n_snapshots=6, grid=(16, 24, 24), steps=50)


def gyre_case():
    settings, src, seeds = W.config1(n_particles=GYRE["n"])
    settings["SaveInterval"] = GYRE["save_interval"]
    return settings, src, seeds


def fourier_case():
    settings, src, seeds = W.config2(n_particles=FOURIER["n"], n_snapshots=FOURIER["n_snapshots"],
                                     grid=FOURIER["grid"], steps=FOURIER["steps"])
    return settings, src, seeds


def filter_case(dim, n=12288):
    """One Euler step (h = 1/16 s, exact in float32) through a field whose value is its own grid
    coordinate (u = x index, v = y index, w = z index), the same in two snapshots: the new
    position minus the old, times 16, is exactly what the texture filter returned at the old
    one.  Seeds cover the fractional coordinates densely in [1, 6) on every axis, below 8 so
    that p + h v is exact in float32."""
    shape = (8, 12, 16) if dim == 3 else (12, 16)
    grids = np.meshgrid(*[np.arange(k, dtype=np.float32) for k in shape], indexing="ij")
    comps = [grids[-1], grids[-2]] + ([grids[0]] if dim == 3 else [])      # u = x, v = y, w = z
    wind = [[c.copy() for c in comps] for _ in range(2)]
    k = np.arange(n, dtype=np.float64)
    fr = [(k + 0.5) / n, np.mod(k * 0.6180339887498949, 1.0), np.mod(k * 0.4142135623730951, 1.0)]
    seeds = np.stack([1.0 + 5.0 * fr[d] for d in range(dim)], axis=1).astype(np.float32)
    settings = dict(Space=0 if dim == 3 else 1, Integrator=0, WindfieldMode=1, DeltaT=0.0625,
                    DataTimeDistance=1.0, GridScale=[1.0] * dim, Offset=[0.0] * dim, SaveInterval=1,
                    BorderMode=0, CurvatureMode=0, MaximumSimulationTime=0.0625)
    return settings, W.SnapshotSource(wind), seeds


# ------------------------------------------------------------ the option matrix
# Option combinations of the reference's kernel beyond the two benchmark configurations, each
# instantiated unmodified by oracle/ref_harness (OPT_VARIANTS).  2D: a 32 x 24 Fourier field (1 km)
# or a 36 x 18 field in degrees for sphere coordinates; 3D: a 24 x 20 x 12 field (1 km, 250 m).
OPTION_CASES = {
    "2d_loopx_euler": dict(Integrator=0, BorderMode=1),
    "2d_loopy_rk4": dict(BorderMode=2),
    "2d_loopxy_rk4": dict(BorderMode=3),
    "2d_loopxy_sphere": dict(BorderMode=3, SphereRadius=6.371e6),
    "2d_loopy_sphere_euler": dict(Integrator=0, BorderMode=2, SphereRadius=6.371e6),
    "2d_fasttotal_reverse": dict(CurvatureMode=2, Reverse=True),
    "2d_windfield_constant": dict(WindfieldMode=0),
    "2d_loopx_fasttotal_sphere": dict(BorderMode=1, CurvatureMode=2, SphereRadius=6.371e6),
    "3d_individual_length": dict(CurvatureMode=3, AbortMode=1, MaximumLength=15000.0),
    "3d_fitlength_uplift_constant_euler": dict(Integrator=0, AbortMode=2, MaximumLength=15000.0, UpLiftMode=1),
    "3d_uplift_dynamic_topography": dict(UpLiftMode=2, topography=True),
    "3d_constants_volume_expression": dict(CurvatureMode=1, ConstantsMode=1, AdditionalVolumeMode=1,
                                           AdditionalCompute=["T*ka + kb - z/1000"]),
    "3d_constants_dynamic_reverse": dict(ConstantsMode=2, Reverse=True, AdditionalCompute=["ka*u + kb*v"]),
    "3d_constant_wind_length_reverse_euler": dict(Integrator=0, CurvatureMode=1, AbortMode=1,
                                                  MaximumLength=12000.0, WindfieldMode=0, Reverse=True),
}
OPTION_N = 400


def option_case(name):
    """Settings and inputs of an option-matrix case, regenerated from seeds: (settings, wind,
    seeds, volumes, constants, uplift, topography)."""
    opts = dict(OPTION_CASES[name])
    topo = opts.pop("topography", False)
    dim = 2 if name.startswith("2d") else 3
    seed = sum(map(ord, name)) % 1000
    n_snap = 8
    rng = np.random.default_rng(seed)
    volumes = constants = uplift = topography = None
    if dim == 2:
        sphere = opts.get("SphereRadius", 0.0) > 0
        shape = (18, 36) if sphere else (24, 32)
        field = W.FourierField(shape, (1000.0, 1000.0), n_modes=16, seed=seed, rms=(7.0710678, 7.0710678))
        base = dict(Space=1, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=[1000.0, 1000.0], Offset=[0.0, 0.0], SaveInterval=5, BorderMode=0, CurvatureMode=0,
                    MaximumSimulationTime=3600.0)
        lo, hi = [0.0, 0.0], [32000.0, 24000.0]
        if sphere:
            # degrees: 10-degree cells, latitude -90..90, 10-hour steps
            base.update(GridScale=[10.0, 10.0], Offset=[0.0, -90.0], DeltaT=36000.0, DataTimeDistance=360000.0,
                        MaximumSimulationTime=36000.0 * 60)
            lo, hi = [0.0, -85.0], [360.0, 85.0]
        wind = [field.snapshot(600.0 * k) for k in range(n_snap)]
    else:
        shape = (12, 20, 24)
        field = W.FourierField(shape, (250.0, 1000.0, 1000.0), n_modes=16, seed=seed)
        base = dict(Space=0, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=[1000.0, 1000.0, 250.0], Offset=[0.0, 0.0, 0.0], SaveInterval=5, BorderMode=0,
                    CurvatureMode=0, MaximumSimulationTime=3600.0)
        lo, hi = [0.0, 0.0, 0.0], [24000.0, 20000.0, 1500.0]
        wind = [field.snapshot(600.0 * k) for k in range(n_snap)]
    settings = dict(base, **opts)
    seeds = W.uniform_seeds(OPTION_N, seed + 1, lo, hi)
    if settings.get("AdditionalVolumeMode", 0):
        volumes = [{"T": W.temperature(shape, 250.0, seed=seed + 2)}]
    if settings.get("ConstantsMode", 0):
        constants = [{"ka": rng.uniform(0.5, 1.5, OPTION_N).astype(np.float32),
                      "kb": rng.uniform(-2.0, 2.0, OPTION_N).astype(np.float32)} for _ in range(n_snap)]
    if settings.get("UpLiftMode", 0):
        uplift = [(rng.standard_normal((OPTION_N, 3)) * np.array([40.0, 40.0, 15.0])).astype(np.float32)
                  for _ in range(n_snap)]
    if topo:
        topography = np.zeros(shape[1:], np.float32)
        topography[:, 16:] = 900.0          # a plateau in x >= 16 km, 900 m high
    return settings, wind, seeds, volumes, constants, uplift, topography


def main(out):
    os.makedirs(out, exist_ok=True)
    settings, src, seeds = gyre_case()
    r = refrun.run(settings, src.wind, seeds)
    np.savez_compressed(os.path.join(out, "gyre_reference.npz"), trajectories=r["trajectories"],
                        status=r["status"], steps=r["steps"], windows=r["windows"],
                        settings=json.dumps(settings))
    settings, src, seeds = fourier_case()
    r = refrun.run(settings, src.wind, seeds, volume=src.volumes[0]["T"])
    np.savez_compressed(os.path.join(out, "fourier_reference.npz"), trajectories=r["trajectories"],
                        status=r["status"], total_curvature=r["total_curvature"],
                        volume_info=r["volume_info"], compute_info=r["compute_info"], steps=r["steps"],
                        windows=r["windows"], settings=json.dumps(settings))
    arrays = {}
    for dim in (2, 3):
        settings, src, seeds = filter_case(dim)
        r = refrun.run(settings, src.wind, seeds)
        arrays[f"positions{dim}d"] = r["trajectories"][:, 1]     # record 0 is the seeds
        arrays[f"status{dim}d"] = r["status"]
    np.savez_compressed(os.path.join(out, "filter_reference.npz"), **arrays)
    options = {}
    for name in OPTION_CASES:
        settings, wind, seeds, volumes, constants, uplift, topography = option_case(name)
        r = refrun.run_options(settings, wind, seeds, volumes=volumes, constants=constants, uplift=uplift,
                               topography=topography)
        for k in ("trajectories", "status", "total_curvature", "lengths", "curvatures"):
            options[f"{name}/{k}"] = r[k]
        for k, v in r["volume_info"].items():
            options[f"{name}/volume_{k}"] = v
        if r["compute_info"]:
            options[f"{name}/compute_0"] = r["compute_info"][0]
        options[f"{name}/steps"] = np.int64(r["steps"])
    np.savez_compressed(os.path.join(out, "options_reference.npz"), **options)
    print("fixtures written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
