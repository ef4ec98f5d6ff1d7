"""Writes the golden fixtures of tests/golden/ from the reference's own CUDA kernel.

Run on a machine with a B200 after `make -C oracle/ref_harness` (which needs the reference
sources) has produced oracle/_ref/libref_integrate.so:

    python tests/golden/make_golden.py [out_dir]

The inputs are regenerated from seeds by pygranite_b200.workloads, so the fixtures hold only
the reference's outputs: positions every 10 steps, abort codes and, for the 3D case, total
curvature, the temperature samples and the expression values; and, in filter_reference.npz,
one Euler step through a field equal to its own grid coordinates (2D and 3D), which exposes
the texture filter's interpolation weights.  The reference filters through
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
    print("fixtures written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
