"""Writes the golden fixtures of tests/golden/ from the reference's own CUDA kernel.

Run on a machine with a B200 after `make -C oracle/ref_harness` (which needs the reference
sources) has produced oracle/_ref/libref_integrate.so:

    python tests/golden/make_golden.py [out_dir]

The inputs are regenerated from seeds by pygranite_b200.workloads, so the fixtures hold only
the reference's outputs: positions every 10 steps, abort codes and, for the 3D case, total
curvature, the temperature samples and the expression values.  The reference filters through
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
    print("fixtures written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
