"""Shared helpers: run the same settings through the engine and through the oracle."""
import numpy as np

from oracle import oracle as orc


def enums(pg):
    return dict(Space=pg.Space, Integrator=pg.Integrator, WindfieldMode=pg.WindfieldMode,
                ConstantsMode=pg.ConstantsMode, AdditionalVolumeMode=pg.AdditionalVolumeMode,
                UpLiftMode=pg.UpLiftMode, BorderMode=pg.BorderMode, CurvatureMode=pg.CurvatureMode,
                AbortMode=pg.AbortMode)


def run_engine(settings: dict, wind, seeds, volumes=None, constants=None, uplift=None, topography=None,
               **extra):
    """Runs through the pygranite surface; returns the oracle's result layout."""
    import pygranite_b200 as pg
    from pygranite_b200 import workloads as W

    s = W.apply_settings(pg.IntegratorSettings(), settings, enums(pg))
    for k, v in extra.items():
        setattr(s, k, v)
    if topography is not None:
        s.Topography = np.ascontiguousarray(topography, np.float32)
    src = W.SnapshotSource(wind, volumes=volumes, constants=constants, uplift=uplift)
    loader = W.make_loader(pg.DataLoader, src)
    res = pg.TrajectoryIntegrator(s, loader, pg.TrajectorySet(seeds)).compute()
    out = dict(trajectories=res.trajectories(), status=np.array([int(a) for a in res.abortReasons()], np.int32),
               lengths=res.individualLengths(), total_curvature=res.totalCurvatures(),
               curvatures=res.curvatures(), loader_calls=loader.calls)
    vol_names = list(volumes[0].keys())[:8] if volumes and settings.get("AdditionalVolumeMode", 0) else []
    out["volume_info"] = {k: res.volumeInfo(k) for k in vol_names}
    out["compute_info"] = [res.computeInfo(i) for i in range(len(settings.get("AdditionalCompute", [])))]
    return out


def run_oracle(settings: dict, wind, seeds, volumes=None, constants=None, uplift=None, topography=None,
               precision="f64", time_mode=0, compensated=False):
    data = orc.Inputs(wind=wind, seeds=seeds, volumes=volumes or [], constants=constants or [],
                      uplift=uplift or [], topography=topography)
    return orc.run(orc.settings(**settings), data, precision=precision, time_mode=time_mode, compensated=compensated)


def cell_error(a, b, cell):
    """|a - b| in grid cells, per record and particle (max over components)."""
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.asarray(cell, np.float64)
    return d.max(axis=-1)


def assert_same(eng, ref, keys=("trajectories", "status")):
    for k in keys:
        a, b = np.asarray(eng[k]), np.asarray(ref[k])
        assert a.shape == b.shape, (k, a.shape, b.shape)
        if a.dtype.kind == "f":
            bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
        else:
            bad = a != b
        assert not bad.any(), f"{k}: {int(bad.sum())} of {a.size} values differ; first at {np.argwhere(bad)[:3].tolist()}"
