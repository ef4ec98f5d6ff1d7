"""The benchmark configuration at its full size, shortened in time (GPU).

The plain 3D RK4 configuration at the size the benchmark times: 192 x 192 x 64 Fourier field,
1,000,000 particles in the lower half of the domain, TotalCurvature, the temperature volume and
sqrt(u*u+v*v)*T, records every 10 steps, compaction and Morton re-sort every 4 launches, the
window-pair layout, every snapshot resident in the ring (int32 node indices over the whole
grid).  200 steps instead of 2,000.  A fixed sample of particle ids spread over the seed array
is compared bit for bit with the float32 oracle: every record of the positions, the abort
codes, the total curvature, the temperature samples and the expression values; the same run
through the pygranite API (3-slot ring fed by the Python loader) is checked the same way.
"""
import numpy as np
import pytest

from pygranite_b200 import capi
from pygranite_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 200
SAMPLE = 2000


def sample_ids(n, m):
    return np.unique(np.linspace(0, n - 1, m).round().astype(np.int64))


@pytest.fixture(scope="module")
def case():
    from oracle import oracle as orc
    settings, src, seeds = W.config2(n_particles=1_000_000, n_snapshots=STEPS // 10 + 1, steps=STEPS)
    ids = sample_ids(seeds.shape[0], SAMPLE)
    ref = orc.run(orc.settings(**settings), orc.Inputs(wind=src.wind, seeds=seeds[ids], volumes=src.volumes),
                  precision="f32")
    return settings, src, seeds, ids, ref


def compare(got, ref):
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["trajectories"], ref["trajectories"])
    assert np.array_equal(got["total_curvature"], ref["total_curvature"])
    assert np.array_equal(got["volume"], ref["volume_info"]["T"])
    assert np.array_equal(got["expression"], ref["compute_info"][0])


def test_full_size_engine_run_matches_the_float32_oracle(case):
    settings, src, seeds, ids, ref = case
    n_snap = len(src.wind)
    eng = capi.Engine(capi.settings_from_reference(settings, ring_slots=n_snap, sort_interval=4))
    eng.set_seeds(seeds)
    for k, snap in enumerate(src.wind):
        eng.load_windfield(k, snap)
    eng.load_volume(0, 0, src.volumes[0]["T"])
    eng.compile_expression(0, settings["AdditionalCompute"][0], ["T"], [])
    eng.run(lambda k: 1 if k < n_snap else 0)
    res = eng.results(pinned=True)
    info = eng.info()
    assert info.records == STEPS // 10 + 1 and info.steps == STEPS
    got = {"trajectories": np.array(res["trajectories"][ids]), "status": res["status"][ids],
           "total_curvature": res["total_curvature"][ids], "volume": np.array(res["volume_info"][0][ids]),
           "expression": np.array(res["compute_info"][0][ids])}
    del res
    eng.close()
    compare(got, ref)


def test_full_size_api_run_matches_the_float32_oracle(case):
    import pygranite_b200 as pg
    settings, src, seeds, ids, ref = case
    enums = dict(Space=pg.Space, Integrator=pg.Integrator, WindfieldMode=pg.WindfieldMode,
                 AdditionalVolumeMode=pg.AdditionalVolumeMode, BorderMode=pg.BorderMode,
                 CurvatureMode=pg.CurvatureMode)
    s = W.apply_settings(pg.IntegratorSettings(), settings, enums)
    res = pg.TrajectoryIntegrator(s, W.make_loader(pg.DataLoader, src), pg.TrajectorySet(seeds)).compute()
    got = {"trajectories": res.trajectories()[ids],
           "status": np.array([int(r) for r in res.abortReasons()], np.int32)[ids],
           "total_curvature": np.asarray(res.totalCurvatures())[ids], "volume": res.volumeInfo("T")[ids],
           "expression": res.computeInfo(0)[ids]}
    assert res.particleSteps() > 0
    compare(got, ref)
