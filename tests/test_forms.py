"""BatchIntegrator and TrajectoryServer (pygranite_b200.forms): the forms driven by pygranite's
own IntegratorSettings, DataLoader and TrajectorySet.  A set in a batch must end exactly where
TrajectoryIntegrator ends it alone with MaximumSimulationTime = lifetime * DeltaT; a served
request starting on a window boundary must match the same plain run.  Compared bit for bit."""
import numpy as np
import pytest

import pygranite_b200 as pg
from pygranite_b200 import forms
from pygranite_b200 import workloads as W
from tests import harness as H


def test_settings_conversion_keeps_every_field():
    s = pg.IntegratorSettings()
    s.Space, s.Integrator, s.BorderMode = pg.Space.Space2D, pg.Integrator.ExplicitEuler, pg.BorderMode.LoopXY
    s.DeltaT, s.DataTimeDistance, s.MaximumSimulationTime, s.SaveInterval = 0.5, 4.0, 16.0, 3
    s.GridScale, s.Offset = [2.0, 3.0], [-1.0, 5.0]
    s.CurvatureMode, s.MinimumAliveParticles, s.Reverse = pg.CurvatureMode.FastTotalCurvature, 17, True
    s.WindStorage, s.Float64Time, s.SortInterval, s.WindLayout = pg.WindStorage.Float16, True, 2, 1
    s.ReferenceFilter = True
    c = forms.c_settings(s)
    assert c.filter_weights == 1
    assert (c.space, c.integrator, c.border_mode, c.curvature_mode) == (1, 0, 3, 2)
    assert (c.delta_t, c.data_time_distance, c.maximum_simulation_time, c.save_interval) == (0.5, 4.0, 16.0, 3)
    assert list(c.grid_scale)[:2] == [2.0, 3.0] and c.grid_scale_len == 2 and list(c.offset)[:2] == [-1.0, 5.0]
    assert (c.minimum_alive, c.reverse, c.storage, c.time_mode, c.sort_interval, c.layout) == (17, 1, 2, 1, 2, 1)


def test_seed_points_from_a_trajectory_set():
    pts = np.random.default_rng(0).random((7, 3)).astype(np.float32)
    assert np.array_equal(forms._points(pg.TrajectorySet(pts)), pts)
    assert np.array_equal(forms._points(pts), pts)


def small_problem(**over):
    settings, src, seeds = W.config2(n_particles=900, n_snapshots=12, grid=(16, 24, 24), steps=100)
    settings = dict(settings, SaveInterval=0, **over)
    return settings, src, seeds


@pytest.mark.gpu
def test_batch_integrator_matches_trajectory_integrator_per_set():
    settings, src, seeds = small_problem()
    sets, lives = [seeds[:300], seeds[300:350], seeds[350:]], [100, 37, 64]
    s = W.apply_settings(pg.IntegratorSettings(), settings, H.enums(pg))
    b = forms.BatchIntegrator(s, W.make_loader(pg.DataLoader, src), [pg.TrajectorySet(x) for x in sets], lives)
    out = b.compute()
    again = b.compute()   # a replay of the captured graph
    for j, (x, L) in enumerate(zip(sets, lives)):
        ref = H.run_engine(dict(settings, MaximumSimulationTime=60.0 * L), src.wind, x, volumes=src.volumes)
        r = out[j]
        assert np.array_equal(r.abortReasons(), ref["status"]), j
        assert np.array_equal(r.finalPositions(), ref["trajectories"][:, -1]), j
        assert np.array_equal(r.totalCurvatures(), ref["total_curvature"]), j
        assert np.array_equal(r.volumeInfo("T")[:, -1], ref["volume_info"]["T"][:, -1]), j
        assert np.array_equal(r.computeInfo(0)[:, -1], ref["compute_info"][0][:, -1]), j
        assert np.array_equal(again[j].finalPositions(), r.finalPositions())
    b.close()


@pytest.mark.gpu
def test_trajectory_server_matches_a_plain_run():
    settings, src, seeds = small_problem(CurvatureMode=0, AdditionalVolumeMode=0, AdditionalCompute=[])
    s = W.apply_settings(pg.IntegratorSettings(), settings, H.enums(pg))
    srv = forms.TrajectoryServer(s, W.make_loader(pg.DataLoader, src))
    rid = srv.submit(pg.TrajectorySet(seeds), 0.0, 45)
    assert srv.wait(rid, 60.0) == 2
    pos, st = srv.result(rid)
    srv.close()
    ref = H.run_engine(dict(settings, MaximumSimulationTime=60.0 * 45), src.wind, seeds)
    assert np.array_equal(st, ref["status"])
    assert np.array_equal(pos, ref["trajectories"][:, -1])


@pytest.mark.gpu
def test_batch_integrator_with_compensation_and_fast_curvature():
    settings, src, seeds = small_problem(CurvatureMode=2)
    sets, lives = [seeds[:400], seeds[400:]], [80, 23]
    s = W.apply_settings(pg.IntegratorSettings(), settings, H.enums(pg))
    s.CompensatedPositions = True
    s.WindStorage = pg.WindStorage.Float16
    b = forms.BatchIntegrator(s, W.make_loader(pg.DataLoader, src), sets, lives)
    out = b.compute()
    for j, (x, L) in enumerate(zip(sets, lives)):
        ref = H.run_engine(dict(settings, MaximumSimulationTime=60.0 * L), src.wind, x, volumes=src.volumes,
                           CompensatedPositions=True, WindStorage=pg.WindStorage.Float16)
        assert np.array_equal(out[j].abortReasons(), ref["status"]), j
        assert np.array_equal(out[j].finalPositions(), ref["trajectories"][:, -1]), j
        assert np.array_equal(out[j].totalCurvatures(), ref["total_curvature"]), j
    b.close()
