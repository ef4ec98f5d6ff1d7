"""The pygranite surface of pygranite_b200 (no GPU): names, enum values, defaults,
TrajectorySet construction and accessors (source/pygranite.cpp:41-152,
IntegratorSettings.hpp:16-181, TrajectorySet.cpp)."""
import numpy as np
import pytest

import pygranite_b200 as pg


def test_enum_values():
    assert int(pg.Space.Space3D) == 0 and int(pg.Space.Space2D) == 1
    assert int(pg.Integrator.ExplicitEuler) == 0 and int(pg.Integrator.ClassicRungeKutta) == 1
    assert [int(getattr(pg.BorderMode, n)) for n in ("Block", "LoopX", "LoopY", "LoopXY")] == [0, 1, 2, 3]
    assert [int(getattr(pg.CurvatureMode, n)) for n in
            ("Off", "TotalCurvature", "FastTotalCurvature", "IndividualAndTotalCurvature")] == [0, 1, 2, 3]
    assert [int(getattr(pg.AbortMode, n)) for n in ("Time", "Length", "FitLength")] == [0, 1, 2]
    for E in (pg.UpLiftMode, pg.ConstantsMode, pg.AdditionalVolumeMode):
        assert [int(getattr(E, n)) for n in ("Off", "Constant", "Dynamic")] == [0, 1, 2]
    assert int(pg.WindfieldMode.Constant) == 0 and int(pg.WindfieldMode.Dynamic) == 1
    assert [int(getattr(pg.AbortReason, n)) for n in ("Time", "Length", "Domain", "Topography", "Wind")] == [0, 1, 2, 3, 4]


def test_export_values_collisions_follow_registration_order():
    # every enum calls export_values(); the last registration of a name wins (pygranite.cpp:41-100)
    assert pg.Time == pg.AbortMode.Time
    assert pg.Length == pg.AbortMode.Length
    assert pg.Off == pg.ConstantsMode.Off
    assert pg.Constant == pg.ConstantsMode.Constant
    assert pg.Dynamic == pg.ConstantsMode.Dynamic
    assert pg.Domain == pg.AbortReason.Domain and pg.Block == pg.BorderMode.Block


def test_settings_defaults_and_fields():
    s = pg.IntegratorSettings()
    assert s.SphereRadius == 0.0 and s.Space == pg.Space.Space3D and s.Integrator == pg.Integrator.ClassicRungeKutta
    assert s.WindfieldMode == pg.WindfieldMode.Dynamic and s.ConstantsMode == pg.ConstantsMode.Off
    assert s.AdditionalVolumeMode == pg.AdditionalVolumeMode.Off and s.UpLiftMode == pg.UpLiftMode.Off
    assert s.DeltaT == 1.0 and s.DataTimeDistance == 60.0
    assert s.GridScale == [25.0, 25.0, 25.0] and s.Offset == [0.0, 0.0, 0.0]
    assert s.SaveInterval == 1 and s.Reverse is False and s.BorderMode == pg.BorderMode.Block
    assert s.CurvatureMode == pg.CurvatureMode.Off and s.MaximumLength == 0.0
    assert s.MaximumSimulationTime == 100.0 and s.AbortMode == pg.AbortMode.Time
    assert s.MinimumAliveParticles == 0 and s.Topography.shape == (0,) and s.AdditionalCompute == []
    s.GridScale = [1.0, 2.0]
    s.AdditionalCompute = ["x+y"]
    s.Topography = np.ones((3, 4), np.float32)
    assert s.GridScale == [1.0, 2.0] and s.AdditionalCompute == ["x+y"] and s.Topography.shape == (3, 4)


def test_trajectory_set_accessors():
    pts = np.arange(15, dtype=np.float32).reshape(5, 3)
    ts = pg.TrajectorySet(pts)
    assert ts.numberTrajectories() == 5 and ts.lengthTrajectories() == 1
    assert ts.trajectories().shape == (5, 1, 3) and np.array_equal(ts.trajectories()[:, 0], pts)
    assert np.array_equal(ts.trajectory(2), pts[2:3])
    assert np.array_equal(ts.cloud(), pts)
    assert ts.totalCurvatures().shape == (0,) and ts.individualLengths().shape == (0,)
    assert ts.curvatures().shape == (5, 0) and ts.abortReasons() == []
    with pytest.raises(RuntimeError, match="Volume with given key 'T' does not exist"):
        ts.volumeInfo("T")
    with pytest.raises(RuntimeError, match="Volume with given id does not exist"):
        ts.computeInfo(0)
    ts2 = pg.TrajectorySet(np.zeros((4, 2), np.float64))   # converted to float32
    assert ts2.trajectories().dtype == np.float32 and ts2.trajectories().shape == (4, 1, 2)


def test_trajectory_set_rejects_bad_shapes():
    with pytest.raises(RuntimeError, match="Currently only 1 dimensional initial pointsets are supported"):
        pg.TrajectorySet(np.zeros(6, np.float32))
    with pytest.raises(RuntimeError, match="does not support the given type of coordinates"):
        pg.TrajectorySet(np.zeros((3, 4), np.float32))


def test_data_loader_is_subclassable():
    class L(pg.DataLoader):
        def __init__(self):
            pg.DataLoader.__init__(self)

        def step(self):
            return False

        def windfield(self):
            return [np.zeros((2, 2), np.float32)] * 2

    ld = L()
    assert ld.step() is False and len(ld.windfield()) == 2
    assert ld.constants() == {} and ld.additionalVolumes() == {}
