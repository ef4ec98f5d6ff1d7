"""Pins of the CPU oracle (no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned here by analytic
known answers (uniform wind, linear-in-time wind, solid-body rotation), by the texture
address modes the reference configures (3D border, 2D clamp), and by hand-built cases for
every abort reason and for the save / window bookkeeping of the reference's host loop
(TrajectoryIntegrator.tpp:778-995).
"""
import numpy as np
import pytest

from oracle import oracle as orc


def uniform(shape, n_snap, vals):
    return [[np.full(shape, v, np.float32) for v in vals] for _ in range(n_snap)]


def run(settings, wind, seeds, **kw):
    return orc.run(orc.settings(**settings), orc.Inputs(wind=wind, seeds=np.asarray(seeds, np.float32), **kw),
                   precision=kw.pop("precision", "f64") if "precision" in kw else "f64")


@pytest.mark.parametrize("integrator", [0, 1])
@pytest.mark.parametrize("dim", [2, 3])
def test_uniform_wind_is_exact(integrator, dim):
    shape = (8, 16) if dim == 2 else (6, 8, 16)
    vals = [1.0, 0.5] if dim == 2 else [1.0, 0.5, 0.25]
    st = dict(Space=1 if dim == 2 else 0, Integrator=integrator, DeltaT=0.25, DataTimeDistance=1.0,
              GridScale=[1.0] * dim, Offset=[0.0] * dim, MaximumSimulationTime=2.0, SaveInterval=1)
    seeds = [[1.0, 1.0, 1.0][:dim], [2.0, 3.0, 1.5][:dim]]
    for prec in ("f64", "f32"):
        r = orc.run(orc.settings(**st), orc.Inputs(wind=uniform(shape, 4, vals), seeds=np.array(seeds, np.float32)),
                    precision=prec)
        assert r["steps"] == 8
        assert np.array_equal(r["status"], [0, 0])
        expect = np.array(seeds, np.float64) + 2.0 * np.array(vals)
        assert np.allclose(r["trajectories"][:, -1], expect, atol=1e-6)
        # every record advances by v*h
        d = np.diff(r["trajectories"], axis=1)
        assert np.allclose(d, 0.25 * np.array(vals), atol=1e-6)


def test_linear_in_time_wind_rk4_exact():
    """u(t) = a + b t, piecewise-linear in time by construction: RK4 integrates it exactly."""
    a, b, dtd = 0.5, 0.25, 1.0
    wind = [[np.full((8, 64), a + b * k * dtd, np.float32), np.zeros((8, 64), np.float32)] for k in range(8)]
    st = dict(Space=1, Integrator=1, DeltaT=0.125, DataTimeDistance=dtd, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
              MaximumSimulationTime=4.0, SaveInterval=0)
    r = run(st, wind, [[1.0, 4.0]])
    T = 4.0
    assert np.isclose(r["trajectories"][0, -1, 0], 1.0 + a * T + b * T * T / 2, atol=1e-9)
    st["Integrator"] = 0
    r = run(st, wind, [[1.0, 4.0]])
    h, n = 0.125, 32
    euler = 1.0 + a * T + b * h * h * n * (n - 1) / 2
    assert np.isclose(r["trajectories"][0, -1, 0], euler, atol=1e-9)


def rotation_field(n=64, omega=0.1, c=32.0):
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    return [[(-omega * (y - c)).astype(np.float32), (omega * (x - c)).astype(np.float32)]]


@pytest.mark.parametrize("integrator,order", [(1, 4), (0, 1)])
def test_solid_body_rotation_convergence_order(integrator, order):
    """Bilinear interpolation of a linear field is exact, so the error is the integrator's."""
    wind = rotation_field(64, 0.5, 32.0)
    errs = []
    for h in ((1.0, 0.5, 0.25) if integrator == 1 else (0.05, 0.025, 0.0125)):
        st = dict(Space=1, Integrator=integrator, WindfieldMode=0, DeltaT=h, DataTimeDistance=1.0,
                  GridScale=[1.0, 1.0], Offset=[0.0, 0.0], MaximumSimulationTime=10.0, SaveInterval=0)
        r = run(st, wind, [[42.0, 32.0]])
        p = r["trajectories"][0, -1]
        ang = 0.5 * 10.0
        exact = np.array([32.0 + 10.0 * np.cos(ang), 32.0 + 10.0 * np.sin(ang)])
        errs.append(np.linalg.norm(p - exact))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(np.abs(rates - order) < 0.3), rates


def test_address_modes_border_3d_clamp_2d():
    # 3D: a particle between the last node and the domain end interpolates toward 0 (border)
    st = dict(Space=0, Integrator=0, WindfieldMode=0, DeltaT=1.0, GridScale=[1.0, 1.0, 1.0],
              Offset=[0.0, 0.0, 0.0], MaximumSimulationTime=1.0, SaveInterval=1)
    r = run(st, uniform((4, 4, 8), 1, [1.0, 0.0, 0.0]), [[7.25, 1.0, 1.0]])
    assert np.isclose(r["trajectories"][0, 1, 0], 7.25 + 0.75)
    # 2D: the same position samples the clamped last node
    st2 = dict(Space=1, Integrator=0, WindfieldMode=0, DeltaT=0.5, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
               MaximumSimulationTime=0.5, SaveInterval=1)
    r = run(st2, uniform((4, 8), 1, [1.0, 0.0]), [[7.25, 1.0]])
    assert np.isclose(r["trajectories"][0, 1, 0], 7.25 + 0.5)


def test_every_abort_reason():
    """3D border addressing makes the wind fall to 0 past the last node, so only a step that
    overshoots the domain end aborts with Domain; a creeping particle stalls (Wind)."""
    wind = uniform((6, 8, 16), 2, [1.0, 0.0, 0.0])
    for snap in wind:
        snap[0][:, :, 0:2] = 0.0       # no wind at x in [0, 1]
    topo = np.zeros((8, 16), np.float32)
    topo[4:, 10:] = 5.0                # terrain at x >= 10, y >= 4
    st = dict(Space=0, Integrator=0, WindfieldMode=0, DeltaT=2.0, GridScale=[1.0, 1.0, 1.0],
              Offset=[0.0, 0.0, 0.0], MaximumSimulationTime=8.0, SaveInterval=1, AbortMode=1, MaximumLength=4.5)
    # the length check runs before the border checks (tpp:252-284)
    seeds = np.array([[14.5, 2.0, 2.5],     # overshoots x = 16           -> Domain, step 0
                      [0.2, 2.0, 2.5],      # no wind                      -> Wind, step 0
                      [6.5, 5.0, 2.5],      # runs into the terrain        -> Topography, step 1
                      [1.5, 2.0, 2.5]], np.float32)   # length 1, 3, 5 > 4.5   -> Length, step 2
    r = orc.run(orc.settings(**st), orc.Inputs(wind=wind, seeds=seeds, topography=topo), precision="f64")
    assert list(r["status"]) == [2, 4, 3, 1]
    assert list(r["step_of_abort"]) == [0, 0, 1, 2]
    t = r["trajectories"]
    # Domain / Wind / Topography keep the last valid position; Length still moves on its step
    assert np.allclose(t[0, -1], seeds[0]) and np.allclose(t[1, -1], seeds[1])
    assert np.allclose(t[2, -1], [8.5, 5.0, 2.5])
    assert np.isclose(r["lengths"][3], 5.0) and np.allclose(t[3, -1], [6.5, 2.0, 2.5])
    # creeping toward the +x end under border addressing never leaves the domain
    st_c = dict(st, DeltaT=0.5, AbortMode=0, MaximumSimulationTime=400.0)
    r = orc.run(orc.settings(**st_c), orc.Inputs(wind=wind, seeds=seeds[:1]), precision="f64")
    assert r["status"][0] == 4 and r["trajectories"][0, -1, 0] < 16.0


def test_fit_length_stops_exactly():
    st = dict(Space=1, Integrator=0, WindfieldMode=0, DeltaT=0.5, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
              MaximumSimulationTime=10.0, SaveInterval=1, AbortMode=2, MaximumLength=2.6)
    r = run(st, uniform((8, 32), 1, [1.0, 0.0]), [[1.0, 1.0]])
    assert r["status"][0] == 1
    assert np.isclose(r["lengths"][0], 2.6)
    assert np.isclose(r["trajectories"][0, -1, 0], 3.6)


def test_save_interval_indexing():
    """Records: the seed, then after every step whose pre-increment counter % SaveInterval == 0."""
    wind = rotation_field(32, 0.05, 16.0)
    base = dict(Space=1, Integrator=1, WindfieldMode=0, DeltaT=0.5, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
                MaximumSimulationTime=10.0)
    all_ = run(dict(base, SaveInterval=1), wind, [[20.0, 16.0]])["trajectories"]
    every3 = run(dict(base, SaveInterval=3), wind, [[20.0, 16.0]])["trajectories"]
    final = run(dict(base, SaveInterval=0), wind, [[20.0, 16.0]])["trajectories"]
    assert all_.shape[1] == 21 and every3.shape[1] == 1 + 7 and final.shape[1] == 2
    assert np.array_equal(every3[0, 1:], all_[0, 1::3])
    assert np.array_equal(final[0, -1], all_[0, -1])


def test_window_schedule_reproduces_float32_time():
    """h = 0.01, DataTimeDistance = 1: the float32 accumulator stays below 1.0 after 100 steps,
    so window 0 runs 101 steps (tpp:990-993)."""
    wind = uniform((4, 8), 16, [0.0, 0.0])
    st = dict(Space=1, Integrator=0, DeltaT=0.01, DataTimeDistance=1.0, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
              MaximumSimulationTime=10.0)
    steps, windows = orc.schedule(orc.settings(**st), orc.Inputs(wind=wind, seeds=np.zeros((1, 2), np.float32)))
    assert len(steps) == 1000 and windows == 10
    switches = [k for k in range(1, 1000) if steps[k]["window"] != steps[k - 1]["window"]]
    assert switches[0] == 101
    t = np.float32(0)
    for _ in range(100):
        t = np.float32(t + np.float32(0.01))
    assert t < np.float32(1.0)


def test_loader_exhaustion_and_constant_windfield():
    wind = uniform((4, 8), 3, [0.1, 0.0])
    st = dict(Space=1, Integrator=0, DeltaT=0.5, DataTimeDistance=1.0, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
              MaximumSimulationTime=100.0)
    r = run(st, wind, [[1.0, 1.0]])
    assert r["windows"] == 2 and r["steps"] == 4     # 3 snapshots -> 2 windows
    r = run(dict(st, WindfieldMode=0), wind, [[1.0, 1.0]])
    assert r["windows"] == 1 and r["steps"] == 200   # constant field: one window to the end time


def test_reverse_is_the_reference_double_negation():
    """Reverse negates dp (tpp:249) and subtracts it again (tpp:282): positions are unchanged."""
    wind = uniform((4, 8), 1, [0.5, 0.25])
    st = dict(Space=1, Integrator=1, WindfieldMode=0, DeltaT=0.5, GridScale=[1.0, 1.0], Offset=[0.0, 0.0],
              MaximumSimulationTime=2.0)
    a = run(st, wind, [[1.0, 1.0]])["trajectories"]
    b = run(dict(st, Reverse=True), wind, [[1.0, 1.0]])["trajectories"]
    assert np.array_equal(a, b)


def test_float32_build_tracks_float64():
    from pygranite_b200 import workloads as W
    settings, src, seeds = W.config1(n_particles=500)
    data = orc.Inputs(wind=src.wind, seeds=seeds)
    r64 = orc.run(orc.settings(**settings), data, precision="f64")
    r32 = orc.run(orc.settings(**settings), data, precision="f32")
    assert (r64["status"] == r32["status"]).mean() > 0.99
    err = np.abs(r32["trajectories"].astype(np.float64) - r64["trajectories"]) / np.array([2 / 256, 1 / 128])
    assert np.median(err[:, -1]) < 1e-3


def test_expression_and_volume_in_oracle():
    wind = uniform((4, 6, 8), 2, [1.0, 0.0, 0.0])
    T = np.zeros((4, 6, 8), np.float32) + np.arange(8, dtype=np.float32)   # T = x index
    st = dict(Space=0, Integrator=1, WindfieldMode=0, DeltaT=1.0, GridScale=[1.0, 1.0, 1.0],
              Offset=[0.0, 0.0, 0.0], MaximumSimulationTime=2.0, AdditionalVolumeMode=1,
              AdditionalCompute=["T*2 + u"])
    r = orc.run(orc.settings(**st), orc.Inputs(wind=wind, seeds=np.array([[1.5, 2.0, 2.0]], np.float32),
                                               volumes=[{"T": T}]), precision="f64")
    assert np.allclose(r["volume_info"]["T"][0], [2.5, 3.5])
    assert np.allclose(r["compute_info"][0][0], [6.0, 8.0])
