"""Parity of the CUDA engine with the oracle (GPU).

Every case runs the same inputs through pygranite_b200 (sm_100a kernels) and through the
CPU oracle.  Against the float32 oracle build, which follows the kernel's float operation
order, positions, abort codes, lengths, curvature, volume samples and expression values are
compared bit for bit; only cases that call transcendental functions (cosf in the sphere
transform, acosf in FastTotalCurvature, exp/sin/... in expressions) use a tolerance, written
in the test.  Against the float64 oracle (the accuracy reference) errors are reported in grid cells.
"""
import numpy as np
import pytest

from pygranite_b200 import workloads as W
from tests import harness as H

pytestmark = pytest.mark.gpu


def rng_field(shape, n_snap, seed, scale=1.0, zero_box=None):
    rng = np.random.default_rng(seed)
    snaps = []
    for _ in range(n_snap):
        comps = []
        for c in range(len(shape)):
            a = (rng.standard_normal(shape) * scale).astype(np.float32)
            if zero_box is not None:
                a[zero_box] = 0.0
            comps.append(a)
        snaps.append(comps)
    return snaps


def problem2d(n=3000, n_snap=6, seed=0, zero=True):
    shape = (32, 48)   # (ny, nx)
    zb = (slice(10, 14), slice(20, 26)) if zero else None
    wind = rng_field(shape, n_snap, seed, 1.0, zb)
    seeds = np.random.default_rng(seed + 100).uniform([0, 0], [48, 32], (n, 2)).astype(np.float32)
    base = dict(Space=1, Integrator=1, WindfieldMode=1, DeltaT=0.5, DataTimeDistance=4.0,
                GridScale=[1.0, 1.0], Offset=[0.0, 0.0], SaveInterval=1, MaximumSimulationTime=16.0)
    return base, wind, seeds


def problem3d(n=3000, n_snap=6, seed=0, zero=True):
    shape = (12, 20, 24)   # (nz, ny, nx)
    zb = (slice(2, 5), slice(6, 9), slice(8, 12)) if zero else None
    wind = rng_field(shape, n_snap, seed, 1.0, zb)
    for s in wind:
        s[2] *= 0.2
    seeds = np.random.default_rng(seed + 200).uniform([0, 0, 0], [24, 20, 12], (n, 3)).astype(np.float32)
    base = dict(Space=0, Integrator=1, WindfieldMode=1, DeltaT=0.5, DataTimeDistance=4.0,
                GridScale=[1.0, 1.0, 1.0], Offset=[0.0, 0.0, 0.0], SaveInterval=1, MaximumSimulationTime=16.0)
    return base, wind, seeds


# ---------------------------------------------------------------- benchmark configurations

def test_config1_double_gyre_bitexact():
    from pygranite_b200 import workloads as W
    settings, src, seeds = W.config1(n_particles=3000)
    eng = H.run_engine(settings, src.wind, seeds)
    ref32 = H.run_oracle(settings, src.wind, seeds, precision="f32")
    H.assert_same(eng, ref32)
    assert eng["trajectories"].shape == (3000, 1001, 2)
    # loader calls: one in the constructor + one after every window (tpp:887, cpp:252)
    assert eng["loader_calls"] == 1 + ref32["windows"]
    ref64 = H.run_oracle(settings, src.wind, seeds, precision="f64")
    err = H.cell_error(eng["trajectories"], ref64["trajectories"], [2 / 256, 1 / 128])
    final = err[:, -1]
    print(f"config1 vs f64: max {err.max():.3e} rms {np.sqrt((err ** 2).mean()):.3e} cells; "
          f"final median {np.median(final):.3e}")
    assert np.median(final) < 1e-3


def test_config2_small_bitexact():
    from pygranite_b200 import workloads as W
    settings, src, seeds = W.config2(n_particles=4000, n_snapshots=6, grid=(16, 24, 24), steps=50)
    eng = H.run_engine(settings, src.wind, seeds, volumes=src.volumes)
    ref = H.run_oracle(settings, src.wind, seeds, volumes=src.volumes, precision="f32")
    H.assert_same(eng, ref, ("trajectories", "status", "total_curvature"))
    assert np.array_equal(eng["volume_info"]["T"], ref["volume_info"]["T"])
    assert np.array_equal(eng["compute_info"][0], ref["compute_info"][0])
    assert eng["trajectories"].shape[1] == 1 + 5
    assert set(np.unique(eng["status"])) <= {0, 2, 4}


# ---------------------------------------------------------------- option coverage

EXACT_2D = {
    "euler": dict(Integrator=0),
    "rk4": dict(),
    "loopx": dict(BorderMode=1),
    "loopy": dict(BorderMode=2),
    "loopxy": dict(BorderMode=3),
    "reverse": dict(Reverse=True),
    "windfield_constant": dict(WindfieldMode=0),
    "abort_length": dict(AbortMode=1, MaximumLength=6.0),
    "abort_fitlength": dict(AbortMode=2, MaximumLength=6.0),
    "save_every_3": dict(SaveInterval=3),
    "save_final_only": dict(SaveInterval=0),
    "offset_and_scale": dict(GridScale=[0.5, 2.0], Offset=[-3.0, 5.0]),
    "single_scale": dict(GridScale=[0.75], Offset=[1.0]),
}


@pytest.mark.parametrize("name", sorted(EXACT_2D))
def test_options_2d_bitexact(name):
    base, wind, seeds = problem2d(seed=len(name))
    settings = dict(base, **EXACT_2D[name])
    if name == "offset_and_scale":
        seeds = (seeds * np.array([0.5, 2.0], np.float32) + np.array([-3.0, 5.0], np.float32)).astype(np.float32)
    if name == "single_scale":
        seeds = (seeds * 0.75 + 1.0).astype(np.float32)
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    keys = ("trajectories", "status") + (("lengths",) if settings.get("AbortMode", 0) else ())
    H.assert_same(eng, ref, keys)


EXACT_3D = {
    "euler": dict(Integrator=0),
    "rk4": dict(),
    "curv_total": dict(CurvatureMode=1),
    "curv_individual": dict(CurvatureMode=3),
    "abort_length": dict(AbortMode=1, MaximumLength=5.0),
    "abort_fitlength": dict(AbortMode=2, MaximumLength=5.0, CurvatureMode=1),
    "windfield_constant": dict(WindfieldMode=0),
    "reverse": dict(Reverse=True),
    "save_final_only": dict(SaveInterval=0, CurvatureMode=3),
}


@pytest.mark.parametrize("name", sorted(EXACT_3D))
def test_options_3d_bitexact(name):
    base, wind, seeds = problem3d(seed=len(name) + 7)
    settings = dict(base, **EXACT_3D[name])
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    keys = ["trajectories", "status"]
    if settings.get("AbortMode", 0):
        keys.append("lengths")
    if settings.get("CurvatureMode", 0):
        keys.append("total_curvature")
    if settings.get("CurvatureMode", 0) == 3:
        keys.append("curvatures")
    H.assert_same(eng, ref, keys)


def test_uplift_and_topography_3d():
    base, wind, seeds = problem3d(seed=11)
    n = seeds.shape[0]
    rng = np.random.default_rng(5)
    uplift = [(rng.standard_normal((n, 3)) * 0.05).astype(np.float32) for _ in wind]
    topo = np.zeros((20, 24), np.float32)
    topo[:, 16:] = 6.0     # a plateau in x >= 16
    for mode in (1, 2):
        settings = dict(base, UpLiftMode=mode)
        eng = H.run_engine(settings, wind, seeds, uplift=uplift, topography=topo)
        ref = H.run_oracle(settings, wind, seeds, uplift=uplift, topography=topo, precision="f32")
        H.assert_same(eng, ref)
        assert (eng["status"] == 3).any(), "no particle hit the topography"


def test_volumes_constants_expressions():
    base, wind, seeds = problem3d(seed=3)
    n = seeds.shape[0]
    rng = np.random.default_rng(9)
    vols = [{"temp": rng.standard_normal((12, 20, 24)).astype(np.float32),
             "hum": rng.standard_normal((12, 20, 24)).astype(np.float32)} for _ in wind]
    cons = [{"ka": rng.standard_normal(n).astype(np.float32), "kb": rng.standard_normal(n).astype(np.float32)}
            for _ in wind]
    exprs = ["temp*ka + hum/2 - z", "(u*u + v*v + w*w)*kb", "x - y*2.5 + -1"]
    for vm, cm in ((1, 1), (2, 2), (1, 2), (2, 1)):
        settings = dict(base, AdditionalVolumeMode=vm, ConstantsMode=cm, AdditionalCompute=exprs)
        eng = H.run_engine(settings, wind, seeds, volumes=vols, constants=cons)
        ref = H.run_oracle(settings, wind, seeds, volumes=vols, constants=cons, precision="f32")
        H.assert_same(eng, ref)
        for k in ("temp", "hum"):
            assert np.array_equal(eng["volume_info"][k], ref["volume_info"][k]), (vm, cm, k)
        for e in range(len(exprs)):
            assert np.array_equal(eng["compute_info"][e], ref["compute_info"][e]), (vm, cm, e)


def test_transcendental_expressions_within_ulps():
    base, wind, seeds = problem3d(seed=4)
    settings = dict(base, CurvatureMode=3,
                    AdditionalCompute=["sqrt(x*x+y*y)", "exp(z/10) + ln(x+1)", "sin(x)*cos(y) - tan(z/20)",
                                       "atan2(v, u) + asin(w/10) + acos(w/10) + atan(cv)"])
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    H.assert_same(eng, ref, ("trajectories", "status", "curvatures"))
    # CUDA's and glibc's float functions differ by a few ulp.  Each expression sums at most
    # four terms of magnitude <= max(pi, |x|, |value|); tolerance: 4 terms x 4 ulp of that.
    eps = np.finfo(np.float32).eps
    pos = np.abs(eng["trajectories"][:, 1:, :]).max(axis=-1)
    for e in range(4):
        a, b = eng["compute_info"][e], ref["compute_info"][e]
        tol = 16 * eps * np.maximum(np.maximum(np.pi, np.abs(b)), pos)
        bad = ~((np.abs(a - b) <= tol) | (np.isnan(a) & np.isnan(b)))
        assert not bad.any(), (e, np.abs(a - b)[bad][:5], tol[bad][:5])


def test_fast_total_curvature_and_sphere_2d():
    base, wind, seeds = problem2d(seed=21)
    settings = dict(base, CurvatureMode=2)
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    H.assert_same(eng, ref)   # positions do not depend on acosf
    tc_e, tc_r = eng["total_curvature"], ref["total_curvature"]
    assert np.allclose(tc_e, tc_r, rtol=1e-5, atol=1e-5)
    # sphere coordinates (cosf): 10-degree grid over the globe, 1 h steps, tolerance checks
    ny, nx = 18, 36
    wind_s = rng_field((ny, nx), 6, 3, 10.0)
    seeds_s = np.random.default_rng(1).uniform([0, -80], [360, 80], (2000, 2)).astype(np.float32)
    for bm in (2, 3):
        st = dict(Space=1, Integrator=1, WindfieldMode=1, DeltaT=3600.0, DataTimeDistance=21600.0,
                  GridScale=[10.0, 10.0], Offset=[0.0, -90.0], SaveInterval=1, MaximumSimulationTime=86400.0,
                  SphereRadius=6371000.0, BorderMode=bm)
        e = H.run_engine(st, wind_s, seeds_s)
        r = H.run_oracle(st, wind_s, seeds_s, precision="f32")
        assert (e["status"] == r["status"]).mean() > 0.995
        same = e["status"] == r["status"]
        d = np.abs(e["trajectories"][same] - r["trajectories"][same])
        assert np.nanmax(d) < 1e-2, np.nanmax(d)


def test_minimum_alive_particles():
    base, wind, seeds = problem2d(seed=5, n=2000)
    settings = dict(base, MinimumAliveParticles=1500, MaximumSimulationTime=40.0)
    wind = wind + rng_field((32, 48), 6, 77)
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    H.assert_same(eng, ref)
    assert eng["trajectories"].shape[1] < 1 + 80, "MinimumAliveParticles never stopped the run"


@pytest.mark.parametrize("extra", [dict(), dict(SortInterval=1), dict(WindLayout=1, StepsPerLaunch=7),
                                   dict(CompensatedPositions=True, SortInterval=2)])
def test_minimum_alive_stops_inside_a_launch(extra):
    """MinimumAliveParticles with whole-window launches: the engine counts the particles alive
    after every step, and when the count falls below the minimum inside a launch it restores
    the state saved before the launch and runs only the steps the reference runs.  The minimum
    is chosen from the oracle's abort steps so that the stop falls in the middle of a window;
    every output must equal the float32 oracle's step-by-step check."""
    base, wind, seeds = problem3d(seed=11)
    vols = [{"temp": np.random.default_rng(9).standard_normal((12, 20, 24)).astype(np.float32)} for _ in wind]
    settings = dict(base, CurvatureMode=3, SaveInterval=3, AdditionalVolumeMode=1,
                    AdditionalCompute=["x + cv*2", "temp - z"])
    comp = bool(extra.get("CompensatedPositions", False))
    free = H.run_oracle(settings, wind, seeds, volumes=vols, precision="f32", compensated=comp)
    ab = free["step_of_abort"]
    alive_before = lambda k: int(np.sum((ab < 0) | (ab >= k)))  # noqa: E731
    # a step inside a window (8 steps per window) right after particles were lost
    stop = next(k for k in range(11, 30) if k % 8 not in (0, 1) and alive_before(k) < alive_before(k - 1))
    settings["MinimumAliveParticles"] = alive_before(stop) + 1
    ref = H.run_oracle(settings, wind, seeds, volumes=vols, precision="f32", compensated=comp)
    assert ref["steps"] == stop
    eng = H.run_engine(settings, wind, seeds, volumes=vols, **extra)
    H.assert_same(eng, ref, ("trajectories", "status", "total_curvature", "curvatures"))
    assert np.array_equal(eng["volume_info"]["temp"], ref["volume_info"]["temp"])
    for k in range(2):
        assert np.array_equal(eng["compute_info"][k], ref["compute_info"][k])


def test_loader_exhaustion_truncates_like_reference():
    base, wind, seeds = problem3d(seed=8, n_snap=3)
    settings = dict(base, MaximumSimulationTime=100.0)    # needs 25 windows, 2 available
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    H.assert_same(eng, ref)
    assert ref["windows"] == 2 and eng["trajectories"].shape[1] == 1 + ref["steps"]


LAUNCH_SHAPES = [dict(StepsPerLaunch=1), dict(StepsPerLaunch=7), dict(BlockSize=32),
                 dict(BlockSize=256, RingSlots=8), dict(RingSlots=4, StepsPerLaunch=3),
                 dict(SortInterval=1), dict(SortInterval=1, StepsPerLaunch=1), dict(SortInterval=2, StepsPerLaunch=3),
                 dict(SortInterval=1, RingSlots=8, StepsPerLaunch=5),
                 dict(WindLayout=1), dict(WindLayout=1, SortInterval=2, StepsPerLaunch=3)]


@pytest.mark.parametrize("extra", LAUNCH_SHAPES)
def test_launch_shape_does_not_change_results(extra):
    """Launch granularity, block size, ring depth and compaction / re-sorting of the live
    particles change nothing: every output stays bit-identical to the float32 oracle."""
    base, wind, seeds = problem3d(seed=2)
    vols = [{"temp": np.random.default_rng(4).standard_normal((12, 20, 24)).astype(np.float32)} for _ in wind]
    # the lean variants defer volume / expression values to a kernel after each launch (records
    # every 3 steps: several per window, launches split to one save step each)
    for extra_settings, exprs in ((dict(CurvatureMode=3, SaveInterval=2), ["x + cv*2", "temp - z"]),
                                  (dict(CurvatureMode=1, SaveInterval=0), ["x*2", "temp - z"]),
                                  (dict(CurvatureMode=1, SaveInterval=3), ["x*2", "temp - z + u*v"])):
        settings = dict(base, AdditionalVolumeMode=1, AdditionalCompute=exprs, **extra_settings)
        ref = H.run_oracle(settings, wind, seeds, volumes=vols, precision="f32")
        eng = H.run_engine(settings, wind, seeds, volumes=vols, **extra)
        H.assert_same(eng, ref, ("trajectories", "status", "total_curvature", "curvatures"))
        assert np.array_equal(eng["volume_info"]["temp"], ref["volume_info"]["temp"])
        for k in range(2):
            assert np.array_equal(eng["compute_info"][k], ref["compute_info"][k])


def test_compaction_with_minimum_alive_and_2d():
    base, wind, seeds = problem2d(seed=6, n=2000)
    wind = wind + rng_field((32, 48), 6, 78)
    for settings in (dict(base, MinimumAliveParticles=1200, MaximumSimulationTime=40.0),
                     dict(base, BorderMode=3, AbortMode=2, MaximumLength=8.0, CurvatureMode=2)):
        ref = H.run_oracle(settings, wind, seeds, precision="f32")
        eng = H.run_engine(settings, wind, seeds, SortInterval=1, StepsPerLaunch=2)
        keys = ("trajectories", "status") + (("lengths",) if settings.get("AbortMode") else ())
        H.assert_same(eng, ref, keys)


def round_storage(a, storage):
    """The float32 -> storage -> float32 round trip of the device ring (round to nearest even)."""
    return W.round_storage(a, {"Float16": "f16", "BFloat16": "bf16"}.get(storage, "f32"))


# storage error bounds in grid cells after 100 steps (99th percentile over particles alive in
# both runs; a few particles in strained regions of the field diverge regardless of
# precision and dominate the RMS, which is reported).  From a float64 oracle run on the
# rounded field: BF16 keeps 8 mantissa bits, FP16 11.
STORAGE_P99_BOUND = {"Float32": 1e-4, "Float16": 5e-3, "BFloat16": 3e-2}


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("storage", ["BFloat16", "Float16", "Float32"])
def test_precision_forms_against_float64(storage, layout):
    """Precision form: 16-bit wind storage, float32 stages, Kahan-compensated positions and
    float64 time weights.
    (1) Bit for bit against the float32 oracle with the same compensation on the field
        rounded exactly as the device ring stores it.
    (2) Against the float64 oracle on the original field: the storage error stays within
        STORAGE_P99_BOUND.  Particles that end within one cell of an upper domain face are
        left out of the status comparison: under the reference's border addressing they
        creep toward the face and stall (Wind), at a step set by the float resolution."""
    import pygranite_b200 as pg
    from pygranite_b200 import workloads as W
    settings, src, seeds = W.config2(n_particles=3000, n_snapshots=12, grid=(16, 32, 32), steps=100)
    settings["CurvatureMode"] = 0
    cell = np.array([1000.0, 1000.0, 250.0])
    eng = H.run_engine(settings, src.wind, seeds, volumes=src.volumes, WindStorage=getattr(pg.WindStorage, storage),
                       CompensatedPositions=True, Float64Time=True, WindLayout=layout)
    rounded = [[round_storage(p, storage) for p in snap] for snap in src.wind]
    ref32 = H.run_oracle(settings, rounded, seeds, volumes=src.volumes, precision="f32", time_mode=1,
                         compensated=True)
    H.assert_same(eng, ref32)
    ref = H.run_oracle(settings, src.wind, seeds, volumes=src.volumes, precision="f64", time_mode=1)
    upper = np.array([32000.0, 32000.0, 4000.0])
    near = (np.abs(eng["trajectories"][:, -1] - upper) < cell).any(axis=1) | \
        (np.abs(ref["trajectories"][:, -1] - upper) < cell).any(axis=1)
    agree = (eng["status"] == ref["status"])[~near].mean()
    assert agree > 0.995, agree
    alive = (eng["status"] == 0) & (ref["status"] == 0)
    err = H.cell_error(eng["trajectories"][alive], ref["trajectories"][alive], cell)
    for rec in (1, 2, 5, 10):
        x = err[:, rec]
        print(f"{storage} step {rec * 10:4d}: rms {np.sqrt((x ** 2).mean()):.2e} p50 {np.median(x):.2e} "
              f"p99 {np.percentile(x, 99):.2e} max {x.max():.2e} cells")
    assert float(np.percentile(err[:, 10], 99)) < STORAGE_P99_BOUND[storage]


def test_errors_match_reference_messages():
    import pygranite_b200 as pg
    from pygranite_b200 import workloads as W
    base, wind, seeds = problem2d(n=10)
    s = W.apply_settings(pg.IntegratorSettings(), dict(base, Space=0), H.enums(pg))
    loader = W.make_loader(pg.DataLoader, W.SnapshotSource(wind))
    with pytest.raises(RuntimeError, match="Dimensions of IntegratorSettings and provided TrajectorySet do not match"):
        pg.TrajectoryIntegrator(s, loader, pg.TrajectorySet(seeds))
    s = W.apply_settings(pg.IntegratorSettings(), dict(base, CurvatureMode=1), H.enums(pg))
    integ = pg.TrajectoryIntegrator(s, W.make_loader(pg.DataLoader, W.SnapshotSource(wind)), pg.TrajectorySet(seeds))
    with pytest.raises(RuntimeError, match="No kernel could be picked"):
        integ.compute()
    s = W.apply_settings(pg.IntegratorSettings(), dict(base, AdditionalCompute=["x + w"]), H.enums(pg))
    integ = pg.TrajectoryIntegrator(s, W.make_loader(pg.DataLoader, W.SnapshotSource(wind)), pg.TrajectorySet(seeds))
    with pytest.raises(RuntimeError, match="undefinded token 'w'"):
        integ.compute()
    s = W.apply_settings(pg.IntegratorSettings(), base, H.enums(pg))
    with pytest.raises(RuntimeError, match="Cannot increment loader"):
        pg.TrajectoryIntegrator(s, W.make_loader(pg.DataLoader, W.SnapshotSource(wind[:1])), pg.TrajectorySet(seeds))


def test_loader_exception_propagates():
    import pygranite_b200 as pg
    from pygranite_b200 import workloads as W
    base, wind, seeds = problem2d(n=100)

    class Boom(Exception):
        pass

    class BadLoader(pg.DataLoader):
        def __init__(self):
            pg.DataLoader.__init__(self)
            self.k = 0

        def step(self):
            self.k += 1
            if self.k > 2:
                raise Boom("loader failed")
            return True

        def windfield(self):
            return wind[min(self.k, len(wind) - 1)]

    s = W.apply_settings(pg.IntegratorSettings(), base, H.enums(pg))
    integ = pg.TrajectoryIntegrator(s, BadLoader(), pg.TrajectorySet(seeds))
    with pytest.raises(Boom):
        integ.compute()


EDGE_CASES = {
    "one_particle": dict(n=1),
    "zero_steps": dict(MaximumSimulationTime=0.0),
    "shorter_than_a_step": dict(MaximumSimulationTime=0.25),
    "save_interval_longer_than_run": dict(SaveInterval=1000),
    "window_equals_step": dict(DeltaT=4.0, MaximumSimulationTime=16.0),
    "single_snapshot_constant": dict(WindfieldMode=0, n_snap=1),
}


@pytest.mark.parametrize("name", sorted(EDGE_CASES))
@pytest.mark.parametrize("space", [2, 3])
def test_edge_cases_bitexact(name, space):
    """Degenerate sizes and schedules: one particle, no step at all, a run shorter than one
    step, records rarer than the run, one step per window, one constant snapshot."""
    case = dict(EDGE_CASES[name])
    n = case.pop("n", 500)
    n_snap = case.pop("n_snap", 6)
    base, wind, seeds = (problem2d if space == 2 else problem3d)(n=max(n, 2), n_snap=n_snap, seed=31)
    seeds = seeds[:n]
    settings = dict(base, **case)
    eng = H.run_engine(settings, wind, seeds)
    ref = H.run_oracle(settings, wind, seeds, precision="f32")
    H.assert_same(eng, ref)


def test_compiled_expressions_equal_the_interpreter_and_the_oracle(monkeypatch):
    """The lean kernels defer volume / expression values to a kernel after each launch, whose
    expressions are compiled to straight-line code at run time (jit.cu); with GR_JIT=0 the
    bytecode interpreter evaluates them instead.  Both give the float32 oracle's values; the
    transcendental cases within the ulps of the interpreter test above."""
    from pygranite_b200 import capi
    base, wind, seeds = problem3d(seed=11)
    temp = [np.random.default_rng(12 + k).standard_normal((12, 20, 24)).astype(np.float32) for k in range(len(wind))]
    exprs = ["sqrt(u*u+v*v)*temp", "temp - z/3 + x*y - 1.25", "(u - v)/(w + 4) * -2"]
    settings = dict(base, CurvatureMode=1, AdditionalVolumeMode=2, SaveInterval=3, AdditionalCompute=exprs)
    ref = H.run_oracle(settings, wind, seeds, volumes=[{"temp": t} for t in temp], precision="f32")
    runs = {}
    for jit in ("1", "0"):
        monkeypatch.setenv("GR_JIT", jit)
        eng = capi.Engine(capi.settings_from_reference(settings, ring_slots=len(wind), sort_interval=2))
        eng.set_seeds(seeds)
        for k, snap in enumerate(wind):
            eng.load_windfield(k, snap)
            eng.load_volume(k, 0, temp[k])
        for e, code in enumerate(exprs):
            eng.compile_expression(e, code, ["temp"], [])
        eng.run(lambda k: 1 if k < len(wind) else 0)
        runs[jit] = (eng.results(), eng.stats().jit_launches)
        eng.close()
    assert runs["1"][1] > 0, "the run-time compiled kernel did not run"
    assert runs["0"][1] == 0
    for jit, (res, _) in runs.items():
        H.assert_same(res, ref, ("trajectories", "status", "total_curvature"))
        assert np.array_equal(res["volume_info"][0], ref["volume_info"]["temp"]), jit
        for e in range(len(exprs)):
            assert np.array_equal(res["compute_info"][e], ref["compute_info"][e]), (jit, e)


def test_deferred_values_with_lifetimes_match_shorter_oracle_runs():
    """Per-particle lifetimes with deferred volume / expression values, one plain run (the lean
    kernel, compaction every 2 launches): a particle whose lifetime ends retires with its final
    values, and its later records repeat its last state.  Set A lives 13 steps (its last step
    saves record 5), set B the whole run; each equals the float32 oracle run of that set alone
    with MaximumSimulationTime = lifetime * DeltaT."""
    from pygranite_b200 import capi
    base, wind, seeds = problem3d(seed=13)
    temp = np.random.default_rng(14).standard_normal((12, 20, 24)).astype(np.float32)
    exprs = ["sqrt(u*u+v*v)*temp", "temp - z*0.5 + x"]
    settings = dict(base, CurvatureMode=1, AdditionalVolumeMode=1, SaveInterval=3, AdditionalCompute=exprs)
    n = seeds.shape[0]
    half = n // 2
    life_a = 13
    lifes = np.full(n, int(settings["MaximumSimulationTime"] / settings["DeltaT"]), np.int32)
    lifes[:half] = life_a
    eng = capi.Engine(capi.settings_from_reference(settings, ring_slots=len(wind), sort_interval=2))
    eng.set_seeds(seeds)
    eng.set_lifetimes(lifes)
    for k, snap in enumerate(wind):
        eng.load_windfield(k, snap)
    eng.load_volume(0, 0, temp)
    for e, code in enumerate(exprs):
        eng.compile_expression(e, code, ["temp"], [])
    eng.run(lambda k: 1 if k < len(wind) else 0)
    res = eng.results()
    eng.close()
    vols = [{"temp": temp}]
    ref_a = H.run_oracle(dict(settings, MaximumSimulationTime=life_a * settings["DeltaT"]), wind, seeds[:half],
                         volumes=vols, precision="f32")
    ref_b = H.run_oracle(settings, wind, seeds[half:], volumes=vols, precision="f32")
    la = ref_a["trajectories"].shape[1]
    assert la == 6
    pos, vol, cmp = res["trajectories"], res["volume_info"][0], res["compute_info"]
    assert np.array_equal(pos[:half, :la], ref_a["trajectories"])
    assert np.array_equal(pos[:half, la:], np.repeat(ref_a["trajectories"][:, -1:], pos.shape[1] - la, axis=1))
    assert np.array_equal(vol[:half, :la - 1], ref_a["volume_info"]["temp"])
    assert np.array_equal(vol[:half, la - 1:], np.repeat(ref_a["volume_info"]["temp"][:, -1:], vol.shape[1] - la + 1, axis=1))
    for e in range(len(exprs)):
        assert np.array_equal(cmp[e][:half, :la - 1], ref_a["compute_info"][e])
        assert np.array_equal(cmp[e][:half, la - 1:], np.repeat(ref_a["compute_info"][e][:, -1:], cmp[e].shape[1] - la + 1, axis=1))
        assert np.array_equal(cmp[e][half:], ref_b["compute_info"][e])
    assert np.array_equal(pos[half:], ref_b["trajectories"])
    assert np.array_equal(vol[half:], ref_b["volume_info"]["temp"])
    assert np.array_equal(res["status"][:half], ref_a["status"]) and np.array_equal(res["status"][half:], ref_b["status"])
    assert np.array_equal(res["total_curvature"][:half], ref_a["total_curvature"])
    assert np.array_equal(res["total_curvature"][half:], ref_b["total_curvature"])
