"""Golden fixtures from the reference's own CUDA kernel.

tests/golden/*.npz were written by tests/golden/make_golden.py: the reference's `integrate`
kernel (TrajectoryIntegrator.tpp:108-457, instantiated unmodified from its sources by
oracle/ref_harness) run on a B200 with the reference's texture setup and host loop.  The
inputs are regenerated here from seeds.  The reference interpolates through texture hardware
with 8-bit weights, so positions are matched within stated tolerances.  Abort codes, step
counts, windows and record counts are matched exactly, except the border-creep stalls.  Under
3D border addressing a particle creeping toward an upper face stalls (Wind) at a step that
depends on the interpolation's rounding; those particles (within one cell of an upper face)
are excluded.

filter_reference.npz pins the texture filter itself: the oracle with weights rounded to the
nearest 1/256 (filter_weights=1) reproduces the reference bit for bit in 2D and within one
1/256 weight step in 3D.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden import make_golden as MG

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(HERE, name))


def cells(a, b, cell):
    return (np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / np.asarray(cell)).max(-1)


def check_gyre(res, g):
    assert res["trajectories"].shape == g["trajectories"].shape
    assert np.array_equal(res["status"], g["status"])
    e = cells(res["trajectories"], g["trajectories"], [2 / 256, 1 / 128])
    # 8-bit texture weights: after 100 steps the median difference stays below 1e-4 cells,
    # after 1000 below 1e-3
    assert np.median(e[:, 10]) < 1e-4 and np.median(e[:, 100]) < 1e-3, (np.median(e[:, 10]), np.median(e[:, 100]))
    assert e.max() < 0.05


def check_fourier(res, f):
    assert res["trajectories"].shape == f["trajectories"].shape
    upper = np.array([24000.0, 24000.0, 4000.0])
    cell = np.array([1000.0, 1000.0, 250.0])
    near = (np.abs(f["trajectories"][:, -1] - upper) < cell).any(1) | \
        (np.abs(res["trajectories"][:, -1] - upper) < cell).any(1)
    assert np.array_equal(res["status"][~near], f["status"][~near])
    e = cells(res["trajectories"], f["trajectories"], cell)
    assert np.median(e[:, 1]) < 1e-3 and np.median(e[:, -1]) < 3e-3
    both = (res["status"] == 0) & (f["status"] == 0)
    tc_rel = np.abs(res["total_curvature"][both] - f["total_curvature"][both]) / np.abs(res["total_curvature"][both])
    assert np.median(tc_rel) < 5e-3
    vol = res["volume_info"]["T"] if isinstance(res["volume_info"], dict) else res["volume_info"]
    assert np.median(np.abs(vol - f["volume_info"])) < 0.02       # Kelvin; field noise 2 K
    cmp_, ref_cmp = res["compute_info"][0], f["compute_info"]
    nz = ref_cmp != 0            # particles that aborted on their first step keep the initial 0
    assert np.median(np.abs(cmp_[nz] - ref_cmp[nz]) / np.abs(ref_cmp[nz])) < 2e-3


def test_fixture_bookkeeping():
    g, f = load("gyre_reference.npz"), load("fourier_reference.npz")
    sg, sf = json.loads(str(g["settings"])), json.loads(str(f["settings"]))
    assert int(g["steps"]) == 1000 and int(g["windows"]) == 10 and g["trajectories"].shape == (256, 101, 2)
    assert int(f["steps"]) == 50 and f["trajectories"].shape == (512, 6, 3)
    assert sg["SaveInterval"] == MG.GYRE["save_interval"] and sf["AdditionalCompute"] == ["sqrt(u*u+v*v)*T"]


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_oracle_matches_reference_kernel_gyre(precision):
    s, src, seeds = MG.gyre_case()
    res = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds), precision)
    g = load("gyre_reference.npz")
    assert res["steps"] == int(g["steps"]) and res["windows"] == int(g["windows"])
    check_gyre(res, g)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_oracle_matches_reference_kernel_fourier(precision):
    s, src, seeds = MG.fourier_case()
    res = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds, volumes=src.volumes), precision)
    f = load("fourier_reference.npz")
    assert res["steps"] == int(f["steps"])
    check_fourier(res, f)


@pytest.mark.gpu
def test_engine_matches_reference_kernel():
    from tests import harness as H
    s, src, seeds = MG.gyre_case()
    check_gyre(H.run_engine(s, src.wind, seeds), load("gyre_reference.npz"))
    s, src, seeds = MG.fourier_case()
    check_fourier(H.run_engine(s, src.wind, seeds, volumes=src.volumes), load("fourier_reference.npz"))


# ------------------------------------------------------------ the texture filter itself
# filter_reference.npz: one Euler step of the reference kernel through a field equal to its own
# grid coordinates (make_golden.filter_case), so each new position encodes the weight the
# texture unit used.  The oracle's filter_weights=1 mode (fractions rounded to the nearest
# 1/256) is the model checked here.

def _filter_run(dim, filter_weights):
    s, src, seeds = MG.filter_case(dim)
    return orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds), "f32",
                   filter_weights=filter_weights)


def test_texture_filter_2d_is_nearest_256th():
    g = load("filter_reference.npz")
    r = _filter_run(2, 1)
    assert np.array_equal(r["status"], g["status2d"])
    assert np.array_equal(r["trajectories"][:, 1], g["positions2d"])        # every particle, bit for bit
    exact = _filter_run(2, 0)
    assert not np.array_equal(exact["trajectories"][:, 1], g["positions2d"])


def test_texture_filter_3d_within_one_256th():
    # 3D (cudaArray, border addressing): the z weights are the nearest 1/256 for every sample;
    # x and y weights differ from it by one 1/256 step for some samples (about 2% on the
    # 16-node x axis, a third on the 12-node y axis), never by more.
    g = load("filter_reference.npz")
    r = _filter_run(3, 1)
    assert np.array_equal(r["status"], g["status3d"])
    got, ref = r["trajectories"][:, 1], g["positions3d"]
    same = (got == ref).mean(0)
    assert same[2] == 1.0 and same[0] > 0.95 and same[1] > 0.6, same
    step = np.abs(got.astype(np.float64) - ref) * 16 * 256     # h = 1/16: weight difference in 1/256
    assert step.max() <= 1.0 + 1e-6, step.max()


def test_texture_weight_mode_tracks_the_gyre_fixture():
    # with 1/256 weights the float32 oracle reproduces most of the reference's 2D run bit for bit
    s, src, seeds = MG.gyre_case()
    g = load("gyre_reference.npz")
    tex = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds), "f32", filter_weights=1)
    ideal = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds), "f32")
    same = lambda r: np.all(r["trajectories"][:, 1] == g["trajectories"][:, 1], axis=1).mean()  # noqa: E731
    assert same(tex) > 0.85 and same(ideal) < 0.2, (same(tex), same(ideal))
    e_tex = cells(tex["trajectories"], g["trajectories"], [2 / 256, 1 / 128])
    e_ideal = cells(ideal["trajectories"], g["trajectories"], [2 / 256, 1 / 128])
    assert np.median(e_tex[:, 10]) < np.median(e_ideal[:, 10]) / 5


@pytest.mark.gpu
def test_engine_reference_filter_matches_the_reference_kernel():
    # IntegratorSettings.ReferenceFilter: the engine rounds its interpolation weights like the
    # reference's texture unit (nearest 1/256).  It equals the oracle's texture mode bit for bit,
    # hence the reference's own 2D outputs bit for bit.
    from tests import harness as H
    g = load("filter_reference.npz")
    for dim in (2, 3):
        s, src, seeds = MG.filter_case(dim)
        eng = H.run_engine(s, src.wind, seeds, ReferenceFilter=True)
        ora = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds), "f32", filter_weights=1)
        assert np.array_equal(eng["trajectories"], ora["trajectories"]), dim
        assert np.array_equal(eng["status"], ora["status"]), dim
    s, src, seeds = MG.filter_case(2)
    assert np.array_equal(H.run_engine(s, src.wind, seeds, ReferenceFilter=True)["trajectories"][:, 1],
                          g["positions2d"])
    s, src, seeds = MG.gyre_case()
    gy = load("gyre_reference.npz")
    eng = H.run_engine(s, src.wind, seeds, ReferenceFilter=True)
    assert np.all(eng["trajectories"][:, 1] == gy["trajectories"][:, 1], axis=1).mean() > 0.85
    s, src, seeds = MG.fourier_case()
    eng = H.run_engine(s, src.wind, seeds, volumes=src.volumes, ReferenceFilter=True)
    ora = orc.run(orc.settings(**s), orc.Inputs(wind=src.wind, seeds=seeds, volumes=src.volumes), "f32",
                  filter_weights=1)
    H.assert_same(eng, ora, ("trajectories", "status", "total_curvature"))
    assert np.array_equal(eng["volume_info"]["T"], ora["volume_info"]["T"])
    assert np.array_equal(eng["compute_info"][0], ora["compute_info"][0])


# ------------------------------------------------------------ the option matrix
# options_reference.npz: the reference's kernel instantiated for the option combinations of
# make_golden.OPTION_CASES (TrajectoryIntegrator.tpp:13-104 loop borders and sphere
# coordinates, 233-280 uplift and length aborts, 335-361 curvature, 396-435 constants,
# icc:131-137 topography, 249 / 282 reverse, constant wind).  The oracle's texture-weight mode
# (fractions rounded to the nearest 1/256) and the engine's ReferenceFilter are compared with it
# within tolerances: the texture unit's own arithmetic is not documented beyond its 8-bit
# weights, so values drift apart by float rounding over the run.

def options_fixture():
    return load("options_reference.npz")


def option_fixture_case(f, name):
    keys = {k.split("/", 1)[1] for k in f.files if k.startswith(name + "/")}
    return {k: f[f"{name}/{k}"] for k in keys}


def check_option_case(name, res, ref):
    """Abort codes, positions, lengths, curvature and expression values against the reference
    kernel's.  Tolerances (the reference interpolates in texture hardware; see the module
    docstring): abort codes equal for at least 95% of the particles (a particle at a border or
    length threshold within rounding may stop a step apart); positions of the particles alive in
    both, in grid cells: median < 3e-4 after 5 steps and < 1e-2 after 60, 90th percentile < 0.5
    after 60 (sphere coordinates with pole crossings amplify differences); lengths and
    expression values: median relative difference < 2e-3; total and per-step curvature < 2e-2;
    volume samples: median < 0.02 K."""
    settings = make_golden_settings(name)
    cell = np.asarray(settings["GridScale"], np.float64)
    assert res["trajectories"].shape == ref["trajectories"].shape, (res["trajectories"].shape, ref["trajectories"].shape)
    same = (res["status"] == ref["status"]).mean()
    assert same >= 0.95, (name, same)
    both = (res["status"] == 0) & (ref["status"] == 0)
    e = cells(res["trajectories"][both], ref["trajectories"][both], cell)
    if e.size:
        assert np.median(e[:, 1]) < 3e-4 and np.median(e[:, -1]) < 1e-2, (name, np.median(e[:, 1]), np.median(e[:, -1]))
        assert np.percentile(e[:, -1], 90) < 0.5, (name, np.percentile(e[:, -1], 90))

    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        ok = np.isfinite(a) & np.isfinite(b) & (np.abs(b) > 1e-12)
        return np.median(np.abs(a[ok] - b[ok]) / np.abs(b[ok])) if ok.any() else 0.0

    if settings.get("AbortMode", 0):
        assert rel(res["lengths"][both], ref["lengths"][both]) < 2e-3, name
    if settings.get("CurvatureMode", 0):
        assert rel(res["total_curvature"][both], ref["total_curvature"][both]) < 2e-2, name
    if settings.get("CurvatureMode", 0) == 3:
        assert res["curvatures"].shape == ref["curvatures"].shape
        assert rel(res["curvatures"][both], ref["curvatures"][both]) < 2e-2, name
    if settings.get("AdditionalCompute"):
        assert rel(res["compute_info"][0][both], ref["compute_0"][both]) < 2e-3, name
    if settings.get("AdditionalVolumeMode", 0):
        assert np.median(np.abs(res["volume_info"]["T"][both] - ref["volume_T"][both])) < 0.02, name


def make_golden_settings(name):
    return MG.option_case(name)[0]


@pytest.mark.parametrize("name", sorted(MG.OPTION_CASES))
def test_oracle_matches_reference_kernel_options(name):
    f = options_fixture()
    settings, wind, seeds, volumes, constants, uplift, topography = MG.option_case(name)
    res = orc.run(orc.settings(**settings), orc.Inputs(wind=wind, seeds=seeds, volumes=volumes or [],
                                                       constants=constants or [], uplift=uplift or [],
                                                       topography=topography), "f32", filter_weights=1)
    ref = option_fixture_case(f, name)
    assert res["steps"] == int(ref["steps"])
    check_option_case(name, res, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(MG.OPTION_CASES))
def test_engine_matches_reference_kernel_options(name):
    from tests import harness as H
    f = options_fixture()
    settings, wind, seeds, volumes, constants, uplift, topography = MG.option_case(name)
    res = H.run_engine(settings, wind, seeds, volumes=volumes, constants=constants, uplift=uplift,
                       topography=topography, ReferenceFilter=True)
    check_option_case(name, res, option_fixture_case(f, name))
