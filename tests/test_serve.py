"""Serving: trajectory requests with continuous batching (gr_server_*).

Every request's result must be the same alone and in any mix of concurrent requests
(per-particle arithmetic depends only on the particle and the field's step clock), and a
request that starts on a window boundary must equal a plain engine run over the same
snapshots.  Both are compared bit for bit.
"""
import threading

import numpy as np
import pytest

from pygranite_b200 import capi
from pygranite_b200 import workloads as W

GRID = (16, 32, 32)
N_SNAP = 13


def field():
    f = W.FourierField(GRID, (250.0, 1000.0, 1000.0), n_modes=32, seed=5)
    return [f.snapshot(600.0 * k) for k in range(N_SNAP)]


def settings(storage=1, ring_slots=0, **kw):
    d = dict(Space=0, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
             GridScale=[1000.0, 1000.0, 250.0], Offset=[0.0, 0.0, 0.0], SaveInterval=0, BorderMode=0,
             CurvatureMode=0, MaximumSimulationTime=60.0 * 10 * (N_SNAP - 1))
    d.update(kw)
    return capi.settings_from_reference(d, storage=storage, ring_slots=ring_slots)


def seeds(n, seed):
    nz, ny, nx = GRID
    return W.uniform_seeds(n, seed, [0.0, 0.0, 0.0], [nx * 1000.0, ny * 1000.0, nz * 250.0 / 2])


def make_server(snaps, storage=1, budget=0):
    srv = capi.Server(settings(storage), N_SNAP, GRID, hbm_budget=budget)
    for k, s in enumerate(snaps):
        srv.set_snapshot(k, s)
    srv.start()
    return srv


def requests(k, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for j in range(k):
        n = int(np.exp(rng.uniform(np.log(10), np.log(3000))))
        start = float(rng.integers(0, 10 * (N_SNAP - 1))) * 60.0
        out.append(dict(seeds=seeds(n, 1000 + j), start=start, steps=int(rng.integers(5, 150)),
                        integrator=int(rng.random() < 0.8)))
    return out


def run_alone(srv, r):
    rid = srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"])
    assert srv.wait(rid, 60.0) == capi.GR_REQ_DONE
    pos, st, info = srv.result(rid)
    srv.release(rid)
    return pos, st


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 1])
def test_request_is_the_same_alone_and_in_the_mix(storage):
    snaps = field()
    reqs = requests(24, seed=storage)
    srv = make_server(snaps, storage)
    alone = [run_alone(srv, r) for r in reqs[:6]]
    # the mix: every request submitted at once from two threads
    ids = [None] * len(reqs)

    def submit(lo, hi):
        for j in range(lo, hi):
            r = reqs[j]
            ids[j] = srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"])
    th = [threading.Thread(target=submit, args=(0, 12)), threading.Thread(target=submit, args=(12, 24))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for j, rid in enumerate(ids):
        assert srv.wait(rid, 120.0) == capi.GR_REQ_DONE, j
    for j in range(6):
        pos, st, info = srv.result(ids[j])
        assert np.array_equal(st, alone[j][1]), j
        assert np.array_equal(pos, alone[j][0]), j
    stats = srv.stats()
    assert stats.completed == 6 + 24 and stats.pending == 0 and stats.active == 0
    assert stats.particle_steps > 0 and stats.windows > 0
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("w0", [0, 3])
def test_request_on_a_window_boundary_equals_a_plain_run(w0):
    snaps = field()
    sd = seeds(700, 77)
    steps = 47
    srv = make_server(snaps, storage=0)
    rid = srv.submit(sd, w0 * 600.0, steps, 1)
    assert srv.wait(rid, 60.0) == capi.GR_REQ_DONE
    pos, st, info = srv.result(rid)
    assert info.start_step == 10 * w0 and info.steps == steps
    srv.close()
    eng = capi.Engine(settings(storage=0, ring_slots=N_SNAP, MaximumSimulationTime=60.0 * steps))
    eng.set_seeds(sd)
    for k in range(N_SNAP - w0):
        eng.load_windfield(k, snaps[w0 + k])
    eng.run(lambda k: 1 if k < N_SNAP - w0 else 0)
    ref = eng.results(volumes=False, compute=False)
    assert np.array_equal(st, ref["status"])
    assert np.array_equal(pos, ref["trajectories"][:, -1])


@pytest.mark.gpu
def test_small_budget_defers_admission_and_cancel():
    snaps = field()
    reqs = requests(12, seed=7)
    big = make_server(snaps)
    alone = [run_alone(big, r) for r in reqs]
    big.close()
    # room for about 4000 particles per pool: requests queue for the next sweep
    srv = make_server(snaps, budget=4000 * 160)
    assert srv.stats().capacity_particles < 5000
    ids = [srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"]) for r in reqs]
    extra = srv.submit(seeds(50, 9), 0.0, 100, 1)
    srv.cancel(extra)
    for j, rid in enumerate(ids):
        assert srv.wait(rid, 120.0) == capi.GR_REQ_DONE
        pos, st, _ = srv.result(rid)
        assert np.array_equal(st, alone[j][1]) and np.array_equal(pos, alone[j][0]), j
    assert srv.wait(extra, 10.0) == capi.GR_REQ_CANCELLED
    s = srv.stats()
    assert s.peak_particles <= 2 * s.capacity_particles
    # requests that all end with the field: when three or more of them are admitted in the same
    # sweep, their results outgrow the pinned staging of one window and are returned over the
    # next ones.  Which sweep admits a request depends on when the server thread sees it, so the
    # batch is submitted again (results checked every time) until that has happened.
    late = [dict(seeds=seeds(1900, 300 + j), start=0.0, steps=10_000, integrator=j % 2) for j in range(4)]
    ref = [run_alone(srv, r) for r in late]
    for attempt in range(4):
        ids = [srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"]) for r in late]
        for j, rid in enumerate(ids):
            assert srv.wait(rid, 120.0) == capi.GR_REQ_DONE
            pos, st, info = srv.result(rid)
            assert info.steps == 10 * (N_SNAP - 1)
            assert np.array_equal(st, ref[j][1]) and np.array_equal(pos, ref[j][0]), (attempt, j)
            srv.release(rid)
        if srv.stats().staged_later > 0:
            break
    assert srv.stats().staged_later > 0
    srv.close()


def test_server_rejects_unsupported_settings_without_gpu():
    with pytest.raises(capi.GraniteError, match="positions only"):
        capi.Server(settings(CurvatureMode=1), N_SNAP, GRID)
    with pytest.raises(capi.GraniteError, match="at least two snapshots"):
        capi.Server(settings(), 1, GRID)


@pytest.mark.gpu
def test_two_dimensional_field_alone_and_in_the_mix():
    grid2 = (32, 48)
    f = W.FourierField(grid2, (1000.0, 1000.0), n_modes=32, seed=8, rms=(7.0710678, 7.0710678))
    snaps = [f.snapshot(600.0 * k) for k in range(N_SNAP)]
    st = capi.settings_from_reference(dict(Space=1, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                                           GridScale=[1000.0, 1000.0], Offset=[0.0, 0.0], SaveInterval=0,
                                           BorderMode=3, MaximumSimulationTime=600.0 * (N_SNAP - 1)), storage=2)
    srv = capi.Server(st, N_SNAP, grid2)
    for k, s in enumerate(snaps):
        srv.set_snapshot(k, s)
    srv.start()
    rng = np.random.default_rng(3)
    reqs = [dict(seeds=W.uniform_seeds(int(rng.integers(20, 800)), 50 + j, [0.0, 0.0], [48000.0, 32000.0]),
                 start=float(rng.integers(0, 100)) * 60.0, steps=int(rng.integers(5, 120)), integrator=j % 2)
            for j in range(10)]
    alone = [run_alone(srv, r) for r in reqs[:3]]
    ids = [srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"]) for r in reqs]
    for j, rid in enumerate(ids):
        assert srv.wait(rid, 120.0) == capi.GR_REQ_DONE
        if j < 3:
            pos, status, _ = srv.result(rid)
            assert np.array_equal(status, alone[j][1]) and np.array_equal(pos, alone[j][0]), j
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 1])
def test_mid_window_requests_match_the_float32_oracle(storage):
    """Requests that start inside a window (start times off the step grid too, rounded down to
    it), Euler and RK4, submitted together: each result against the float32 oracle run whose
    particles join the field's clock at the request's start step (the time and window driver of
    TrajectoryIntegrator.tpp:778-995, entered mid-run), on the field as the ring stores it."""
    from oracle import oracle as orc
    snaps = field()
    name = {0: "f32", 1: "bf16"}[storage]
    stored = [[W.round_storage(p, name) for p in s] for s in snaps]
    reqs = [dict(seeds=seeds(300 + 50 * j, 500 + j), start=60.0 * k0 + off, steps=steps, integrator=integ)
            for j, (k0, off, steps, integ) in enumerate([(3, 0.0, 41, 1), (17, 12.5, 60, 1), (26, 59.0, 33, 0),
                                                         (44, 30.0, 70, 0), (58, 1.0, 55, 1), (71, 45.0, 49, 0)])]
    srv = make_server(snaps, storage)
    ids = [srv.submit(r["seeds"], r["start"], r["steps"], r["integrator"]) for r in reqs]
    for j, (rid, r) in enumerate(zip(ids, reqs)):
        assert srv.wait(rid, 120.0) == capi.GR_REQ_DONE, j
        pos, st, info = srv.result(rid)
        k0 = int(np.floor(r["start"] / 60.0))
        assert info.start_step == k0 and info.steps == r["steps"]
        assert k0 % 10 != 0, "the start must fall inside a window"
        base = dict(Space=0, Integrator=r["integrator"], WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=[1000.0, 1000.0, 250.0], Offset=[0.0, 0.0, 0.0], SaveInterval=0, BorderMode=0,
                    CurvatureMode=0, MaximumSimulationTime=60.0 * 10 * (N_SNAP - 1))
        ref = orc.run(orc.settings(**base), orc.Inputs(wind=stored, seeds=r["seeds"]), precision="f32",
                      start_step=k0, step_limit=k0 + r["steps"])
        assert np.array_equal(st, ref["status"]), j
        assert np.array_equal(pos, ref["trajectories"][:, -1]), j
    srv.close()
