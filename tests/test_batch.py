"""Batching: seed sets of uneven size and lifetime in one graph-captured run.

A set with lifetime L in a batch must end exactly where a plain run of that set alone ends
with MaximumSimulationTime = L * DeltaT: per-particle arithmetic, the step schedule (a prefix
of the longer run's) and the final record are the same, so final positions and abort codes
are compared bit for bit.  Host-side parts (the workload generator, prefix property of the
schedule) run without a GPU.
"""
import numpy as np
import pytest

from pygranite_b200 import capi
from pygranite_b200 import workloads as W

SMALL = dict(n_sets=10, grid3=(16, 32, 32), grid2=(32, 64), n_min=20, n_max=3000, life_min=5, life_max=120,
             frac3d=0.6, seed=3)


def test_batch_sets_statistics():
    sets = W.batch_sets(512, seed=0)
    n = np.array([s["n"] for s in sets])
    life = np.array([s["life"] for s in sets])
    assert n.min() >= 100 and n.max() <= 200_000 and life.min() >= 100 and life.max() <= 5000
    # log-uniform counts: the median sits near the geometric mean of the bounds
    assert 2000 < np.median(n) < 10000
    assert 0.6 < np.mean([s["dim"] == 3 for s in sets]) < 0.8
    assert sets == W.batch_sets(512, seed=0)


@pytest.mark.parametrize("life", [1, 7, 10, 23, 120])
def test_schedule_of_a_shorter_run_is_a_prefix(life):
    w = W.BatchWorkload(**SMALL)
    full = capi.settings_from_reference(dict(w.settings(3), MaximumSimulationTime=60.0 * 1000))
    short = capi.settings_from_reference(dict(w.settings(3), MaximumSimulationTime=60.0 * life))
    fi, fp = capi.plan(full)
    si, sp = capi.plan(short)
    assert si.steps == life
    for k in ("window", "flags", "weights"):
        assert np.array_equal(sp[k], fp[k][:life])


def group_engine(w, dim, storage=0, **extra):
    seeds, lifes, spans = w.group(dim)
    eng = capi.Engine(capi.settings_from_reference(w.settings(dim), ring_slots=w.n_snapshots, storage=storage,
                                                   **extra))
    eng.set_seeds(seeds)
    eng.set_lifetimes(lifes)
    for k in range(w.n_snapshots):
        eng.load_windfield(k, w.snapshot(dim, k))
    return eng, spans


def plain_run(w, j, storage=0, save_interval=0):
    """One set alone, MaximumSimulationTime = lifetime * DeltaT."""
    s = w.sets[j]
    st = dict(w.settings(s["dim"]), MaximumSimulationTime=60.0 * s["life"], SaveInterval=save_interval)
    eng = capi.Engine(capi.settings_from_reference(st, ring_slots=w.n_snapshots, storage=storage))
    eng.set_seeds(w.seeds(j))
    for k in range(w.n_snapshots):
        eng.load_windfield(k, w.snapshot(s["dim"], k))
    eng.run(lambda k: 1 if k < w.n_snapshots else 0)
    out = eng.results(volumes=False, compute=False)
    out["info"] = eng.info()
    eng.close()
    return out


def plain_final(w, j, storage=0):
    out = plain_run(w, j, storage)
    return out["trajectories"][:, -1], out["status"], out["info"]


def finals(eng):
    return eng.final_positions(), eng.results(volumes=False, compute=False)["status"]


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 1])
def test_batch_matches_plain_run_per_set(storage):
    w = W.BatchWorkload(**SMALL)
    e3, spans3 = group_engine(w, 3, storage)
    e2, spans2 = group_engine(w, 2, storage)
    batch = capi.Batch([e3, e2])
    batch.run()
    first = {d: finals(e) for d, e in ((3, e3), (2, e2))}
    st = batch.stats()
    assert st.captures == 1 and st.replays == 1 and st.kernel_launches > 0 and st.nodes > st.kernel_launches
    ps_plain = 0
    for dim, eng, spans in ((3, e3, spans3), (2, e2, spans2)):
        pos, status = first[dim]
        for j, off, cnt in spans:
            ref_pos, ref_status, info = plain_final(w, j, storage)
            ps_plain += info.particle_steps
            assert np.array_equal(status[off:off + cnt], ref_status), j
            assert np.array_equal(pos[off:off + cnt], ref_pos), j
    assert st.particle_steps == ps_plain
    # a replay gives the same results and does not capture again
    batch.run()
    assert batch.stats().captures == 1 and batch.stats().replays == 2
    for d, e in ((3, e3), (2, e2)):
        pos, status = finals(e)
        assert np.array_equal(pos, first[d][0]) and np.array_equal(status, first[d][1])
    batch.close()


@pytest.mark.gpu
def test_batch_recaptures_after_changes_and_tuning_keeps_results():
    w = W.BatchWorkload(**SMALL)
    e3, spans3 = group_engine(w, 3)
    batch = capi.Batch([e3])
    batch.run()
    ref = finals(e3)
    r = e3.tune(trial_steps=20)
    assert r.trials >= 6 and r.particle_steps_per_s > 0
    assert r.block_size in (64, 128, 256) and r.sort_interval in (1, 2, 4, 8) and r.grid_waves in (1, 2, 4)
    batch.run()
    assert batch.stats().captures == 2
    pos, status = finals(e3)
    assert np.array_equal(pos, ref[0]) and np.array_equal(status, ref[1])
    # new seeds: the graph is rebuilt and follows them
    seeds, lifes, _ = w.group(3)
    e3.set_seeds(seeds[::-1].copy())
    e3.set_lifetimes(lifes[::-1].copy())
    batch.run()
    assert batch.stats().captures == 3
    pos2, status2 = finals(e3)
    assert np.array_equal(pos2[::-1], ref[0]) and np.array_equal(status2[::-1], ref[1])
    batch.close()


@pytest.mark.gpu
def test_lifetimes_in_a_plain_run_and_records_after_the_lifetime():
    w = W.BatchWorkload(**dict(SMALL, n_sets=4))
    e3, spans = group_engine(w, 3, save_interval=10, sort_interval=2)
    e3.run(lambda k: 1 if k < w.n_snapshots else 0)
    out = e3.results(volumes=False, compute=False)
    info = e3.info()
    assert info.steps == max(w.sets[j]["life"] for j, _, _ in spans)
    for j, off, cnt in spans:
        ref = plain_run(w, j, save_interval=10)
        ref_pos, ref_status, _ = plain_final(w, j)
        traj = out["trajectories"][off:off + cnt]
        lp = ref["trajectories"].shape[1]
        assert np.array_equal(out["status"][off:off + cnt], ref_status)
        # the records the set's own run writes are the same ...
        assert np.array_equal(traj[:, :lp], ref["trajectories"]), j
        # ... and every later record repeats the state after its lifetime
        for r in range(lp, info.records):
            assert np.array_equal(traj[:, r], ref_pos), (j, r)


@pytest.mark.gpu
@pytest.mark.parametrize("storage", [0, 1])
def test_batched_sets_match_the_float32_oracle(storage):
    """Each set of the batch against the float32 oracle run of that set alone
    (MaximumSimulationTime = lifetime * DeltaT, TrajectoryIntegrator.tpp:778-995), on the
    field as the ring stores it (BF16: the float32 snapshots rounded to nearest even)."""
    from oracle import oracle as orc
    w = W.BatchWorkload(**SMALL)
    name = {0: "f32", 1: "bf16"}[storage]
    engines = {d: group_engine(w, d, storage) for d in (3, 2)}
    batch = capi.Batch([engines[3][0], engines[2][0]])
    batch.run()
    checked = {3: set(), 2: set()}
    for dim, (eng, spans) in engines.items():
        pos, status = finals(eng)
        for j, off, cnt in spans:
            life = w.sets[j]["life"]
            snaps = [[W.round_storage(p, name) for p in w.snapshot(dim, k)] for k in range(life // 10 + 2)]
            st = orc.settings(**dict(w.settings(dim), MaximumSimulationTime=60.0 * life))
            ref = orc.run(st, orc.Inputs(wind=snaps, seeds=w.seeds(j)), precision="f32")
            assert np.array_equal(status[off:off + cnt], ref["status"]), (dim, j)
            assert np.array_equal(pos[off:off + cnt], ref["trajectories"][:, -1]), (dim, j)
            checked[dim].add(life)
    batch.close()
    # sets of different lifetimes on each field
    assert len(checked[3]) >= 4 and len(checked[2]) >= 3, checked
