"""Batching and serving with pygranite's own objects.

`BatchIntegrator` and `TrajectoryServer` take an `IntegratorSettings` and a `DataLoader`
like `TrajectoryIntegrator(settings, loader, set)` does, and run on the engine's batch graph
(gr_batch_*) and request server (gr_server_*).  Neither exists in the reference, which
integrates one seed set per `TrajectoryIntegrator`.

Both read every snapshot they need from the loader up front (`windfield()` for the current
snapshot, `step()` to advance), so the whole field is resident on the device (batching) or in
pinned host memory (serving).
"""
from __future__ import annotations

import numpy as np

from . import capi

_ENUMS = ("Space", "Integrator", "WindfieldMode", "ConstantsMode", "AdditionalVolumeMode", "UpLiftMode",
          "BorderMode", "CurvatureMode", "AbortMode")


def c_settings(s, **extra) -> capi.Settings:
    """gr_settings from a pygranite IntegratorSettings, engine options included."""
    d = {k: int(getattr(s, k)) for k in _ENUMS}
    d.update(Reverse=bool(s.Reverse), MinimumAliveParticles=int(s.MinimumAliveParticles),
             SphereRadius=float(s.SphereRadius), DeltaT=float(s.DeltaT), DataTimeDistance=float(s.DataTimeDistance),
             MaximumLength=float(s.MaximumLength), MaximumSimulationTime=float(s.MaximumSimulationTime),
             GridScale=[float(x) for x in s.GridScale], Offset=[float(x) for x in s.Offset],
             SaveInterval=int(s.SaveInterval))
    opts = dict(storage=int(s.WindStorage), time_mode=1 if s.Float64Time else 0,
                compensated=1 if s.CompensatedPositions else 0, ring_slots=int(s.RingSlots),
                steps_per_launch=int(s.StepsPerLaunch), sort_interval=int(s.SortInterval),
                block_size=int(s.BlockSize), device=int(s.Device), layout=int(s.WindLayout),
                filter_weights=1 if s.ReferenceFilter else 0)
    opts.update(extra)
    return capi.settings_from_reference(d, **opts)


def _points(seeds):
    """Seed positions (n, dim) float32 from a TrajectorySet or an array."""
    if hasattr(seeds, "trajectories"):
        return np.ascontiguousarray(seeds.trajectories()[:, -1], np.float32)
    return np.ascontiguousarray(seeds, np.float32)


def _pull_snapshots(loader, needed):
    """Snapshots 0 .. needed-1 from a DataLoader (fewer if it runs dry), with their volumes."""
    wind, vols = [list(loader.windfield())], [dict(loader.additionalVolumes())]
    while len(wind) < needed and loader.step():
        wind.append(list(loader.windfield()))
        vols.append(dict(loader.additionalVolumes()))
    return wind, vols


class SetResult:
    """Results of one seed set of a batch; accessors named as TrajectorySet's."""

    def __init__(self, traj, status, lengths, tc, curv, vols, cmps):
        self._traj, self._status, self._lengths, self._tc = traj, status, lengths, tc
        self._curv, self._vols, self._cmps = curv, vols, cmps

    def trajectories(self):
        """(n, records, dim): records after the set's lifetime repeat its last state."""
        return self._traj

    def finalPositions(self):
        return self._traj[:, -1]

    def abortReasons(self):
        return self._status

    def individualLengths(self):
        return self._lengths

    def totalCurvatures(self):
        return self._tc

    def curvatures(self):
        return self._curv

    def volumeInfo(self, name):
        return self._vols[name]

    def computeInfo(self, index):
        return self._cmps[index]


class BatchIntegrator:
    """Seed sets of uneven size and lifetime (integrator steps) on one windfield, advanced
    together and replayed as one CUDA graph.  Set j ends exactly where
    TrajectoryIntegrator(settings with MaximumSimulationTime = lifetimes[j] * DeltaT, loader,
    sets[j]).compute() ends.  Per-particle constants and uplift are not supported here."""

    def __init__(self, settings, loader, sets, lifetimes):
        if int(settings.ConstantsMode) or int(settings.UpLiftMode):
            raise NotImplementedError("per-particle constants and uplift are not batched")
        pts = [_points(s) for s in sets]
        life = [int(x) for x in lifetimes]
        if len(pts) != len(life) or not pts:
            raise ValueError("one lifetime per seed set is needed")
        self.settings, self.counts = settings, [len(p) for p in pts]
        seeds = np.concatenate(pts)
        lifes = np.concatenate([np.full(n, L, np.int32) for n, L in zip(self.counts, life)])
        plan = c_settings(settings)
        plan.maximum_simulation_time = min(plan.maximum_simulation_time, max(life) * float(settings.DeltaT))
        info, _ = capi.plan(plan, with_steps=False)
        needed = info.windows + 1 if int(settings.WindfieldMode) == 1 else 1
        wind, vols = _pull_snapshots(loader, needed)
        e = self.engine = capi.Engine(c_settings(settings, ring_slots=max(3, len(wind))))
        e.set_seeds(seeds)
        e.set_lifetimes(lifes)
        for k, w in enumerate(wind):
            e.load_windfield(k, w)
        vm = int(settings.AdditionalVolumeMode)
        self.vol_names = list(vols[0].keys())[:8] if vm else []
        for k, v in enumerate((vols if vm == 2 else vols[:1]) if self.vol_names else []):
            for j, name in enumerate(self.vol_names):
                e.load_volume(k, j, v[name])
        topo = np.asarray(settings.Topography, np.float32)
        if topo.size:
            e.set_topography(topo)
        for j, code in enumerate(settings.AdditionalCompute):
            e.compile_expression(j, code, self.vol_names, [])
        self._batch = None

    def tune(self, trial_steps=40):
        """Autotunes layout, block size, sort interval and grid waves (gr_tune)."""
        return self.engine.tune(trial_steps)

    def compute(self):
        """Runs (the first call captures the graph, later calls replay it); one SetResult per set."""
        if self._batch is None:
            self._batch = capi.Batch([self.engine])
        self._batch.run()
        out = self.engine.results()
        res, off = [], 0
        for n in self.counts:
            sl = slice(off, off + n)
            vols = {name: out["volume_info"][j][sl] for j, name in enumerate(self.vol_names)}
            res.append(SetResult(out["trajectories"][sl], out["status"][sl], out["lengths"][sl],
                                 out["total_curvature"][sl], out["curvatures"][sl], vols,
                                 [c[sl] for c in out["compute_info"]]))
            off += n
        return res

    def close(self):
        if self._batch is not None:
            self._batch.close()
            self._batch = None
        self.engine.close()


class TrajectoryServer:
    """Trajectory requests served with continuous batching over the loader's whole field (every
    snapshot it delivers, kept packed in pinned host memory and streamed through a 4-slot device
    ring).  Positions only: no curvature, volumes, constants, uplift or length abort."""

    def __init__(self, settings, loader, hbm_budget=0, max_snapshots=None):
        self.settings = settings
        wind, _ = _pull_snapshots(loader, max_snapshots or (1 << 62))
        self.server = capi.Server(c_settings(settings), len(wind), np.shape(wind[0][0]), hbm_budget=hbm_budget)
        for k, w in enumerate(wind):
            self.server.set_snapshot(k, w)
        self.server.start()

    def submit(self, seeds, start_time, steps, integrator=None):
        """Request id; integrator defaults to settings.Integrator (0 Euler, 1 RK4)."""
        integ = int(self.settings.Integrator) if integrator is None else int(integrator)
        return self.server.submit(_points(seeds), start_time, steps, integ)

    def wait(self, rid, timeout=-1.0):
        return self.server.wait(rid, timeout)

    def result(self, rid):
        """(final positions (n, dim), abort reasons (n)) of a finished request."""
        pos, st, _ = self.server.result(rid)
        return pos, st

    def info(self, rid):
        return self.server.info(rid)

    def cancel(self, rid):
        self.server.cancel(rid)

    def release(self, rid):
        self.server.release(rid)

    def stats(self):
        return self.server.stats()

    def close(self):
        self.server.close()
