#!/usr/bin/env python
"""particle-steps/s of the trajectory step path on B200.

Workload (one `step` of this benchmark = one full simulation of the plain 3D RK4 FP32
configuration): u,v,w on a 192x192x64 grid (1 km, 1 km, 250 m) from seeded Fourier modes,
600 s snapshots, 1,000,000 particles in the lower half of the domain, h = 60 s for 2,000 RK4
steps, records every 10 steps, TotalCurvature, one constant temperature volume and the
expression sqrt(u*u+v*v)*T.  201 snapshots so that 2,000 steps fit (48 x 600 s would end the
run after 470 steps; the spacing is unchanged).  A particle-step is one alive particle
advanced by one integrator step.

value : device-resident — every snapshot already packed in HBM (ring of 201 slots), seeds
        on the device; timed with the engine's CUDA events (max over ranks).
e2e   : the pygranite API, TrajectoryIntegrator(settings, loader, TrajectorySet(seeds))
        .compute(), with the loader serving host snapshots into a 3-slot device ring; every
        H2D upload and the D2H copy of the records are inside the timed region.  Loader arrays
        and results in page-locked host memory (pinned_empty, PinnedResults); the defaults
        (pageable numpy both ways) are reported beside it as e2e.pageable.
--impl reference : the reference has no CPU implementation of the path; the CPU oracle port
        (float64, OpenMP on all host cores) runs bounded samples of the same workload.
"""
import argparse
import gc
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# algorithmic bytes per particle-step of the plain 3D configuration: 4 stages x 2 snapshots x
# 3 components x 8 corners x element bytes, + 8 corners x 4 B of the volume, + position read /
# write and status (28 B), + previous position and curvature (20 B), + records every 10 steps
BYTES_PER_PARTICLE_STEP = {
    "f32": 850, "bf16": 466, "f16": 466,
}
WORKLOAD = "trajectory-3d-rk4-curvature-volume-expr"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--particles", type=int, default=1_000_000)
    p.add_argument("--sim-steps", type=int, default=2000)
    p.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"])
    p.add_argument("--steps-per-launch", type=int, default=0)
    p.add_argument("--sort-interval", type=int, default=8,
                   help="launches between compaction / Morton re-sorts of the live particles (0 = off)")
    p.add_argument("--layout", type=int, default=0, help="0: window-pair wind layout, 1: ring slots")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-native", action="store_true", help="skip the native-loader run")
    p.add_argument("--cpu-particles", type=int, default=1_000_000)
    p.add_argument("--cpu-steps", type=int, default=200)
    p.add_argument("--ref-steps", type=int, default=20, help="reference arm: steps of the workload's prefix")
    p.add_argument("--parity-sample", type=int, default=2000,
                   help="particles of the timed run checked against the float32 / float64 oracle (0 = off)")
    p.add_argument("--no-forms", action="store_true", help="plain workload: skip the batch / serve / precision forms")
    p.add_argument("--workload", default="plain", choices=["plain", "batch", "serve", "precision"],
                   help="plain: the 3D RK4 configuration; batch: 512 seed sets of uneven size and lifetime; "
                        "serve: a Poisson stream of requests on the request server")
    p.add_argument("--prec-particles", type=int, default=4_000_000)
    p.add_argument("--prec-steps", type=int, default=5000)
    p.add_argument("--prec-sample", type=int, default=256, help="particles checked against the float64 oracle")
    p.add_argument("--serve-rate", type=float, default=200.0, help="requests per second")
    p.add_argument("--serve-seconds", type=float, default=60.0, help="length of the arrival stream")
    p.add_argument("--serve-storage", default="bf16", choices=["f32", "bf16", "f16"])
    p.add_argument("--batch-storage", default="bf16", choices=["f32", "bf16", "f16"])
    p.add_argument("--batch-sets", type=int, default=512)
    p.add_argument("--tune-steps", type=int, default=40, help="steps per autotuner trial (0 = no tuning)")
    p.add_argument("--batch-life-max", type=int, default=5000, help="longest lifetime of the batching workload")
    p.add_argument("--no-plain", action="store_true", help="batch: skip the one-run-per-set baseline")
    p.add_argument("--no-acc", action="store_true", help="batch: skip the float64 accuracy sample")
    p.add_argument("--serve-budget-gb", type=float, default=0.0, help="serve: HBM budget (0 = 1/4 of free)")
    p.add_argument("--serve-acc", type=int, default=2, help="serve: requests checked against the float64 oracle")
    p.add_argument("--acc-life", type=int, default=500,
                   help="accuracy sample: sets with at most this lifetime are checked against the float64 oracle")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload(args, rank):
    from pygranite_b200 import workloads as W
    n_snap = args.sim_steps // 10 + 1
    settings, src, seeds = W.config2(n_particles=args.particles, n_snapshots=n_snap, steps=args.sim_steps,
                                     seed=rank)
    return settings, src, seeds


class ClockSampler:
    """nvidia-smi sampling during the timed region (clock, power, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def combine_ranks(dist, time_ms, particle_steps, device):
    """Whole-job figures across ranks: the slowest rank's device time and the summed work
    (replicas: every rank integrates its own particle set, no data-path collective)."""
    if dist is None:
        return time_ms, particle_steps
    import torch
    t = torch.tensor([float(time_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(particle_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_kernel_profile(storage):
    """Per-particle-step figures of the step kernel from the committed ncu summary
    (profiles/advance_kernel_counters.json): DRAM bytes and warp instructions per
    particle-step, with the capture they come from."""
    path = os.path.join(ROOT, "profiles", "advance_kernel_counters.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(storage)


def cpu_baseline(args, settings, src, seeds, threads=None):
    """float64 oracle (OpenMP) on a bounded sample of the same workload."""
    from oracle import oracle as orc
    n = min(args.cpu_particles, seeds.shape[0])
    threads = threads or (os.cpu_count() or 1)
    data = orc.Inputs(wind=src.wind[: args.cpu_steps // 10 + 2], seeds=seeds[:n], volumes=src.volumes)
    r = orc.run(orc.settings(**settings), data, precision="f64", threads=threads, step_limit=args.cpu_steps)
    value = r["particle_steps"] / max(r["seconds"], 1e-9)
    return dict(value=value, unit="particle-steps/s", cores=threads, kind="port",
                sample=f"{n} particles x {r['steps']} RK4 steps of the same workload (float64 oracle)")


CELL_3D = np.array([1000.0, 1000.0, 250.0])


def sample_ids(n, m):
    """m particle ids spread evenly over the seed array."""
    return np.unique(np.linspace(0, n - 1, min(m, n)).round().astype(np.int64))


def plain_oracle(settings, src, seeds, ids):
    """float32 and float64 oracle runs of the sampled particles on the same snapshots (the
    checker; particles are independent, so a subset runs exactly as inside the full set)."""
    from oracle import oracle as orc
    data = orc.Inputs(wind=src.wind, seeds=seeds[ids], volumes=src.volumes)
    th = os.cpu_count() or 1
    return (orc.run(orc.settings(**settings), data, precision="f32", threads=th),
            orc.run(orc.settings(**settings), data, precision="f64", threads=th))


def check_plain(got, ref32, ref64):
    """got: the sampled rows of a run (trajectories, status, total_curvature, T samples,
    expression values).  Bit-for-bit comparison with the float32 oracle, and the position
    error in grid cells against the float64 oracle after 100 and 400 steps (records 10, 40) and at
    the end, over particles not yet aborted in either run at that record."""
    traj, status = got["trajectories"], got["status"]
    checks = {
        "positions": bool(np.array_equal(traj, ref32["trajectories"])),
        "status": bool(np.array_equal(status, ref32["status"])),
        "total_curvature": bool(np.array_equal(got["total_curvature"], ref32["total_curvature"])),
        "volume_T": bool(np.array_equal(got["volume"], ref32["volume_info"]["T"])),
        "expression": bool(np.array_equal(got["expression"], ref32["compute_info"][0])),
    }
    bad = np.any(traj != ref32["trajectories"], axis=(1, 2)) | (status != ref32["status"])
    L = traj.shape[1]
    f64 = {}
    for rec in sorted({min(10, L - 1), min(40, L - 1), L - 1}):
        k = 10 * rec
        live = ((ref64["step_of_abort"] < 0) | (ref64["step_of_abort"] >= k)) & \
               ((ref32["step_of_abort"] < 0) | (ref32["step_of_abort"] >= k))
        d = (np.abs(traj[live, rec].astype(np.float64) - ref64["trajectories"][live, rec]) / CELL_3D).max(axis=1)
        f64[f"after_{k}_steps"] = {"particles": int(d.size),
                                   "cell_rms": float(np.sqrt(np.mean(d ** 2))) if d.size else None,
                                   "cell_p50": float(np.median(d)) if d.size else None,
                                   "cell_p99": float(np.percentile(d, 99)) if d.size else None,
                                   "cell_max": float(d.max()) if d.size else None}
    return {"f32_bitexact": all(checks.values()), "checks": checks, "sample": int(traj.shape[0]), "records": int(L),
            "mismatched_particles": int(bad.sum()), "status_vs_f64_differ": int(np.sum(status != ref64["status"])),
            "f64": f64}


def plain_config(args, world):
    """The `config` object of the plain workload, the same in both arms."""
    n_snap = args.sim_steps // 10 + 1
    return {"workload": WORKLOAD, "particles_per_gpu": args.particles, "sim_steps": args.sim_steps,
            "snapshots": n_snap, "grid": [192, 192, 64], "storage": args.storage,
            "parallelism": f"replicas{world}",
            "l2": f"inputs larger than L2 ({n_snap} snapshots, {n_snap * 192 * 192 * 64 * 16 / 1e9:.1f} GB ring)",
            "records_every": 10, "sort_interval": args.sort_interval, "steps_per_launch": args.steps_per_launch,
            "wind_layout": ["window-pair", "ring"][args.layout]}


def reference_gpu_available():
    from oracle.ref_harness import refrun
    return refrun.available()


def run_reference(args):
    """The reference's own implementation of the path: its `integrate` kernel, instantiated
    unmodified from its sources (oracle/_ref, built by oracle/ref_harness), run by a host loop
    that restates its computeLoop_ (one launch, one synchronisation and the record copies per
    step, snapshots uploaded between windows) on a bounded prefix of the same workload.  Headline:
    the launch shape as shipped (TrajectoryIntegrator.tpp:790-796 swaps the arguments of sdiv, so
    one 512-thread block does all the work); beside it the same with BLOCKS = ceil(N / THREADS).
    The float64 CPU oracle (OpenMP) is reported as cpu_baseline.  Without the built kernel the
    CPU oracle is the value."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from pygranite_b200 import workloads as W
    prefix = args.ref_steps
    n_snap = max(prefix, args.cpu_steps) // 10 + 3
    settings, src, seeds = W.config2(n_particles=args.particles, n_snapshots=n_snap, steps=args.sim_steps, seed=0)
    cb = cpu_baseline(args, settings, src, seeds)
    line = {"impl": "reference", "metric": "particle-steps/s", "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Fourier-mode field)",
            "config": plain_config(args, 1), "cpu_baseline": cb}
    if not reference_gpu_available():
        line.update(value=cb["value"], dtype="f64", ms_per_step=None,
                    reference_gpu={"unavailable": "oracle/_ref/libref_integrate.so not built (needs the reference's "
                                                  "sources: make -C oracle/ref_harness REF=<checkout>)"},
                    e2e={"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return 0
    from oracle.ref_harness import refrun
    vol = src.volumes[0]["T"]
    out = {}
    for fixed in (False, True):
        ms = ps = h2d = d2h = 0.0
        for k in range(args.warmup + args.steps):
            r = refrun.run(settings, src.wind, seeds, volume=vol, blocks_fixed=fixed, step_limit=prefix,
                           count_steps=True)
            if k >= args.warmup:
                ms += r["loop_ms"]
                ps += r["particle_steps"]
                h2d += r["h2d_bytes"]
                d2h += r["d2h_bytes"]
        out["blocks_fixed" if fixed else "as_shipped"] = {
            "value": ps / (ms / 1e3), "unit": "particle-steps/s", "ms_per_step": ms / args.steps,
            "launch": f"{r['blocks']} x {r['threads']} threads", "steps": int(r["steps"]),
            "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps)}
    ship = out["as_shipped"]
    line.update(value=ship["value"], ms_per_step=ship["ms_per_step"],
                reference_gpu=dict(out, sample=f"{args.particles} particles x the first {prefix} RK4 steps of the "
                                               "workload; wall clock of the step loop (launch, synchronise, record "
                                               "copies every 10 steps, snapshot uploads between windows)"),
                e2e={"value": ship["value"], "unit": "particle-steps/s",
                     "h2d_bytes_per_step": ship["h2d_bytes_per_step"],
                     "d2h_bytes_per_step": ship["d2h_bytes_per_step"]})
    print(json.dumps(line), flush=True)
    return 0


# algorithmic bytes per particle-step of plain RK4 with the final record only, per
# (dimension, storage): 4 stages x 2 snapshots x components x corners x element bytes
# + position read / write + status
RK4_FINAL_BYTES = {(3, "f32"): 796, (3, "bf16"): 412, (3, "f16"): 412,
                   (2, "f32"): 276, (2, "bf16"): 148, (2, "f16"): 148}
BATCH_WORKLOAD = "batch-512-sets-3d-2d-rk4"


def _cell_err(got, got_st, ref, ref_st, cell):
    both = (ref_st == 0) & (got_st == 0)
    d = (np.abs(np.asarray(got, np.float64) - ref) / cell).max(axis=1)[both]
    return d, int(np.sum(ref_st != got_st))


def _summ(d):
    d = np.concatenate(d) if d else np.zeros(0)
    if not d.size:
        return {"particles": 0}
    return {"particles": int(d.size), "cell_rms": float(np.sqrt(np.mean(d ** 2))),
            "cell_p99": float(np.percentile(d, 99)), "cell_max": float(d.max())}


def batch_accuracy(w, storage, sample, batch_final, plain_final, horizon):
    """Final-position error in grid cells against the float64 oracle on sampled particles.

    sample[dim] = [(set, count)]; batch_final / plain_final[(dim, horizon_key)][set] =
    (positions, status) of the batched run and of the float32 plain run.  Two horizons: a
    fixed one (`horizon` steps, every sampled set) and each set's own lifetime.  Errors are
    taken over particles alive in both runs; differing abort codes are counted.  Over long
    horizons this 3D field amplifies any rounding (float32 and float64 arithmetic part by
    cells after a few hundred steps), so the float32 plain path's own error is reported
    beside the batched one; "same_field" compares with a float64 run on the stored
    (rounded) field."""
    from oracle import oracle as orc
    from pygranite_b200 import workloads as W
    out = {}
    for dim in sorted(sample):
        cell = np.array([1000.0, 1000.0, 250.0][:dim])
        res = {}
        for hkey in ("fixed", "lifetime"):
            acc = {"batched_vs_f64": [], "batched_vs_f64_same_field": [], "plain_f32_vs_f64": []}
            mism = {k: 0 for k in acc}
            steps = []
            for j, m in sample[dim]:
                life = w.sets[j]["life"] if hkey == "lifetime" else horizon
                if (dim, hkey) not in batch_final or j not in batch_final[(dim, hkey)]:
                    continue
                seeds = w.seeds(j)[:m]
                snaps = [w.snapshot(dim, k) for k in range(life // 10 + 2)]
                st = orc.settings(**dict(w.settings(dim), MaximumSimulationTime=60.0 * life))
                ref = orc.run(st, orc.Inputs(wind=snaps, seeds=seeds), precision="f64")
                rsn = [[W.round_storage(p, storage) for p in sn] for sn in snaps]
                ref_s = orc.run(st, orc.Inputs(wind=rsn, seeds=seeds), precision="f64")
                bp, bs = batch_final[(dim, hkey)][j]
                pp, ps_ = plain_final[(dim, hkey)][j]
                for key, (gp, gs, r) in {"batched_vs_f64": (bp, bs, ref),
                                         "batched_vs_f64_same_field": (bp, bs, ref_s),
                                         "plain_f32_vs_f64": (pp, ps_, ref)}.items():
                    d, mm = _cell_err(gp[:m], gs[:m], r["trajectories"][:, -1], r["status"], cell)
                    acc[key].append(d)
                    mism[key] += mm
                steps.append(life)
            res[hkey] = {"steps": steps if hkey == "lifetime" else horizon, "sets": len(steps)}
            for key in acc:
                res[hkey][key] = dict(_summ(acc[key]), status_mismatch=mism[key])
        out[f"{dim}d"] = res
    return out


def run_batch(args, world, rank, local, pg_dist, storages=None):
    """512 seed sets batched in one graph per wind storage (16-bit by default) vs one plain
    FP32 run per set.  storages: the batched storages to measure (default: --batch-storage);
    the first one is the headline."""
    import torch
    from pygranite_b200 import capi
    from pygranite_b200 import workloads as W

    storages = list(storages or [args.batch_storage])
    w = W.BatchWorkload(n_sets=args.batch_sets, life_max=args.batch_life_max, seed=rank)
    n_snap = w.n_snapshots
    code = {"f32": 0, "bf16": 1, "f16": 2}
    groups, eng_b, eng_p, spans = {}, {bst: {} for bst in storages}, {}, {}
    for dim in (3, 2):
        seeds, lifes, sp = w.group(dim)
        if not sp:
            continue
        groups[dim] = (seeds, lifes)
        spans[dim] = sp
        for bst in storages:
            e = capi.Engine(capi.settings_from_reference(w.settings(dim), ring_slots=n_snap, storage=code[bst],
                                                         device=local, sort_interval=args.sort_interval))
            e.set_seeds(seeds)
            e.set_lifetimes(lifes)
            eng_b[bst][dim] = e
        if not args.no_plain:
            eng_p[dim] = capi.Engine(capi.settings_from_reference(w.settings(dim), ring_slots=n_snap, storage=0,
                                                                  device=local, sort_interval=args.sort_interval))
    t0 = time.perf_counter()
    for k in range(n_snap):
        for dim in groups:
            snap = w.snapshot(dim, k)
            for bst in storages:
                eng_b[bst][dim].load_windfield(k, snap)
            if dim in eng_p:
                eng_p[dim].load_windfield(k, snap)
    load_s = time.perf_counter() - t0
    resident = lambda s: 1 if s < n_snap else 0  # noqa: E731
    loc = {j: (d, off, cnt) for d in spans for j, off, cnt in spans[d]}
    per_set, horizon = 64, 100
    sample = {d: [(j, min(per_set, cnt)) for j, off, cnt in spans[d] if w.sets[j]["life"] <= args.acc_life][:6]
              for d in spans}
    sampled = {j for d in sample for j, _ in sample[d]}

    results = {}
    for bst in storages:
        eb = eng_b[bst]
        # ---- autotuner, then one graph over both field groups
        tuned = {}
        for dim, e in eb.items():
            if args.tune_steps > 0:
                r = e.tune(trial_steps=args.tune_steps)
                tuned[f"{dim}d"] = {"layout": ["window-pair", "ring"][r.layout], "block_size": r.block_size,
                                    "sort_interval": r.sort_interval, "grid_waves": r.grid_waves,
                                    "trials": r.trials, "trial_rate": r.particle_steps_per_s}
        batch = capi.Batch([eb[d] for d in sorted(eb)])
        for _ in range(max(1, args.warmup)):
            batch.run()
        torch.cuda.synchronize()
        if pg_dist:
            pg_dist.barrier()
        sampler = ClockSampler(local)
        sampler.start()
        time.sleep(0.3)
        g_ms, g_ps, ps_dim = 0.0, 0, {d: 0 for d in eb}
        for _ in range(args.steps):
            batch.run()
            st = batch.stats()
            g_ms += st.graph_ms
            g_ps += st.particle_steps
            for d, e in eb.items():
                ps_dim[d] += e.stats().particle_steps
        sampler.stop()
        clocks = sampler.summary()
        bst_stats = batch.stats()
        t_max, ps_all = combine_ranks(pg_dist, g_ms, g_ps, "cuda")
        value = ps_all / (t_max / 1e3)

        # ---- end to end: new host seeds every step (same counts: the graph replays), final
        # positions and abort codes back to the host
        e2e_s, e2e_ps, h2d, d2h = 0.0, 0, 0, 0
        for k in range(0 if args.no_e2e else 1 + max(1, args.e2e_steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for d in sorted(eb):
                eb[d].set_seeds(groups[d][0])
            batch.run()
            outs = [(eb[d].final_positions(), eb[d].status()) for d in sorted(eb)]
            dt = time.perf_counter() - t0
            if k >= 1:
                e2e_s += dt
                e2e_ps += batch.stats().particle_steps
                h2d = sum(groups[d][0].nbytes for d in eb)
                d2h = sum(p.nbytes + s_.nbytes for p, s_ in outs)
        assert batch.stats().captures == bst_stats.captures, "new seeds of the same counts must not capture again"
        e_t, e_ps = combine_ranks(pg_dist, e2e_s * 1e3, e2e_ps, "cuda")
        e2e = None if args.no_e2e else {
            "value": e_ps / (e_t / 1e3), "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": max(1, args.e2e_steps),
            "path": "capi.Engine.set_seeds (host) + capi.Batch.run + final positions / status to host"}
        final = {}
        for d in spans:
            pos, st = eb[d].final_positions(), eb[d].status()
            final[(d, "lifetime")] = {j: (pos[off:off + cnt], st[off:off + cnt])
                                      for j, off, cnt in spans[d] if j in sampled}
        # fixed horizon: the batch again with every lifetime capped
        if rank == 0 and not args.no_acc and not args.no_plain:
            for d in spans:
                eb[d].set_lifetimes(np.minimum(groups[d][1], horizon))
            batch.run()
            for d in spans:
                pos, st = eb[d].final_positions(), eb[d].status()
                final[(d, "fixed")] = {j: (pos[off:off + cnt], st[off:off + cnt])
                                       for j, off, cnt in spans[d] if j in sampled}
        batch.close()
        for e in eb.values():
            e.close()
        results[bst] = dict(value=value, t_max=t_max, ps_dim=ps_dim, g_ms=g_ms, clocks=clocks, stats=bst_stats,
                            tuned=tuned, e2e=e2e, final=final)

    # ---- plain FP32: one run per set, sequentially, every snapshot resident
    plain_final = {(d, h): {} for d in spans for h in ("lifetime", "fixed")}
    plain_ms, plain_ps = 0.0, 0
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    for j, s in enumerate([] if args.no_plain else w.sets):
        d, off, cnt = loc[j]
        e = eng_p[d]
        e.set_seeds(groups[d][0][off:off + cnt])
        e.update_settings(maximum_simulation_time=60.0 * s["life"])
        e.run(resident)
        st = e.stats()
        plain_ms += st.run_ms
        plain_ps += st.particle_steps
        if j in sampled:
            plain_final[(d, "lifetime")][j] = (e.final_positions(), e.status())
    torch.cuda.synchronize()
    plain_wall = time.perf_counter() - wall0
    p_t, p_ps = combine_ranks(pg_dist, plain_wall * 1e3, plain_ps, "cuda")
    plain_value_wall = p_ps / (p_t / 1e3) if p_ps else None
    pd_t, _ = combine_ranks(pg_dist, plain_ms, plain_ps, "cuda")
    plain_value_dev = p_ps / (pd_t / 1e3) if p_ps else None
    acc = {}
    if rank == 0 and not args.no_acc and not args.no_plain:
        for d in spans:
            for j, m in sample[d]:
                _, off, cnt = loc[j]
                eng_p[d].set_seeds(groups[d][0][off:off + cnt])
                eng_p[d].update_settings(maximum_simulation_time=60.0 * horizon)
                eng_p[d].run(resident)
                plain_final[(d, "fixed")][j] = (eng_p[d].final_positions(), eng_p[d].status())
        for bst in storages:
            acc[bst] = batch_accuracy(w, bst, sample, results[bst]["final"], plain_final, horizon)
    for e in eng_p.values():
        e.close()
    if pg_dist:
        pg_dist.barrier()
    if rank != 0:
        return None

    peak, peak_src = load_peaks()
    plain = None if args.no_plain else {
        "storage": "f32", "value_device": plain_value_dev, "value_wall": plain_value_wall,
        "seconds_wall": p_t / 1e3, "particle_steps": int(p_ps),
        "path": "one capi.Engine.run per set (set_seeds, MaximumSimulationTime = lifetime * 60 s)"}
    per = {}
    for bst in storages:
        r = results[bst]
        alg = sum(r["ps_dim"][d] * RK4_FINAL_BYTES[(d, bst)] for d in r["ps_dim"])
        achieved = alg / (r["g_ms"] / 1e3) / 1e9 if r["g_ms"] > 0 else None
        per[bst] = {
            "value": r["value"], "ms_per_step": r["t_max"] / args.steps,
            "speedup_vs_plain_f32": r["value"] / plain_value_wall if plain_value_wall else None,
            "speedup_vs_plain_f32_device": r["value"] / plain_value_dev if plain_value_dev else None,
            "accuracy": acc.get(bst), "e2e": r["e2e"], "tuned": r["tuned"], "graph_nodes": r["stats"].nodes,
            "clocks": r["clocks"],
            "gpu_launches": int((r["stats"].kernel_launches + r["stats"].aux_launches) * args.steps),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None, "peak_source": peak_src,
                         "bytes_per_particle_step": {f"{d}d": RK4_FINAL_BYTES[(d, bst)] for d in r["ps_dim"]},
                         "kernel": "advance_kernel (graph replay, whole run)"}}
    head = per[storages[0]]
    return {
        "metric": "particle-steps/s", "value": head["value"], "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": storages[0],
        "data": "synthetic (seeded Fourier-mode fields, 3D 192x192x64 and 2D 1024x512)",
        "config": {"workload": BATCH_WORKLOAD, "sets": len(w.sets),
                   "particles_per_gpu": int(sum(s["n"] for s in w.sets)),
                   "sets_3d": int(sum(s["dim"] == 3 for s in w.sets)), "snapshots": n_snap,
                   "lifetimes": [100, args.batch_life_max], "storages": storages, "parallelism": f"replicas{world}",
                   "l2": f"inputs larger than L2 ({n_snap} snapshots per field resident)"},
        "plain": plain, "per_storage": per,
        "speedup_vs_plain_f32": head["speedup_vs_plain_f32"], "accuracy": head["accuracy"], "e2e": head["e2e"],
        "roofline": head["roofline"], "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
        "load_s": load_s,
    }


PRECISION_WORKLOAD = "precision-3d-rk4-4e6x5000"


def run_precision(args, world, rank, local, pg_dist):
    """The plain 3D configuration at 4e6 particles x 5,000 steps: float32 wind, and BF16 / FP16
    wind with Kahan-compensated positions and float64 time weights.  Snapshots are evaluated on
    the device (gr_field) and the float64 oracle gets host copies of the same snapshots."""
    import torch
    from oracle import oracle as orc
    from pygranite_b200 import capi
    from pygranite_b200 import workloads as W

    steps = args.prec_steps
    settings, _, seeds = W.config2(n_particles=args.prec_particles, n_snapshots=2, steps=steps, seed=rank)
    settings = dict(settings, SaveInterval=100, AdditionalVolumeMode=0, AdditionalCompute=[])
    n_snap = steps // 10 + 1
    field = W.FourierField((64, 192, 192), (250.0, 1000.0, 1000.0), n_modes=32, seed=rank)
    fld = capi.Field.fourier(field, 600.0, n_snap, device=local)
    # record r >= 1 holds the state after 100 (r - 1) + 1 steps (records after every 100th step)
    checks = [r for r in (2, 5, 11, 50) if 100 * (r - 1) + 1 <= steps]
    forms = {"f32": dict(storage=0), "bf16": dict(storage=1, compensated=1, time_mode=1),
             "f16": dict(storage=2, compensated=1, time_mode=1)}
    out, hist = {}, {}
    for name, opt in forms.items():
        e = capi.Engine(capi.settings_from_reference(settings, ring_slots=n_snap, device=local, **opt))
        e.set_seeds(seeds)
        for k in range(n_snap):
            fld.load(e, k)
        resident = lambda k: 1 if k < n_snap else 0  # noqa: E731
        e.run(resident)   # warm-up
        torch.cuda.synchronize()
        e.run(resident)
        st = e.stats()
        t_max, ps_all = combine_ranks(pg_dist, st.run_ms, st.particle_steps, "cuda")
        res = e.results(volumes=False, compute=False)
        m = args.prec_sample
        hist[name] = (res["trajectories"][:m, checks], res["status"][:m])
        out[name] = {"value": ps_all / (t_max / 1e3), "run_ms": t_max, "particle_steps": ps_all,
                     "settings": opt}
        del res
        e.close()
    acc = None
    if rank == 0:
        m = args.prec_sample
        snaps = []
        for k in range(n_snap):
            a = fld.snapshot(k)
            snaps.append([a[0], a[1], a[2]])
        ref = orc.run(orc.settings(**settings), orc.Inputs(wind=snaps, seeds=seeds[:m]), precision="f64")
        cell = np.array([1000.0, 1000.0, 250.0])
        acc = {}
        ab = ref["step_of_abort"]
        for name in forms:
            traj, status = hist[name]
            rows = {"final_status_mismatch": int(np.sum(status != ref["status"]))}
            for j, r in enumerate(checks):
                k = 100 * (r - 1) + 1                 # steps the record holds
                live = (ab < 0) | (ab >= k)           # not yet aborted in the float64 run
                d = (np.abs(traj[live, j] - ref["trajectories"][live, r]) / cell).max(axis=1)
                rows[f"after_{k}_steps"] = {
                    "cell_rms": float(np.sqrt(np.mean(d ** 2))) if d.size else None,
                    "cell_p50": float(np.median(d)) if d.size else None,
                    "cell_p99": float(np.percentile(d, 99)) if d.size else None,
                    "cell_max": float(d.max()) if d.size else None, "particles": int(d.size)}
            acc[name] = rows
    fld.close()
    if pg_dist:
        pg_dist.barrier()
    if rank != 0:
        return None
    peak, peak_src = load_peaks()
    return {
        "metric": "particle-steps/s", "value": out["bf16"]["value"], "unit": "particle-steps/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": out["bf16"]["run_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16",
        "data": "synthetic (seeded Fourier-mode field evaluated on the device)",
        "config": {"workload": PRECISION_WORKLOAD, "particles_per_gpu": args.prec_particles, "sim_steps": steps,
                   "snapshots": n_snap, "grid": [192, 192, 64], "records_every": 100,
                   "l2": f"inputs larger than L2 ({n_snap} snapshots resident)"},
        "per_storage": out, "error_vs_f64": acc,
        "error_note": "position error in grid cells of the first particles against the float64 oracle on the same "
                      "float32 snapshots, over particles not yet aborted in the float64 run at that record; the f32 "
                      "row is the plain float32 path.  Particle-step counts differ between rows: in float32 "
                      "arithmetic a particle creeping toward an upper face freezes once its displacement drops below "
                      "half an ulp of its position yet stays above the Wind threshold, and stays alive; compensated "
                      "positions keep creeping like float64 and end with a Wind abort",
        "e2e": None, "roofline": None, "clocks": None, "gpu_launches": None, "peak_source": peak_src, "peak": peak,
    }


SERVE_WORKLOAD = "serve-poisson-3d-512x512x96"


def serve_sample(w, count):
    """Requests checked against the float64 oracle: the shortest ones of each integrator that
    end inside the field; returns their indices and the snapshots they read."""
    clock = int(round(600.0 * (w.n_snapshots - 1) / 60.0))
    picks = []
    for integ in (1, 0):
        cand = [j for j in range(len(w.arrivals)) if w.integrators[j] == integ
                and int(np.floor(w.starts[j] / 60.0 + 1e-9)) + int(w.steps[j]) <= clock]
        cand.sort(key=lambda j: (int(w.steps[j]), int(w.counts[j])))
        picks += cand[:max(1, count // 2)]
    keep = set()
    for j in picks:
        k0 = int(np.floor(w.starts[j] / 60.0 + 1e-9))
        first, last = k0 // 10, (k0 + int(w.steps[j])) // 10 + 1
        keep.update(range(first, min(last, w.n_snapshots - 1) + 1))
    return picks, keep


def serve_accuracy(w, results, host_snaps, storage, m=256):
    """Final-position error in grid cells of sampled served requests against the float64
    oracle on the same float32 snapshots (the oracle's clock starts every particle at the
    request's start step, as the server's does)."""
    from oracle import oracle as orc
    cell = CELL_3D
    any_snap = next(iter(host_snaps.values()))
    wind = [host_snaps.get(k, any_snap) for k in range(w.n_snapshots)]   # unread windows: placeholders
    out = []
    for j, (pos, status, k0, steps) in sorted(results.items()):
        seeds = w.seeds(j)[:m]
        st = orc.settings(**dict(w.settings(), Integrator=int(w.integrators[j])))
        ref = orc.run(st, orc.Inputs(wind=wind, seeds=seeds), precision="f64", start_step=int(k0),
                      step_limit=int(k0 + steps), threads=os.cpu_count() or 1)
        both = (ref["status"] == 0) & (status[:m] == 0)
        d = (np.abs(pos[:m].astype(np.float64) - ref["trajectories"][:, -1]) / cell).max(axis=1)[both]
        out.append({"request": int(j), "integrator": ["euler", "rk4"][int(w.integrators[j])], "start_step": int(k0),
                    "steps": int(steps), "particles": int(d.size),
                    "cell_rms": float(np.sqrt(np.mean(d ** 2))) if d.size else None,
                    "cell_max": float(d.max()) if d.size else None,
                    "status_mismatch": int(np.sum(ref["status"] != status[:m]))})
    return {"vs_f64": out, "storage": storage,
            "note": "served result (" + storage + " wind) against the float64 oracle on the float32 snapshots"}


def run_serve(args, world, rank, local, pg_dist):
    """Requests arrive as a Poisson stream; latency = submit -> results on the host."""
    import torch
    from pygranite_b200 import capi
    from pygranite_b200 import workloads as W

    w = W.ServeWorkload(rate=args.serve_rate, seconds=args.serve_seconds, seed=rank)
    nz, ny, nx = w.grid
    code = {"f32": 0, "bf16": 1, "f16": 2}[args.serve_storage]
    t0 = time.perf_counter()
    srv = capi.Server(capi.settings_from_reference(w.settings(), storage=code, device=local), w.n_snapshots, w.grid,
                      hbm_budget=int(args.serve_budget_gb * (1 << 30)))
    # accuracy sample: the shortest RK4 and Euler requests that end inside the field; the
    # float32 snapshots they read are kept on the host for the float64 oracle
    acc_req, keep = serve_sample(w, args.serve_acc) if rank == 0 else ([], set())
    host_snaps = {}
    dev = W.DeviceFourierField(w.field, device=f"cuda:{local}")
    for k in range(w.n_snapshots):
        planes = dev.snapshot(600.0 * k)
        torch.cuda.synchronize()
        srv.set_snapshot_device(k, [p.data_ptr() for p in planes])
        if k in keep:
            host_snaps[k] = [p.cpu().numpy() for p in planes]
    del dev
    torch.cuda.empty_cache()
    setup_s = time.perf_counter() - t0
    srv.start()
    # warm-up: a few small requests so module loading and first-touch costs are not timed
    for j in range(3):
        rid = srv.submit(w.seeds(j)[:1000], 600.0 * (3 + 5 * j), 50, j % 2)
        srv.wait(rid, 60.0)
        srv.release(rid)
    s0 = srv.stats()
    ps0 = s0.particle_steps
    if pg_dist:
        pg_dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ids = []
    start = time.perf_counter()
    for j in range(len(w.arrivals)):
        sd = w.seeds(j)
        delay = w.arrivals[j] - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(sd, float(w.starts[j]), int(w.steps[j]), int(w.integrators[j])))
    submit_end = time.perf_counter() - start
    lat, queue, nparts, steps_run, acc_out = [], [], 0, 0, {}
    for j, rid in enumerate(ids):
        st = srv.wait(rid, 600.0)
        info = srv.info(rid)
        if st == capi.GR_REQ_DONE:
            lat.append(info.done_s - info.submit_s)
            queue.append(info.admit_s - info.submit_s)
            nparts += info.n
            steps_run += info.steps
            if j in acc_req:
                pos, status = srv.result(rid)[:2]
                acc_out[j] = (pos, status, info.start_step, info.steps)
        srv.release(rid)
    wall = time.perf_counter() - start
    sampler.stop()
    clocks = sampler.summary()
    s1 = srv.stats()
    srv.close()
    ps = s1.particle_steps - ps0
    t_max, ps_all = combine_ranks(pg_dist, wall * 1e3, ps, "cuda")
    value = ps_all / (t_max / 1e3)
    if pg_dist:
        pg_dist.barrier()
    if rank != 0:
        return None
    lat, queue = np.array(lat), np.array(queue)
    pct = lambda a, q: float(np.percentile(a, q)) if a.size else None  # noqa: E731
    accuracy = serve_accuracy(w, acc_out, host_snaps, args.serve_storage) if acc_out else None
    return {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": 1, "warmup": 3, "ms_per_step": t_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.serve_storage,
        "data": "synthetic (seeded Fourier-mode field, Poisson request stream)",
        "config": {"workload": SERVE_WORKLOAD, "grid": [nx, ny, nz], "snapshots": w.n_snapshots, "ring_slots": 4,
                   "rate_per_s": args.serve_rate, "arrival_seconds": args.serve_seconds,
                   "requests": len(ids), "completed": int(lat.size), "particles": int(nparts),
                   "storage": args.serve_storage, "parallelism": f"replicas{world}",
                   "l2": "window pair 403 MB > L2: streamed from HBM"},
        "latency_s": {"p50": pct(lat, 50), "p90": pct(lat, 90), "p99": pct(lat, 99), "max": pct(lat, 100),
                      "mean": float(lat.mean()) if lat.size else None},
        "queue_s": {"p50": pct(queue, 50), "p99": pct(queue, 99)}, "accuracy": accuracy,
        "server": {"windows": s1.windows, "sweeps": s1.sweeps, "jumps": s1.jumps, "deferred": s1.deferred,
                   "peak_particles": s1.peak_particles, "capacity_particles": s1.capacity_particles,
                   "steps_requested_mean": float(np.mean(w.steps)), "steps_run_mean": steps_run / max(1, lat.size),
                   "submit_seconds": submit_end, "setup_s": setup_s},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(s1.h2d_bytes - s0.h2d_bytes),
                "d2h_bytes_per_step": int(s1.d2h_bytes - s0.d2h_bytes),
                "path": "capi.Server.submit (host seeds) -> results on the host; wall clock over the stream"},
        "roofline": None, "clocks": clocks, "gpu_launches": None,
    }


GYRE_WORKLOAD = "gyre-2d-euler-1e4x1000"


def run_gyre(args, world, rank, local, pg_dist):
    """The 2D configuration: double gyre on 256 x 128 nodes, 10,000 particles, 1,000 Euler steps
    of 0.01, a record after every step.  Device-resident (16-slot ring, engine events) and
    through the pygranite API (constructor, Python loader, every record copied out), each run
    checked against the float32 oracle."""
    import torch
    import pygranite_b200 as pg
    from oracle import oracle as orc
    from pygranite_b200 import capi
    from pygranite_b200 import workloads as W

    settings, src, seeds = W.config1()
    n_snap = len(src.wind)
    eng = capi.Engine(capi.settings_from_reference(settings, ring_slots=n_snap, device=local))
    eng.set_seeds(seeds)
    for k, snap in enumerate(src.wind):
        eng.load_windfield(k, snap)
    resident = lambda k: 1 if k < n_snap else 0  # noqa: E731
    for _ in range(max(1, args.warmup)):
        eng.run(resident)
    ms = ps = 0.0
    for _ in range(args.steps):
        eng.run(resident)
        st = eng.stats()
        ms += st.run_ms
        ps += st.particle_steps
    res = eng.results(volumes=False, compute=False)
    eng.close()
    ref = orc.run(orc.settings(**settings), orc.Inputs(wind=src.wind, seeds=seeds), precision="f32",
                  threads=os.cpu_count() or 1)
    device_exact = bool(np.array_equal(res["trajectories"], ref["trajectories"]) and
                        np.array_equal(res["status"], ref["status"]))
    enums = dict(Space=pg.Space, Integrator=pg.Integrator, WindfieldMode=pg.WindfieldMode, BorderMode=pg.BorderMode,
                 CurvatureMode=pg.CurvatureMode)
    api_s, api_ps, api_exact = 0.0, 0, None
    for k in range(1 + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s_ = W.apply_settings(pg.IntegratorSettings(), settings, enums)
        s_.Device = local
        out = pg.TrajectoryIntegrator(s_, W.make_loader(pg.DataLoader, src), pg.TrajectorySet(seeds)).compute()
        traj = out.trajectories()
        dt = time.perf_counter() - t0
        if k >= 1:
            api_s += dt
            api_ps += out.particleSteps()
        if k == args.steps:
            api_exact = bool(np.array_equal(traj, ref["trajectories"]))
    return {"metric": "particle-steps/s", "unit": "particle-steps/s", "dtype": "f32",
            "config": {"workload": GYRE_WORKLOAD, "grid": [256, 128], "snapshots": n_snap, "particles": len(seeds),
                       "steps": 1000, "records": int(res["trajectories"].shape[1])},
            "value": ps / (ms / 1e3), "ms_per_step": ms / args.steps, "f32_bitexact": device_exact,
            "e2e": {"value": api_ps / api_s, "ms_per_step": 1e3 * api_s / args.steps, "f32_bitexact": api_exact,
                    "path": "TrajectoryIntegrator(settings, loader, TrajectorySet(seeds)).compute().trajectories()"}}


# option combinations timed on the benchmark field (device-resident, 1e6 particles x 200 steps)
OPTION_SETS = {
    "rk4_plain": dict(CurvatureMode=0, AdditionalVolumeMode=0, AdditionalCompute=[]),
    "rk4_benchmark_options": dict(),
    "rk4_individual_curvature_length": dict(CurvatureMode=3, AbortMode=1, MaximumLength=60000.0,
                                            AdditionalVolumeMode=0, AdditionalCompute=[]),
    "rk4_fast_total_curvature_reverse": dict(CurvatureMode=2, Reverse=True, AdditionalVolumeMode=0,
                                             AdditionalCompute=[]),
    "euler_fitlength_uplift_topography": dict(Integrator=0, CurvatureMode=0, AbortMode=2, MaximumLength=60000.0,
                                              UpLiftMode=1, AdditionalVolumeMode=0, AdditionalCompute=[]),
    "rk4_kahan": dict(CurvatureMode=0, AdditionalVolumeMode=0, AdditionalCompute=[]),
}


def run_options(args, world, rank, local, pg_dist):
    """Throughput of option combinations beside the benchmark's own, on its field and seeds
    (1e6 particles, 200 steps, records every 10): which kernel variant each runs (lean or
    generic) and its particle-steps/s, device-resident."""
    from pygranite_b200 import capi
    from pygranite_b200 import workloads as W

    steps = 200
    settings, src, seeds = W.config2(n_particles=1_000_000, n_snapshots=steps // 10 + 1, steps=steps, seed=rank)
    n_snap = len(src.wind)
    n = seeds.shape[0]
    rng = np.random.default_rng(3)
    lift = (rng.standard_normal((n, 3)) * np.array([5.0, 5.0, 1.0])).astype(np.float32)
    topo = np.zeros((192, 192), np.float32)
    topo[:, 150:] = 2000.0
    out = {}
    for name, over in OPTION_SETS.items():
        st = dict(settings, **over)
        extra = dict(compensated=1) if name == "rk4_kahan" else {}
        eng = capi.Engine(capi.settings_from_reference(st, ring_slots=n_snap, device=local, **extra))
        eng.set_seeds(seeds)
        for k, snap in enumerate(src.wind):
            eng.load_windfield(k, snap)
        if st.get("AdditionalVolumeMode", 0):
            eng.load_volume(0, 0, src.volumes[0]["T"])
        for e_, code in enumerate(st.get("AdditionalCompute", [])):
            eng.compile_expression(e_, code, ["T"], [])
        if st.get("UpLiftMode", 0):
            eng.load_uplift(0, lift)
            eng.set_topography(topo)
        resident = lambda k: 1 if k < n_snap else 0  # noqa: E731
        eng.run(resident)
        ms = ps = 0.0
        for _ in range(3):
            eng.run(resident)
            s_ = eng.stats()
            ms += s_.run_ms
            ps += s_.particle_steps
        out[name] = {"value": ps / (ms / 1e3), "ms_per_run": ms / 3, "settings": {k: v for k, v in over.items()}}
        eng.close()
    return {"metric": "particle-steps/s", "unit": "particle-steps/s", "dtype": "f32",
            "config": {"workload": "options-3d-1e6x200", "grid": [192, 192, 64], "steps": steps, "records_every": 10},
            "per_option_set": out}


def run_forms(args, world, rank, local):
    """The other configurations and the three forms beside the plain kernel, on one GPU, each its
    own phase after the plain measurement: the 2D double gyre, option combinations, batching
    (BF16 and FP16 graphs against one plain FP32 run per set), serving (the Poisson request
    stream) and precision (the 4e6-particle, 5,000-step configuration per storage).  A phase
    that fails reports its error instead of a figure."""
    import copy
    import traceback
    import torch
    forms = {}
    for name, fn, kw in (("gyre", run_gyre, {}), ("options", run_options, {}), ("precision", run_precision, {}),
                         ("batch", run_batch, {"storages": ["bf16", "f16"]}), ("serve", run_serve, {})):
        a = copy.copy(args)
        a.steps, a.warmup = min(args.steps, 5), min(args.warmup, 2)
        t0 = time.perf_counter()
        try:
            forms[name] = fn(a, world, rank, local, None, **kw)
        except Exception as exc:  # reported in the line; the plain figures stand
            forms[name] = {"error": f"{type(exc).__name__}: {exc}", "trace": traceback.format_exc()[-2000:]}
        if isinstance(forms[name], dict):
            forms[name]["phase_s"] = time.perf_counter() - t0
        gc.collect()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return forms


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("batch", "serve", "precision"):
        world, rank, local = dist_env()
        import torch
        torch.cuda.set_device(local)
        pg_dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
            pg_dist = dist
        run = {"batch": run_batch, "serve": run_serve, "precision": run_precision}[args.workload]
        line = run(args, world, rank, local, pg_dist)
        if line is not None:
            print(json.dumps(line), flush=True)
        if pg_dist:
            pg_dist.destroy_process_group()
        return 0

    world, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    pg_dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
        pg_dist = dist

    from pygranite_b200 import capi
    import pygranite_b200 as pg
    from pygranite_b200 import workloads as W

    settings, src, seeds = workload(args, rank)
    n_snap = len(src.wind)
    storage = {"f32": 0, "bf16": 1, "f16": 2}[args.storage]

    # ---------------- device-resident engine: every snapshot in the ring before timing
    cs = capi.settings_from_reference(settings, ring_slots=n_snap, storage=storage, device=local,
                                      steps_per_launch=args.steps_per_launch, sort_interval=args.sort_interval,
                                      layout=args.layout)
    eng = capi.Engine(cs)
    eng.set_seeds(seeds)
    for k, snap in enumerate(src.wind):
        eng.load_windfield(k, snap)
    eng.load_volume(0, 0, src.volumes[0]["T"])
    eng.compile_expression(0, settings["AdditionalCompute"][0], ["T"], [])
    resident = lambda s: 1 if s < n_snap else 0  # noqa: E731

    for _ in range(args.warmup):
        eng.run(resident)
    torch.cuda.synchronize()
    if pg_dist:
        pg_dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    tot_ms = kern_ms = 0.0
    ps = launches = aux = 0
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        eng.run(resident)
        st = eng.stats()
        tot_ms += st.run_ms
        kern_ms += st.kernel_ms
        ps += st.particle_steps
        launches += st.launches
        aux += st.aux_launches
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    sampler.stop()
    clocks = sampler.summary()
    if pg_dist:
        pg_dist.barrier()
    info = eng.info()

    # max over ranks of the device time, sum of the particle-steps
    t_max, ps_all = combine_ranks(pg_dist, tot_ms, ps, "cuda")
    value = ps_all / (t_max / 1e3)

    # ---------------- the timed run's own output against the oracle (after the timed region):
    # a fixed sample of particle ids spread over the seed array, every record
    parity, ids, refs = None, None, None
    if args.parity_sample > 0 and rank == 0 and storage == 0:
        res = eng.results(pinned=True)
        ids = sample_ids(seeds.shape[0], args.parity_sample)
        got = {"trajectories": np.array(res["trajectories"][ids]), "status": res["status"][ids],
               "total_curvature": res["total_curvature"][ids], "volume": np.array(res["volume_info"][0][ids]),
               "expression": np.array(res["compute_info"][0][ids])}
        del res
        gc.collect()
        refs = plain_oracle(settings, src, seeds, ids)
        parity = check_plain(got, *refs)
        parity["run"] = "the last timed run (device-resident engine)"
    eng.close()

    # ---------------- end to end through the pygranite API (host snapshots, 3-slot ring)
    # Timed per step: the TrajectoryIntegrator constructor, compute() with every snapshot
    # uploaded from host memory through the Python loader, and every record copied out to host
    # arrays.  Headline: the loader serves page-locked arrays (pinned_empty) and the results land
    # in page-locked arrays (PinnedResults), so both directions are single DMAs.  Beside it, the
    # defaults: pageable numpy in, fresh numpy arrays out (staging copies on host cores).
    e2e = None
    if not args.no_e2e:
        enums = dict(Space=pg.Space, Integrator=pg.Integrator, WindfieldMode=pg.WindfieldMode,
                     AdditionalVolumeMode=pg.AdditionalVolumeMode, BorderMode=pg.BorderMode,
                     CurvatureMode=pg.CurvatureMode)
        h2d = seeds.nbytes + sum(p.nbytes for snap in src.wind for p in snap) + src.volumes[0]["T"].nbytes

        def e2e_run(source, pinned_results, check):
            s = W.apply_settings(pg.IntegratorSettings(), settings, enums)
            s.WindStorage = [pg.WindStorage.Float32, pg.WindStorage.BFloat16, pg.WindStorage.Float16][storage]
            s.Device = local
            s.SortInterval = args.sort_interval
            s.StepsPerLaunch = args.steps_per_launch
            s.WindLayout = args.layout
            s.PinnedResults = pinned_results
            e_ps, e_s, d2h, reps, par = 0, 0.0, 0, [], None
            for k in range(1 + args.e2e_steps):
                gc.collect()   # the previous step's garbage, outside the timed region
                torch.cuda.synchronize()
                if pg_dist:
                    pg_dist.barrier()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                t0 = time.perf_counter()
                ev0.record()
                loader = W.make_loader(pg.DataLoader, source)
                integ = pg.TrajectoryIntegrator(s, loader, pg.TrajectorySet(seeds))
                t1 = time.perf_counter()
                res = integ.compute()
                t2 = time.perf_counter()
                del integ   # engine teardown is part of the step
                ev1.record()
                torch.cuda.synchronize()
                dt = max(time.perf_counter() - t0, ev0.elapsed_time(ev1) / 1e3)
                reps.append({"ctor_ms": round(1e3 * (t1 - t0), 1), "compute_ms": round(1e3 * (t2 - t1), 1),
                             "total_ms": round(1e3 * dt, 1)})
                if k >= 1:
                    e_s += dt
                    e_ps += res.particleSteps()   # counted by this run's own engine
                    d2h = res.trajectories().nbytes + res.computeInfo(0).nbytes + res.volumeInfo("T").nbytes + \
                        res.totalCurvatures().nbytes + 4 * seeds.shape[0]
                if check and k == args.e2e_steps and refs is not None:
                    # the last timed step's TrajectorySet, through the reference's accessors
                    got = {"trajectories": res.trajectories()[ids],
                           "status": np.array([int(r) for r in res.abortReasons()], np.int32)[ids],
                           "total_curvature": np.asarray(res.totalCurvatures())[ids],
                           "volume": res.volumeInfo("T")[ids], "expression": res.computeInfo(0)[ids]}
                    par = check_plain(got, *refs)
                    par["run"] = "the last timed pygranite-API run (TrajectorySet accessors)"
                del res
            e_t, e_psa = combine_ranks(pg_dist, e_s, e_ps, "cuda")
            out = {"value": e_psa / e_t, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps,
                   "ms_per_step": 1e3 * e_t / max(1, args.e2e_steps), "particle_steps": int(e_psa), "reps": reps}
            if par is not None:
                out["parity"] = par
            return out

        # the same snapshots and volume, copied once into page-locked memory (data preparation,
        # outside the timed region)
        nz_, ny_, nx_ = src.wind[0][0].shape
        pinned_wind = capi.pinned_empty((n_snap, 3, nz_, ny_, nx_))
        for k, snap in enumerate(src.wind):
            for c in range(3):
                pinned_wind[k, c] = snap[c]
        pinned_T = capi.pinned_empty(src.volumes[0]["T"].shape)
        pinned_T[...] = src.volumes[0]["T"]
        psrc = W.SnapshotSource([[pinned_wind[k, c] for c in range(3)] for k in range(n_snap)],
                                volumes=[{"T": pinned_T}])
        e2e = e2e_run(psrc, True, True)
        e2e["host_buffers"] = "page-locked: loader arrays from pinned_empty, IntegratorSettings.PinnedResults = True"
        if world == 1:
            e2e["pageable"] = e2e_run(src, False, False)
            e2e["pageable"]["host_buffers"] = "pageable numpy loader arrays, results in fresh numpy arrays (the defaults)"
        else:
            # N processes share one host: the pageable variant's extra 4 GB per rank is left out
            e2e["pageable"] = None
        del psrc, pinned_wind, pinned_T
        gc.collect()
        capi.host_cache_trim()   # give the page-locked snapshots back before the next phase

    # ---------------- native loader: snapshots evaluated on the device (gr_field_loader) into
    # the default 3-slot ring; nothing crosses from the host but seeds and results
    native = None
    if not args.no_native:
        field = W.FourierField((64, 192, 192), (250.0, 1000.0, 1000.0), n_modes=32, seed=rank)
        f = capi.Field.fourier(field, 600.0, n_snap, device=local)
        ncs = capi.settings_from_reference(settings, storage=storage, device=local,
                                           steps_per_launch=args.steps_per_launch, sort_interval=args.sort_interval,
                                           layout=args.layout)
        n_s, n_ps, n_ms = 0.0, 0, 0.0
        for k in range(2):
            ne = capi.Engine(ncs)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ne.set_seeds(seeds)
            f.load(ne, 0)
            f.load(ne, 1)
            ne.load_volume(0, 0, src.volumes[0]["T"])
            ne.compile_expression(0, settings["AdditionalCompute"][0], ["T"], [])
            ne.run_native(f)
            out = ne.results(pinned=True)
            dt = time.perf_counter() - t0
            if k == 1:
                n_s, n_ps, n_ms = dt, ne.stats().particle_steps, ne.stats().run_ms
            del out
            ne.close()
        f.close()
        nt, nps = combine_ranks(pg_dist, n_s * 1e3, n_ps, "cuda")
        native = {"value": nps / (nt / 1e3), "unit": "particle-steps/s", "run_ms": n_ms,
                  "path": "capi.Engine.run_native(capi.Field.fourier): snapshots evaluated on the device into the "
                          "3-slot ring; seeds in and every record out to page-locked host arrays"}

    if pg_dist:
        pg_dist.barrier()
    if rank != 0:
        if pg_dist:
            pg_dist.destroy_process_group()
        return 0

    peak, peak_src = load_peaks()
    bpps = BYTES_PER_PARTICLE_STEP[args.storage]
    avg_launch_ms = kern_ms / max(launches, 1)
    ps_launch = ps / max(launches, 1)
    achieved = ps * bpps / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else None
    prof = load_kernel_profile(args.storage)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (prof["dram_bytes_per_particle_step"] * ps_launch) if prof else None,
                "peak_source": peak_src, "bytes_per_particle_step": bpps,
                "bytes_note": "gather-equivalent: every corner of every stage counted as if fetched from HBM; the "
                              "window pair is L2-resident, so this fraction can exceed 1",
                "kernel": "advance_kernel<3,RK4,Pair<float>>", "avg_launch_ms": avg_launch_ms,
                "particle_steps_per_launch": ps_launch}
    if prof:
        rate = ps / (kern_ms / 1e3)                 # particle-steps per second of step-kernel time
        dram_gbs = prof["dram_bytes_per_particle_step"] * rate / 1e9
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        issue_peak = 148 * 4 * sm_mhz * 1e6         # warp instructions per second, 4 schedulers per SM
        issue = prof["warp_inst_per_particle_step"] * rate
        roofline.update(dram_gbs=dram_gbs, dram_frac=dram_gbs / peak, issue_frac=issue / issue_peak,
                        active_bound="issue (instruction throughput)" if issue / issue_peak > dram_gbs / peak
                        else "hbm", profile=prof.get("source"))
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(args, settings, src, seeds)
    del src
    gc.collect()
    forms = None
    if world == 1 and not args.no_forms:
        forms = run_forms(args, world, rank, local)
    cfg = plain_config(args, world)
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.storage, "data": "synthetic (seeded Fourier-mode field)", "config": cfg,
        "run": {"records": int(info.records), "steps_run": int(info.steps),
                "particle_steps_per_run": int(ps / max(1, args.steps))},
        "parity": parity, "e2e": e2e, "native_loader": native, "roofline": roofline, "cpu_baseline": cpu,
        "clocks": clocks, "gpu_launches": int(launches + aux), "wall_s": wall, "forms": forms,
    }
    print(json.dumps(line), flush=True)
    if pg_dist:
        pg_dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
