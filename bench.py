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
        .compute(), with the loader serving host numpy snapshots into a 3-slot device ring;
        every H2D upload and the D2H copy of the records are inside the timed region.
--impl reference : the reference has no CPU implementation of the path; the CPU oracle port
        (float64, OpenMP on all host cores) runs bounded samples of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

BYTES_PER_PARTICLE_STEP = {  # algorithmic bytes per particle-step (roofline section)
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
    p.add_argument("--sort-interval", type=int, default=4,
                   help="launches between compaction / Morton re-sorts of the live particles (0 = off)")
    p.add_argument("--layout", type=int, default=0, help="0: window-pair wind layout, 1: ring slots")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-particles", type=int, default=20000)
    p.add_argument("--cpu-steps", type=int, default=100)
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


def load_traffic_per_particle_step(storage):
    """DRAM bytes per particle-step from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "advance_kernel_traffic.json")
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


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    settings, src, seeds = workload(args, 0)
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline(args, settings, src, seeds)
        if k >= args.warmup:
            vals.append(cb["value"])
    value = float(np.mean(vals))
    cb["value"] = value
    line = {"impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Fourier-mode field)",
            "config": {"workload": WORKLOAD, "particles": args.particles, "sim_steps": args.sim_steps},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

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
    eng.close()

    # ---------------- end to end through the pygranite API (host snapshots, 3-slot ring)
    e2e = None
    if not args.no_e2e:
        enums = dict(Space=pg.Space, Integrator=pg.Integrator, WindfieldMode=pg.WindfieldMode,
                     AdditionalVolumeMode=pg.AdditionalVolumeMode, BorderMode=pg.BorderMode,
                     CurvatureMode=pg.CurvatureMode)
        s = W.apply_settings(pg.IntegratorSettings(), settings, enums)
        s.WindStorage = [pg.WindStorage.Float32, pg.WindStorage.BFloat16, pg.WindStorage.Float16][storage]
        s.Device = local
        s.SortInterval = args.sort_interval
        s.StepsPerLaunch = args.steps_per_launch
        s.WindLayout = args.layout
        h2d = seeds.nbytes + sum(p.nbytes for snap in src.wind for p in snap) + src.volumes[0]["T"].nbytes
        e_ps, e_s, d2h = 0, 0.0, 0
        for k in range(1 + args.e2e_steps):
            torch.cuda.synchronize()
            if pg_dist:
                pg_dist.barrier()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            ev0.record()
            loader = W.make_loader(pg.DataLoader, src)
            res = pg.TrajectoryIntegrator(s, loader, pg.TrajectorySet(seeds)).compute()
            ev1.record()
            torch.cuda.synchronize()
            dt = max(time.perf_counter() - t0, ev0.elapsed_time(ev1) / 1e3)
            if k >= 1:
                e_s += dt
                e_ps += info.particle_steps
                d2h = res.trajectories().nbytes + res.computeInfo(0).nbytes + res.volumeInfo("T").nbytes + \
                    res.totalCurvatures().nbytes + 4 * seeds.shape[0]
            del res
        e_t, e_psa = combine_ranks(pg_dist, e_s, e_ps, "cuda")
        e2e = {"value": e_psa / e_t, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps}

    if pg_dist:
        pg_dist.barrier()
    if rank != 0:
        if pg_dist:
            pg_dist.destroy_process_group()
        return 0

    peak, peak_src = load_peaks()
    bpps = BYTES_PER_PARTICLE_STEP[args.storage]
    achieved = ps * bpps / (kern_ms / 1e3) / 1e9 if kern_ms > 0 else None
    tpps = load_traffic_per_particle_step(args.storage)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (tpps * ps / max(launches, 1)) if tpps else None,
                "peak_source": peak_src, "bytes_per_particle_step": bpps,
                "kernel": "advance_kernel<3,RK4>", "avg_launch_ms": kern_ms / max(launches, 1),
                "particle_steps_per_launch": ps / max(launches, 1)}
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(args, settings, src, seeds)
    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.storage, "data": "synthetic (seeded Fourier-mode field)",
        "config": {"workload": WORKLOAD, "particles_per_gpu": args.particles, "sim_steps": args.sim_steps,
                   "snapshots": n_snap, "grid": [192, 192, 64], "storage": args.storage,
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (201 snapshots, 7.6 GB ring)",
                   "records": int(info.records), "steps_run": int(info.steps),
                   "sort_interval": args.sort_interval, "steps_per_launch": args.steps_per_launch,
                   "wind_layout": ["window-pair", "ring"][args.layout]},
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": int(launches + aux), "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    if pg_dist:
        pg_dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
