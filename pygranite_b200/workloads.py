"""Seeded synthetic wind fields and seed sets for the benchmark configurations.

No public dataset is involved: every field is generated from a fixed seed.
  * double gyre (2D, analytic) on [0,2] x [0,1];
  * Fourier-mode fields (2D / 3D): a sum of seeded random modes with a k^(-5/3) amplitude
    spectrum, scaled to a target RMS, phases advected linearly in time;
  * a temperature volume T = 290 K - 6.5 K/km * z + 2 K seeded noise.
`SnapshotLoader` serves precomputed snapshots through pygranite's DataLoader interface
(source/granite/DataLoader.hpp:26-81): windfield() returns snapshot k, step() advances k.
"""
from __future__ import annotations

import math

import numpy as np


# ----------------------------------------------------------------- double gyre (config 1)

def double_gyre(nx=256, ny=128, n_snapshots=16, A=0.1, eps=0.25, omega=2 * math.pi / 10, dt=1.0,
                lx=2.0, ly=1.0):
    """u = -dpsi/dy, v = dpsi/dx with psi = A sin(pi f(x,t)) sin(pi y),
    f = eps sin(wt) x^2 + (1 - 2 eps sin(wt)) x; nodes x_i = i*lx/nx, y_j = j*ly/ny."""
    x = np.arange(nx, dtype=np.float64) * (lx / nx)
    y = np.arange(ny, dtype=np.float64) * (ly / ny)
    X, Y = np.meshgrid(x, y)  # (ny, nx)
    snaps = []
    for k in range(n_snapshots):
        t = k * dt
        a = eps * math.sin(omega * t)
        b = 1.0 - 2.0 * eps * math.sin(omega * t)
        f = a * X * X + b * X
        dfdx = 2.0 * a * X + b
        u = -math.pi * A * np.sin(math.pi * f) * np.cos(math.pi * Y)
        v = math.pi * A * np.cos(math.pi * f) * np.sin(math.pi * Y) * dfdx
        snaps.append([u.astype(np.float32), v.astype(np.float32)])
    return snaps


def uniform_seeds(n, seed, lo, hi):
    """n points uniform in the box [lo, hi) (numpy PCG64 generator with the given seed)."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    return (lo + rng.random((n, lo.size)) * (hi - lo)).astype(np.float32)


# ----------------------------------------------------------------- Fourier-mode fields

class FourierField:
    """Sum of `n_modes` random plane waves per component, amplitude ~ |k|^(-5/3).

    shape = (nz, ny, nx) for 3D or (ny, nx) for 2D; spacing in metres per axis (same order).
    |k| is log-uniform between 2*pi/L_max and 2*pi/(4*dx); phases advance as -k.U t with
    U = `advect` (m/s).  Each component is scaled so its RMS over the grid at t = 0 equals
    `rms[c]`.  Snapshots are evaluated as a rank-n_modes separable product, so a snapshot
    costs one small complex matrix product per component.
    """

    def __init__(self, shape, spacing, n_modes=32, seed=0, rms=(7.0710678, 7.0710678, 0.1),
                 advect=(5.0, 3.0, 0.0), dtype=np.float32):
        self.shape = tuple(shape)
        self.dim = len(shape)
        self.spacing = tuple(float(s) for s in spacing)
        self.dtype = dtype
        rng = np.random.default_rng(seed)
        axes = [np.arange(n) * d for n, d in zip(self.shape, self.spacing)]  # z,y,x order
        extent = max(n * d for n, d in zip(self.shape, self.spacing))
        dmin = min(d for d in self.spacing[-2:])
        kmin, kmax = 2 * math.pi / extent, 2 * math.pi / (4 * dmin)
        adv = np.asarray(advect[: self.dim][::-1] if self.dim == 3 else advect[:2][::-1], np.float64)
        self.comps = []
        for c in range(self.dim):
            kmag = np.exp(rng.uniform(math.log(kmin), math.log(kmax), n_modes))
            direction = rng.normal(size=(n_modes, self.dim))
            if self.dim == 3:
                direction[:, 0] *= 0.25  # flatter modes in the vertical
            direction /= np.linalg.norm(direction, axis=1, keepdims=True)
            kvec = direction * kmag[:, None]           # (modes, dim) in axis order (z,y,x)
            amp = kmag ** (-5.0 / 3.0)
            phase0 = rng.uniform(0, 2 * math.pi, n_modes)
            omega = kvec @ adv
            factors = [np.exp(1j * np.outer(kvec[:, a], axes[a])) for a in range(self.dim)]
            self.comps.append(dict(amp=amp, phase0=phase0, omega=omega, factors=factors, scale=1.0, kvec=kvec))
        for c in range(self.dim):
            r = float(np.sqrt(np.mean(self._eval(c, 0.0).astype(np.float64) ** 2)))
            self.comps[c]["scale"] = (rms[c] / r) if r > 0 else 0.0

    def _eval(self, c, t):
        m = self.comps[c]
        coef = m["amp"] * np.exp(1j * (m["phase0"] - m["omega"] * t))  # (modes,)
        f = m["factors"]
        if self.dim == 3:
            fz, fy, fx = f
            a = (coef[:, None] * fz).T                     # (nz, modes)
            b = (fy[:, :, None] * fx[:, None, :]).reshape(len(coef), -1)   # (modes, ny*nx)
            val = (a @ b).real.reshape(self.shape)
        else:
            fy, fx = f
            a = (coef[:, None] * fy).T                     # (ny, modes)
            val = (a @ fx).real
        return (val * m.get("scale", 1.0)).astype(self.dtype)

    def snapshot(self, t):
        return [self._eval(c, t) for c in range(self.dim)]


class DeviceFourierField:
    """A FourierField's modes evaluated on a CUDA device with torch (complex64): the same
    wave vectors, amplitudes, phases and RMS scaling, for fields too large to generate on the
    host in reasonable time.  Snapshots are float32 CUDA tensors in (z, y, x) / (y, x) order."""

    def __init__(self, field: FourierField, device="cuda"):
        import torch
        self.torch, self.field, self.device = torch, field, device
        self.parts = []
        for m in field.comps:
            f = [torch.as_tensor(x, dtype=torch.complex64, device=device) for x in m["factors"]]
            if field.dim == 3:
                fz, fy, fx = f
                b = (fy[:, :, None] * fx[:, None, :]).reshape(fy.shape[0], -1)
                self.parts.append((fz, b))
            else:
                fy, fx = f
                self.parts.append((fy, fx))

    def snapshot(self, t):
        torch = self.torch
        out = []
        for m, (lead, b) in zip(self.field.comps, self.parts):
            coef = m["amp"] * np.exp(1j * (m["phase0"] - m["omega"] * t))
            c = torch.as_tensor(coef, dtype=torch.complex64, device=self.device)
            a = (c[:, None] * lead).T
            val = (a @ b).real.reshape(self.field.shape) * float(m.get("scale", 1.0))
            out.append(val.to(torch.float32).contiguous())
        return out


def temperature(shape, spacing_z, seed=1):
    """T = 290 - 6.5e-3 * z + 2 * N(0,1) noise, z = iz * spacing_z (metres)."""
    nz = shape[0]
    rng = np.random.default_rng(seed)
    z = (np.arange(nz, dtype=np.float64) * spacing_z)[:, None, None]
    return (290.0 - 6.5e-3 * z + 2.0 * rng.standard_normal(shape)).astype(np.float32)


# ----------------------------------------------------------------- loader

class SnapshotSource:
    """Precomputed snapshots plus optional volumes / constants / uplift per snapshot."""

    def __init__(self, wind, volumes=None, constants=None, uplift=None):
        self.wind = wind
        self.volumes = volumes or []
        self.constants = constants or []
        self.uplift = uplift or []


def make_loader(base_cls, source: SnapshotSource):
    """A DataLoader subclass of `base_cls` (pygranite's DataLoader) serving `source`."""

    class SnapshotLoader(base_cls):
        def __init__(self):
            base_cls.__init__(self)
            self.k = 0
            self.calls = 0

        def step(self):
            self.calls += 1
            if self.k + 1 < len(source.wind):
                self.k += 1
                return True
            return False

        def windfield(self):
            return source.wind[self.k]

        def additionalVolumes(self):
            if not source.volumes:
                return {}
            return source.volumes[min(self.k, len(source.volumes) - 1)]

        def constants(self):
            if not source.constants:
                return {}
            return source.constants[min(self.k, len(source.constants) - 1)]

        def uplift(self):
            if not source.uplift:
                return np.zeros((0,), np.float32)
            return source.uplift[min(self.k, len(source.uplift) - 1)]

    return SnapshotLoader()


# ----------------------------------------------------------------- benchmark configurations

def config1(n_particles=10_000, n_snapshots=16):
    """Plain 2D Euler FP32: double gyre on 256 x 128 over [0,2] x [0,1], h = 0.01 x 1000 steps."""
    settings = dict(Space=1, Integrator=0, WindfieldMode=1, DeltaT=0.01, DataTimeDistance=1.0,
                    GridScale=[2.0 / 256, 1.0 / 128], Offset=[0.0, 0.0], SaveInterval=1,
                    BorderMode=0, CurvatureMode=0, MaximumSimulationTime=10.0)
    src = SnapshotSource(double_gyre(256, 128, n_snapshots))
    seeds = uniform_seeds(n_particles, 0, [0.0, 0.0], [2.0, 1.0])
    return settings, src, seeds


def config2(n_particles=1_000_000, n_snapshots=201, grid=(64, 192, 192), steps=2000, seed=0):
    """Plain 3D RK4 FP32 on a Fourier field (1 km x 1 km x 250 m), 600 s snapshots, h = 60 s,
    TotalCurvature, a constant temperature volume and the expression sqrt(u*u+v*v)*T."""
    nz, ny, nx = grid
    field = FourierField(grid, (250.0, 1000.0, 1000.0), n_modes=32, seed=seed)
    wind = [field.snapshot(600.0 * k) for k in range(n_snapshots)]
    T = temperature(grid, 250.0, seed=seed + 1)
    settings = dict(Space=0, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=[1000.0, 1000.0, 250.0], Offset=[0.0, 0.0, 0.0], SaveInterval=10,
                    BorderMode=0, CurvatureMode=1, MaximumSimulationTime=60.0 * steps,
                    AdditionalVolumeMode=1, AdditionalCompute=["sqrt(u*u+v*v)*T"])
    src = SnapshotSource(wind, volumes=[{"T": T}])
    seeds = uniform_seeds(n_particles, seed, [0.0, 0.0, 0.0], [nx * 1000.0, ny * 1000.0, nz * 250.0 / 2])
    return settings, src, seeds


def round_storage(a, storage):
    """The float32 -> storage -> float32 round trip of the device ring (round to nearest even);
    storage is "f32", "bf16" or "f16"."""
    a = np.ascontiguousarray(a, np.float32)
    if storage == "f16":
        return a.astype(np.float16).astype(np.float32)
    if storage == "bf16":
        u = a.view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
        return u.astype(np.uint32).view(np.float32)
    return a


def batch_sets(n_sets=512, n_min=100, n_max=200_000, life_min=100, life_max=5000, frac3d=0.7, seed=0):
    """Seed-set descriptors of the batching workload: particle counts log-uniform in
    [n_min, n_max], lifetimes (RK4 steps) uniform in [life_min, life_max], a fraction `frac3d`
    on the 3D field and the rest on the 2D field."""
    rng = np.random.default_rng(seed)
    counts = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_sets))).astype(np.int64)
    lifes = rng.integers(life_min, life_max + 1, n_sets)
    is3d = rng.random(n_sets) < frac3d
    return [dict(n=int(counts[j]), life=int(lifes[j]), dim=3 if is3d[j] else 2, seed=seed * 100_003 + j)
            for j in range(n_sets)]


class BatchWorkload:
    """The batching configuration: seed sets of uneven size and lifetime on a 3D field (the
    plain 3D configuration's Fourier field, 1 km x 1 km x 250 m) and a 2D Fourier field of the
    same spectrum (1 km spacing), 600 s snapshots, h = 60 s RK4, final records only."""

    def __init__(self, n_sets=512, grid3=(64, 192, 192), grid2=(512, 1024), n_min=100, n_max=200_000,
                 life_min=100, life_max=5000, frac3d=0.7, seed=0):
        self.grid3, self.grid2 = tuple(grid3), tuple(grid2)
        self.sets = batch_sets(n_sets, n_min, n_max, life_min, life_max, frac3d, seed)
        self.life_max = max(s["life"] for s in self.sets)
        self.n_snapshots = (self.life_max * 60 + 599) // 600 + 1
        self.field3 = FourierField(self.grid3, (250.0, 1000.0, 1000.0), n_modes=32, seed=seed)
        self.field2 = FourierField(self.grid2, (1000.0, 1000.0), n_modes=32, seed=seed + 7,
                                   rms=(7.0710678, 7.0710678))

    def settings(self, dim):
        gs = [1000.0, 1000.0, 250.0] if dim == 3 else [1000.0, 1000.0]
        return dict(Space=0 if dim == 3 else 1, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=gs, Offset=[0.0] * len(gs), SaveInterval=0, BorderMode=0, CurvatureMode=0,
                    MaximumSimulationTime=60.0 * self.life_max)

    def snapshot(self, dim, k):
        return (self.field3 if dim == 3 else self.field2).snapshot(600.0 * k)

    def seeds(self, j):
        s = self.sets[j]
        if s["dim"] == 3:
            nz, ny, nx = self.grid3
            return uniform_seeds(s["n"], s["seed"], [0.0, 0.0, 0.0], [nx * 1000.0, ny * 1000.0, nz * 250.0 / 2])
        ny, nx = self.grid2
        return uniform_seeds(s["n"], s["seed"], [0.0, 0.0], [nx * 1000.0, ny * 1000.0])

    def group(self, dim):
        """Concatenated seeds, lifetimes and the (set index, offset, count) of every set on
        the field of dimension `dim`."""
        idx = [j for j, s in enumerate(self.sets) if s["dim"] == dim]
        seeds, lifes, spans, off = [], [], [], 0
        for j in idx:
            sd = self.seeds(j)
            seeds.append(sd)
            lifes.append(np.full(len(sd), self.sets[j]["life"], np.int32))
            spans.append((j, off, len(sd)))
            off += len(sd)
        if not idx:
            return np.zeros((0, dim), np.float32), np.zeros(0, np.int32), []
        return np.concatenate(seeds), np.concatenate(lifes), spans

    def particle_steps_upper(self):
        return sum(s["n"] * s["life"] for s in self.sets)


class ServeWorkload:
    """The serving configuration: a Poisson stream of trajectory requests on a 3D field of the
    plain configuration's spectrum at 512 x 512 x 96 nodes (1 km, 1 km, 250 m), 120 snapshots
    600 s apart.  Each request: seeds uniform in the lower half of the domain (count
    log-uniform in [n_min, n_max]), a start time uniform over the field window, a step count
    uniform in [steps_min, steps_max], RK4 with probability p_rk4, else Euler."""

    def __init__(self, rate=200.0, seconds=60.0, grid=(96, 512, 512), n_snapshots=120, n_min=1000, n_max=500_000,
                 steps_min=200, steps_max=3000, p_rk4=0.8, seed=0):
        self.grid, self.n_snapshots, self.seed = tuple(grid), n_snapshots, seed
        self.field = FourierField(self.grid, (250.0, 1000.0, 1000.0), n_modes=32, seed=seed)
        rng = np.random.default_rng(seed + 17)
        t, arrivals = 0.0, []
        while True:
            t += rng.exponential(1.0 / rate)
            if t >= seconds:
                break
            arrivals.append(t)
        k = len(arrivals)
        self.arrivals = np.array(arrivals)
        self.counts = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), k))).astype(np.int64)
        self.starts = rng.uniform(0.0, 600.0 * (n_snapshots - 1), k)
        self.steps = rng.integers(steps_min, steps_max + 1, k)
        self.integrators = (rng.random(k) < p_rk4).astype(np.int32)

    def settings(self):
        return dict(Space=0, Integrator=1, WindfieldMode=1, DeltaT=60.0, DataTimeDistance=600.0,
                    GridScale=[1000.0, 1000.0, 250.0], Offset=[0.0, 0.0, 0.0], SaveInterval=0, BorderMode=0,
                    CurvatureMode=0, MaximumSimulationTime=600.0 * (self.n_snapshots - 1))

    def seeds(self, j):
        nz, ny, nx = self.grid
        return uniform_seeds(int(self.counts[j]), self.seed * 1_000_003 + j, [0.0, 0.0, 0.0],
                             [nx * 1000.0, ny * 1000.0, nz * 250.0 / 2])


def apply_settings(obj, settings: dict, enums=None):
    """Sets reference-named fields on a pygranite IntegratorSettings instance."""
    for k, v in settings.items():
        if enums is not None and k in enums:
            v = enums[k](v)
        setattr(obj, k, v)
    return obj
