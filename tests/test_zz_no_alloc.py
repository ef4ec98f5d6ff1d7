"""The allocation-free entry point gr_advance_noalloc (GPU).

It exists for callers that cannot call cudaMalloc: plug-in hosts whose device memory belongs
to their own pool allocator, and real-time loops that forbid allocation after start-up.  Its
results must equal what gr_run computes for the same particles and snapshots: compared bit for
bit (the tolerance of the parity tests for this path), on two calls in a row, since every call
reuses the same device scratch array.  This file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from pygranite_b200 import capi

pytestmark = pytest.mark.gpu


def field(shape, seed):
    rng = np.random.default_rng(seed)
    return [[rng.standard_normal(shape).astype(np.float32) for _ in range(len(shape))] for _ in range(2)]


def run_engine(settings, wind, seeds):
    eng = capi.Engine(settings)
    eng.set_seeds(seeds)
    for k, snap in enumerate(wind):
        eng.load_windfield(k, snap)
    eng.run(lambda s: 0)
    out = eng.results(volumes=False, compute=False)
    ps = eng.info().particle_steps
    eng.close()
    return out["trajectories"][:, -1], out["status"], ps


def packed(torch, snap):
    """node-major packed snapshot: float4 {u, v, w, 0} (3D) or float2 {u, v} (2D)"""
    comps = [torch.from_numpy(c) for c in snap]
    if len(comps) == 3:
        comps.append(torch.zeros_like(comps[0]))
    return torch.stack(comps, dim=-1).contiguous().cuda()


def run_noalloc(torch, settings, wind, seeds, steps, dtd):
    dim = seeds.shape[1]
    back, front = packed(torch, wind[0]), packed(torch, wind[1])
    pos = [torch.from_numpy(np.ascontiguousarray(seeds[:, d])).cuda() for d in range(dim)]
    pz = pos[2].data_ptr() if dim == 3 else None
    status = torch.zeros(seeds.shape[0], dtype=torch.int32, device="cuda")
    ps = capi.advance_noalloc(settings, wind[0][0].shape, back.data_ptr(), front.data_ptr(), 0.0, dtd, 0.0, steps,
                              pos[0].data_ptr(), pos[1].data_ptr(), pz, status.data_ptr(), seeds.shape[0])
    torch.cuda.synchronize()
    return np.stack([p.cpu().numpy() for p in pos], axis=1), status.cpu().numpy(), ps


def test_noalloc_matches_gr_run_twice():
    torch = pytest.importorskip("torch")
    # call 1: 3D RK4, block borders
    shape3 = (12, 20, 24)
    wind3 = field(shape3, 1)
    seeds3 = np.random.default_rng(2).uniform([0, 0, 0], [24, 20, 12], (3000, 3)).astype(np.float32)
    s3 = capi.default_settings(space=0, integrator=1, delta_t=0.5, data_time_distance=4.0,
                               maximum_simulation_time=4.0, grid_scale=[1.0, 1.0, 1.0], offset=[0.0, 0.0, 0.0],
                               save_interval=0)
    ref_pos, ref_st, ref_ps = run_engine(s3, wind3, seeds3)
    pos, st, ps = run_noalloc(torch, s3, wind3, seeds3, steps=8, dtd=4.0)
    assert np.array_equal(st, ref_st)
    assert np.array_equal(pos, ref_pos)
    assert ps == ref_ps
    # call 2 (same scratch array): 2D Euler with a periodic x border
    shape2 = (32, 48)
    wind2 = field(shape2, 3)
    seeds2 = np.random.default_rng(4).uniform([0, 0], [48, 32], (2000, 2)).astype(np.float32)
    s2 = capi.default_settings(space=1, integrator=0, delta_t=0.25, data_time_distance=8.0,
                               maximum_simulation_time=5.0, grid_scale=[1.0, 1.0], offset=[0.0, 0.0],
                               save_interval=0, border_mode=1)
    ref_pos, ref_st, ref_ps = run_engine(s2, wind2, seeds2)
    pos, st, ps = run_noalloc(torch, s2, wind2, seeds2, steps=20, dtd=8.0)
    assert np.array_equal(st, ref_st)
    assert np.array_equal(pos, ref_pos)
    assert ps == ref_ps


def test_noalloc_rejects_oversized_and_unsupported_requests():
    s = capi.default_settings(space=0, delta_t=0.5)
    dummy = 1 << 20   # never dereferenced: the arguments are rejected first
    with pytest.raises(capi.GraniteError, match="GR_NOALLOC_MAX_STEPS"):
        capi.advance_noalloc(s, (4, 4, 4), dummy, dummy, 0.0, 1.0, 0.0, 4097, dummy, dummy, dummy, dummy, 10)
    unsupported = [dict(curvature_mode=1), dict(windfield_mode=0), dict(time_mode=1), dict(minimum_alive=5),
                   dict(volume_mode=1), dict(abort_mode=1), dict(storage=1), dict(compensated=1)]
    for kw in unsupported:
        s = capi.default_settings(space=0, delta_t=0.5, **kw)
        with pytest.raises(capi.GraniteError, match="plain integrator only"):
            capi.advance_noalloc(s, (4, 4, 4), dummy, dummy, 0.0, 1.0, 0.0, 4, dummy, dummy, dummy, dummy, 10)
    s = capi.default_settings(space=0, delta_t=0.5)
    for start in (-0.5, 1.0, 2.0):   # the first step must start inside [time_back, time_front)
        with pytest.raises(capi.GraniteError, match="time_start"):
            capi.advance_noalloc(s, (4, 4, 4), dummy, dummy, 0.0, 1.0, start, 4, dummy, dummy, dummy, dummy, 10)
