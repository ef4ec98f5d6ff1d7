"""Native loaders (gr_field_*): analytic windfields evaluated on the device.

Snapshots are compared with the host generators of the benchmark inputs (workloads.py), which
evaluate the same formulas in float64 with numpy: after rounding to float32 they agree within
two units in the last place of the field's largest value (the trigonometric functions of CUDA
and glibc may differ in the last float64 bit, and the Fourier sum is accumulated in another
order).  A run fed by the native loader is compared with the same run fed from numpy snapshots.
"""
import numpy as np
import pytest

from pygranite_b200 import capi
from pygranite_b200 import workloads as W


def ulp_bound(ref):
    return 2.0 * np.spacing(np.float32(np.abs(ref).max()))


def test_field_arguments_are_checked_without_gpu():
    with pytest.raises(capi.GraniteError, match="Invalid Space"):
        one = np.ones(4)
        p = lambda a: a.ctypes.data_as(capi.ctypes.POINTER(capi.ctypes.c_double))  # noqa: E731
        h = capi.ctypes.c_void_p()
        shape = np.array([4, 4, 4, 4], np.int64)
        capi._check(capi.lib().gr_field_fourier(4, shape.ctypes.data_as(capi.ctypes.POINTER(capi.ctypes.c_int64)),
                                                p(one), 1, p(one), p(one), p(one), p(one), p(one), 1.0, 2, 0,
                                                capi.ctypes.byref(h)))
    with pytest.raises(capi.GraniteError, match="invalid field parameters"):
        capi.Field.double_gyre(dt=-1.0)


@pytest.mark.gpu
def test_double_gyre_snapshots_match_host_generator():
    ref = W.double_gyre(256, 128, 16)
    f = capi.Field.double_gyre()
    for k in (0, 3, 15):
        got = f.snapshot(k)
        for c in range(2):
            assert np.abs(got[c] - ref[k][c]).max() <= ulp_bound(ref[k][c]), (k, c)
    f.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape,spacing,modes", [
    ((16, 24, 32), (250.0, 1000.0, 1000.0), 32),
    ((48, 64), (1000.0, 1000.0), 32),
    # several x blocks (the last one partial), a row count that is no multiple of the rows per
    # block, and mode chunks with a partial last chunk
    ((5, 7, 150), (250.0, 1000.0, 1000.0), 100),
    ((13, 300), (1000.0, 1000.0), 65),
])
def test_fourier_snapshots_match_host_generator(shape, spacing, modes):
    kw = {} if len(shape) == 3 else dict(rms=(7.0710678, 7.0710678))
    field = W.FourierField(shape, spacing, n_modes=modes, seed=4, **kw)
    f = capi.Field.fourier(field, 600.0, 8)
    for k in (0, 5):
        ref = field.snapshot(600.0 * k)
        got = f.snapshot(k)
        for c in range(len(shape)):
            assert np.abs(got[c] - ref[c]).max() <= ulp_bound(ref[c]), (k, c)
    f.close()


@pytest.mark.gpu
def test_run_with_native_loader_matches_numpy_loader():
    settings, src, seeds = W.config2(n_particles=3000, n_snapshots=6, grid=(16, 24, 24), steps=50)
    field = W.FourierField((16, 24, 24), (250.0, 1000.0, 1000.0), n_modes=32, seed=0)
    results = []
    for native in (False, True):
        eng = capi.Engine(capi.settings_from_reference(settings))
        eng.set_seeds(seeds)
        f = capi.Field.fourier(field, 600.0, len(src.wind)) if native else None
        for k in (0, 1):   # the windfield first: it fixes the grid the volume is checked against
            f.load(eng, k) if native else eng.load_windfield(k, src.wind[k])
        eng.load_volume(0, 0, src.volumes[0]["T"])
        eng.compile_expression(0, settings["AdditionalCompute"][0], ["T"], [])
        if native:
            eng.run_native(f)
        else:
            eng.run(lambda k: (eng.load_windfield(k, src.wind[k]), 1)[1] if k < len(src.wind) else 0)
        results.append(eng.results())
        eng.close()
    a, b = results
    assert a["info"].steps == b["info"].steps == 50
    same = a["status"] == b["status"]
    assert same.mean() > 0.999
    cells = np.abs(a["trajectories"][same] - b["trajectories"][same]) / np.array([1000.0, 1000.0, 250.0])
    assert cells.max() < 1e-3, cells.max()
