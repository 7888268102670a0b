"""cam_power_noalloc -- P(k) binning without any device allocation -- against
the allocating entry point cam_power, through the C ABI.

The no-allocation variant exists for callers that may not call cudaMalloc
(code inside a memory pool or arena it does not own, latency-critical loops
that must not reach the allocator); its scratch is one fixed array built into
the library.  The spectrum it bins comes from cam_fft_r2c into a torch
tensor allocated by the test, not by the entry point.  Two calls in a row
must both match cam_power within the P(k) tolerance of the other tests
(1e-5 of max(|P|, shot-noise level)), so whatever the first call leaves in
the shared scratch cannot leak into the second.  This file is collected
last, so a run that stops at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
from conftest import pk_rel_err
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, TSC, Context

pytestmark = pytest.mark.gpu


def _mesh(n, box, scheme, seed):
    x, y, z = synth.clumped(300_000, box, 3_000, 2.0, 0.8, seed)
    m, _ = orc.assign_f64(scheme, x, y, z, None, orc.Grid.cubic(n, box))
    return m.astype(np.float32)


def _noalloc(spec_dev, n, box, n_obj, opts):
    import torch
    nb = opts.nbins
    pk = np.empty(nb)
    modes = np.empty(nb, np.int64)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.lib().cam_power_noalloc(ctypes.c_void_p(spec_dev.data_ptr()), n, L.F32, box, n_obj,
                                   ctypes.byref(opts), pk.ctypes.data, modes.ctypes.data,
                                   ctypes.c_void_p(stream))
    assert rc == L.CAM_OK, rc
    return pk, modes


@pytest.mark.parametrize("n,box,scheme,nbins", [(64, 1000.0, CIC, 32), (96, 700.0, TSC, 40)])
def test_noalloc_matches_cam_power_twice(ctx, n, box, scheme, nbins):
    import torch
    mesh = _mesh(n, box, scheme, seed=n)
    opts = Context.pk_opts(scheme, nbins=nbins)
    ref = ctx.power(mesh, box, opts)
    spec = ctx.fft_r2c(torch.from_numpy(mesh).cuda())
    torch.cuda.synchronize()
    n_obj = float(mesh.astype(np.float64).sum())
    floor = np.abs(ref.shot_noise) * np.ones(nbins)
    for _ in range(2):
        pk, modes = _noalloc(spec, n, box, n_obj, opts)
        assert np.array_equal(modes, ref.modes)
        assert pk_rel_err(pk, ref.pk, floor) <= 1e-5


def test_noalloc_rejects_oversize(ctx):
    import torch
    opts = Context.pk_opts(CIC, nbins=513)
    spec = torch.zeros((16, 16, 9), dtype=torch.complex64, device="cuda")
    pk = np.empty(513)
    rc = L.lib().cam_power_noalloc(ctypes.c_void_p(spec.data_ptr()), 16, L.F32, 100.0, 1.0,
                                   ctypes.byref(opts), pk.ctypes.data, None, None)
    assert rc == L.CAM_E_UNSUPPORTED
    opts = Context.pk_opts(CIC, nbins=8)
    rc = L.lib().cam_power_noalloc(ctypes.c_void_p(spec.data_ptr()), 4096, L.F32, 100.0, 1.0,
                                   ctypes.byref(opts), pk.ctypes.data, None, None)
    assert rc == L.CAM_E_UNSUPPORTED
