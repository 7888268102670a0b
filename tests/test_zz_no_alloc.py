"""cam_power_noalloc -- P(k) binning without any device allocation -- through
the C ABI, against the FP64 oracle and the allocating entry point cam_power.

The no-allocation variant exists for callers that may not call cudaMalloc:
code that runs inside a memory pool or arena it does not own (a host
application that hands the GPU path pre-sized buffers), or a latency-critical
loop that must never reach the allocator.  Its scratch is one fixed array
built into the library.  The spectrum it bins comes from cam_fft_r2c into a
torch tensor allocated by the test, not by the entry point.

Two calls in a row must both match the oracle's P(k) and cam_power's within
the P(k) tolerance of the other tests (1e-5 of max(|P|, shot-noise level)),
so whatever the first call leaves in the shared scratch cannot leak into the
second; and the second call must not allocate: the library's allocation
counters stay at zero and the device's free memory is unchanged.  This file
is collected last, so a run that stops at the first failure has run every
other test.
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
from conftest import pk_rel_err
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, F64, TSC, Context, alloc_stats

pytestmark = pytest.mark.gpu


def _mesh(n, box, scheme, seed):
    x, y, z = synth.clumped(300_000, box, 3_000, 2.0, 0.8, seed)
    m, _ = orc.assign_f64(scheme, x, y, z, None, orc.Grid.cubic(n, box))
    return m.astype(np.float32)


def _noalloc(spec_dev, n, box, n_obj, opts, prec=F32):
    import torch
    nb = opts.nbins
    pk = np.empty(nb)
    modes = np.empty(nb, np.int64)
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.lib().cam_power_noalloc(ctypes.c_void_p(spec_dev.data_ptr()), n, prec, box, n_obj,
                                   ctypes.byref(opts), pk.ctypes.data, modes.ctypes.data,
                                   ctypes.c_void_p(stream))
    assert rc == L.CAM_OK, rc
    return pk, modes


CASES = [
    # n, box, scheme, nbins, spectrum precision, input type (density with shot noise, or delta without)
    (64, 1000.0, CIC, 32, F32, "density"),
    (96, 700.0, TSC, 40, F32, "density"),
    (64, 800.0, CIC, 32, F64, "density"),
    (48, 600.0, TSC, 24, F32, "delta"),
    (48, 600.0, CIC, 24, F64, "delta"),
]


@pytest.mark.parametrize("n,box,scheme,nbins,prec,kind", CASES)
def test_noalloc_matches_oracle_twice_without_allocating(ctx, n, box, scheme, nbins, prec, kind):
    import torch
    mesh = _mesh(n, box, scheme, seed=n)
    delta = kind == "delta"
    if delta:
        mesh = (mesh / mesh.astype(np.float64).mean() - 1.0).astype(np.float32)
    dt = np.float64 if prec == F64 else np.float32
    mesh = mesh.astype(dt)
    opts = Context.pk_opts(scheme, nbins=nbins, sn_correction=not delta,
                           input_type=L.INPUT_DELTA if delta else L.INPUT_DENSITY)
    ref = ctx.power(mesh, box, opts)
    want = orc.power_grid(mesh.astype(np.float64), box, scheme, nbins, input_type="delta" if delta else "density",
                          sn_corr=not delta)
    spec = ctx.fft_r2c(torch.from_numpy(mesh).cuda())
    torch.cuda.synchronize()
    n_obj = float(mesh.astype(np.float64).sum())
    floor = np.abs(want.shot_noise * want.sum_sn / np.maximum(want.modes, 1)) if not delta else np.zeros(nbins)
    tol = 1e-5 if prec == F32 else 1e-10
    for call in range(2):
        if call == 1:
            alloc_stats(reset=True)
            free0 = torch.cuda.mem_get_info()[0]
        pk, modes = _noalloc(spec, n, box, n_obj, opts, prec)
        if call == 1:
            st = alloc_stats()
            assert st["allocs"] == 0 and st["bytes"] == 0, st
            assert torch.cuda.mem_get_info()[0] == free0
        assert np.array_equal(modes, want.modes)
        assert np.array_equal(modes, ref.modes)
        assert pk_rel_err(pk, want.pk, floor) <= tol
        assert pk_rel_err(pk, ref.pk, floor) <= tol


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


def test_noalloc_refuses_a_capturing_stream(ctx):
    """The call copies tables from the host and synchronises its stream, which
    a CUDA graph cannot record: under capture it must return
    CAM_E_UNSUPPORTED before touching the stream, and the capture must still
    end cleanly."""
    import torch
    opts = Context.pk_opts(CIC, nbins=8)
    spec = torch.zeros((16, 16, 9), dtype=torch.complex64, device="cuda")
    pk = np.empty(8)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.lib().cam_power_noalloc(ctypes.c_void_p(spec.data_ptr()), 16, L.F32, 100.0, 1.0,
                                       ctypes.byref(opts), pk.ctypes.data, None, ctypes.c_void_p(stream))
        out = spec.real * 2.0
    assert rc == L.CAM_E_UNSUPPORTED
    g.replay()
    torch.cuda.synchronize()
    assert float(out.abs().sum()) == 0.0
