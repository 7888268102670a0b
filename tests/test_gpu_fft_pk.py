"""GPU FFT and power spectrum vs the FP64 oracle (through the C ABI).

Bars: FFT relative RMS error <= 2e-6 (float) / 1e-12 (double) of the
spectrum; P(k) within 1e-5 of the FP64 oracle per bin, relative to
max(|P|, SN C/W^2) (the shot-noise level is the floor of shot-noise-
subtracted bins); mode counts bit-exact.
"""
import numpy as np
import pytest

import oracle as orc
from conftest import pk_rel_err
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, F64, NGP, TSC, Context, make_grid

pytestmark = pytest.mark.gpu

SIZES = [8, 12, 16, 24, 32, 48, 64, 96, 128]


def rel_rms(a, b):
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("prec", [F32, F64])
def test_r2c_vs_numpy(ctx, n, prec):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, n, n)) + 0.3
    dt = np.float64 if prec == F64 else np.float32
    got = ctx.fft_r2c(x.astype(dt))
    want = np.fft.rfftn(x.astype(dt).astype(np.float64))
    assert got.shape == want.shape
    assert rel_rms(got, want) <= (1e-12 if prec == F64 else 2e-6)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("prec", [F32, F64])
def test_c2r_vs_numpy(ctx, n, prec):
    rng = np.random.default_rng(100 + n)
    spec = rng.normal(size=(n, n, n // 2 + 1)) + 1j * rng.normal(size=(n, n, n // 2 + 1))
    cdt = np.complex128 if prec == F64 else np.complex64
    got = ctx.fft_c2r(spec.astype(cdt))
    want = np.fft.irfftn(spec.astype(cdt).astype(np.complex128), s=(n, n, n))
    assert rel_rms(got, want) <= (1e-12 if prec == F64 else 2e-6)


# The configurations' mesh sizes (384 and 768 need the radix-3 stages)
LARGE = [(192, F32), (256, F32), (384, F32), (384, F64), (512, F32), (768, F32)]


def _rel_rms_chunked(got, want):
    num = den = 0.0
    for i in range(0, got.shape[0], 32):
        a = np.asarray(got[i:i + 32], np.complex128 if np.iscomplexobj(got) else np.float64)
        b = want[i:i + 32]
        num += float(np.sum(np.abs(a - b) ** 2))
        den += float(np.sum(np.abs(b) ** 2))
    return float(np.sqrt(num / den))


@pytest.mark.parametrize("n,prec", LARGE)
def test_r2c_large_vs_fp64(ctx, n, prec):
    import torch
    rng = np.random.default_rng(n)
    dt = np.float64 if prec == F64 else np.float32
    x = (rng.standard_normal(size=(n, n, n), dtype=np.float32) + 0.3).astype(dt)
    got = ctx.fft_r2c(torch.from_numpy(x).cuda()).cpu().numpy()
    torch.cuda.empty_cache()
    want = orc.rfft3_f64(x)
    del x
    assert got.shape == want.shape
    assert _rel_rms_chunked(got, want) <= (1e-12 if prec == F64 else 2e-6)


@pytest.mark.parametrize("n,prec", [(384, F32), (512, F32), (768, F32), (384, F64)])
def test_c2r_large_vs_fp64(ctx, n, prec):
    import torch
    rng = np.random.default_rng(100 + n)
    h = n // 2 + 1
    cdt = np.complex128 if prec == F64 else np.complex64
    spec = np.empty((n, n, h), cdt)
    spec.real = rng.standard_normal(size=(n, n, h), dtype=np.float32)
    spec.imag = rng.standard_normal(size=(n, n, h), dtype=np.float32)
    got = ctx.fft_c2r(torch.from_numpy(spec).cuda()).cpu().numpy()
    torch.cuda.empty_cache()
    want = orc.irfft3_f64(spec, n)
    del spec
    assert _rel_rms_chunked(got, want) <= (1e-12 if prec == F64 else 2e-6)


@pytest.mark.parametrize("n", [64, 192, 256])
def test_roundtrip_large(ctx, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, n, n)).astype(np.float32)
    back = ctx.fft_c2r(ctx.fft_r2c(x))
    assert rel_rms(back, x) <= 2e-6


def _mesh(n, box, scheme, npart, seed, prec=F32):
    x, y, z = synth.clumped(npart, box, npart // 80, 2.0, 0.8, seed)
    ref, _ = orc.assign_f64(scheme, x, y, z, None, orc.Grid.cubic(n, box))
    return ref.astype(np.float64 if prec == F64 else np.float32)


@pytest.mark.parametrize("scheme", [NGP, CIC, TSC])
@pytest.mark.parametrize("prec", [F32, F64])
def test_power_vs_oracle(ctx, scheme, prec):
    n, box = 64, 1000.0
    mesh = _mesh(n, box, scheme, 300_000, 5, prec)
    opts = Context.pk_opts(scheme, nbins=0, ndel=1.0)
    got = ctx.power(mesh, box, opts)
    ref = orc.power_grid(mesh.astype(np.float64), box, scheme, n // 2)
    assert np.array_equal(got.modes, ref.modes)
    floor = ref.shot_noise * ref.sum_sn / np.maximum(ref.modes, 1)
    err = pk_rel_err(got.pk, ref.pk, floor)
    assert err <= (1e-5 if prec == F32 else 1e-10), err
    assert abs(got.shot_noise - ref.shot_noise) <= 1e-12 * ref.shot_noise
    np.testing.assert_allclose(got.kvector, ref.kcent, rtol=1e-14)


@pytest.mark.parametrize("ndel,kmin,nbins", [(1.5, 0.0, 21), (2.0, 0.5, 12), (1.0, 0.0, 40)])
def test_power_custom_bins(ctx, ndel, kmin, nbins):
    n, box = 48, 700.0
    mesh = _mesh(n, box, TSC, 200_000, 9)
    opts = Context.pk_opts(TSC, nbins=nbins, ndel=ndel, DeltaKmin=kmin)
    got = ctx.power(mesh, box, opts)
    ref = orc.power_grid(mesh.astype(np.float64), box, TSC, nbins, kmin_u=kmin, dk_u=ndel)
    assert np.array_equal(got.modes, ref.modes)
    floor = ref.shot_noise * ref.sum_sn / np.maximum(ref.modes, 1)
    assert pk_rel_err(got.pk, ref.pk, floor) <= 1e-5


def test_power_delta_input_no_corrections(ctx):
    n, box = 32, 300.0
    rng = np.random.default_rng(2)
    delta = rng.normal(size=(n, n, n)).astype(np.float32)
    opts = Context.pk_opts(CIC, nbins=16, ndel=1.0, mas_correction=False, sn_correction=False,
                           input_type=1)
    got = ctx.power(delta, box, opts)
    ref = orc.power_grid(delta.astype(np.float64), box, CIC, 16, input_type="delta", mas_corr=False,
                         sn_corr=False)
    assert np.array_equal(got.modes, ref.modes)
    np.testing.assert_allclose(got.pk, ref.pk, rtol=1e-5)


def test_power_deterministic(ctx):
    mesh = _mesh(64, 1000.0, CIC, 200_000, 13)
    opts = Context.pk_opts(CIC)
    a = ctx.power(mesh, 1000.0, opts).pk
    b = ctx.power(mesh, 1000.0, opts).pk
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


# ---------------------------------------------------------------- cross P(k)
@pytest.mark.parametrize("n,scheme,coeff,prec", [(64, CIC, False, F32), (64, TSC, True, F32), (48, CIC, True, F64)])
def test_cross_power_vs_oracle(ctx, n, scheme, coeff, prec):
    # two correlated tracers of one clumped process: the catalogue and a
    # random half of it, assigned with the same scheme
    box, nb = 500.0, n // 2
    x, y, z = synth.clumped(300_000, box, 3_000, 3.0, 0.8, seed=n + scheme)
    sel = np.random.default_rng(n).random(x.size) < 0.5
    g = orc.Grid.cubic(n, box)
    dt = np.float64 if prec == F64 else np.float32
    mx = orc.assign_f64(scheme, x, y, z, None, g)[0].astype(dt)
    my = orc.assign_f64(scheme, x[sel], y[sel], z[sel], None, g)[0].astype(dt)
    got = ctx.cross_power(mx, my, box, Context.pk_opts(scheme, nbins=nb), want_coeff=coeff)
    ref = orc.cross_power_grid(mx, my, box, scheme, nb, coeff=coeff)
    assert np.array_equal(got["modes"], ref.modes)
    has = ref.modes > 0
    for a, b in ((got["pk"], ref.pk), (got["pk_x"], ref.pk_x), (got["pk_y"], ref.pk_y)):
        assert np.max(np.abs(a - b)[has] / np.abs(b)[has]) <= 1e-5
    if coeff:
        assert np.all(got["pk"][has] <= 1.0 + 1e-6) and np.all(got["pk"][has] > 0.3)


def test_cross_power_mixed_inputs_and_mirror(ctx):
    # X a density, Y an overdensity; and the PowerSpectrumF mirror
    from cosmicatlas_b200.api import Params, PowerSpectrumF
    n, box, nb = 32, 300.0, 16
    x, y, z = synth.clumped(100_000, box, 1_000, 4.0, 0.8, seed=12)
    m = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))[0].astype(np.float32)
    d = (m.astype(np.float64) / m.mean(dtype=np.float64) - 1.0).astype(np.float32)
    got = ctx.cross_power(m, d, box, Context.pk_opts(CIC, nbins=nb), input_type_y=1)
    ref = orc.cross_power_grid(m, d, box, CIC, nb, "density", "delta")
    has = ref.modes > 0
    assert np.max(np.abs(got["pk"] - ref.pk)[has] / np.abs(ref.pk)[has]) <= 1e-5
    ps = PowerSpectrumF(Params(Nft=n, Lbox=box, mass_assignment=CIC, Nnp_data=nb, input_type="density_grid",
                               input_type_two="delta_grid"))
    ps.compute_cross_power_spectrum_grid(True, m.ravel(), d.ravel(), True)
    c = orc.cross_power_grid(m, d, box, CIC, nb, "density", "delta", coeff=True)
    np.testing.assert_allclose(ps.pk0[has], c.pk[has], rtol=1e-5)


# ---------------------------------------------------------------- multipoles
@pytest.mark.parametrize("n,scheme,los,prec", [(64, CIC, 2, F32), (48, TSC, 0, F32), (32, CIC, 1, F64)])
def test_power_multipoles_vs_oracle(ctx, n, scheme, los, prec):
    # a clumped catalogue displaced along the line of sight (a redshift-space
    # like squashing), so that P_2 and P_4 are non-zero
    box, nb = 500.0, n // 2
    x, y, z = synth.clumped(300_000, box, 3_000, 3.0, 0.8, seed=n + los)
    pos = [x, y, z]
    pos[los] = np.mod(pos[los] + 0.6 * np.sin(2 * np.pi * pos[los] / box * 3) * 8.0, box).astype(np.float32)
    dt = np.float64 if prec == F64 else np.float32
    mesh = orc.assign_f64(scheme, *pos, None, orc.Grid.cubic(n, box))[0].astype(dt)
    got = ctx.power_multipoles(mesh, box, Context.pk_opts(scheme, nbins=nb), los)
    p0, p2, p4, md = orc.power_multipoles(mesh, box, scheme, nb, los)
    assert np.array_equal(got["modes"], md)
    floor = p0.shot_noise * p0.sum_sn / np.maximum(p0.modes, 1)
    assert pk_rel_err(got["p0"], p0.pk, floor) <= 1e-5
    # l > 0 carry no shot noise; judge them against the monopole's scale
    scale = np.maximum(np.abs(p0.pk), floor)
    has = md > 0
    assert np.max(np.abs(got["p2"] - p2)[has] / scale[has]) <= 1e-5
    assert np.max(np.abs(got["p4"] - p4)[has] / scale[has]) <= 1e-5


def _context_without_tma():
    import os
    os.environ["CAM_NO_TMA"] = "1"
    try:
        return Context(0)
    finally:
        del os.environ["CAM_NO_TMA"]


@pytest.mark.parametrize("n", [64, 256, 384])
@pytest.mark.parametrize("prec", [F32, F64])
def test_tma_staged_columns_equal_cp_async(ctx, n, prec):
    # the column passes staged by TMA compute exactly what the cp.async
    # kernels compute: only the tile movement differs
    import torch
    rng = np.random.default_rng(7 + n)
    dt = np.float64 if prec == F64 else np.float32
    x = torch.from_numpy(rng.standard_normal(size=(n, n, n)).astype(dt)).cuda()
    c2 = _context_without_tma()
    try:
        a = ctx.fft_r2c(x)
        b = c2.fft_r2c(x)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
        assert torch.equal(ctx.fft_c2r(a), c2.fft_c2r(b))
    finally:
        c2.close()


@pytest.mark.parametrize("scheme", [NGP, CIC, TSC])
@pytest.mark.parametrize("n,nbins,ndel", [(64, 32, 1.0), (128, 64, 1.0), (96, 30, 1.5),
                                          (512, 256, 1.0), (768, 256, 1.5)])  # 8-column tiles at 768
def test_job_pk_binned_in_fft_equals_separate_binning(ctx, scheme, n, nbins, ndel):
    # cam_job_run bins P(k) inside the FFT's last column pass; the separate
    # binning kernel over the stored spectrum gives the same mode counts and
    # the same sums up to rounding: the fused pass forms each mode's
    # |F|^2 / W^2 in FP32 and sums runs of at most one tile row (16 or 8 modes) in FP32 (a few
    # units of 2^-24 per run) before its FP64 bins; the separate one is FP64
    # throughout
    box = 800.0
    x, y, z = synth.clumped(400_000, box, 4_000, 2.0, 0.8, seed=n + scheme)
    g = make_grid(n, box)
    opts = Context.pk_opts(scheme, nbins=nbins, ndel=ndel)
    job = ctx.job(x, y, z, None, g, scheme, F32, pk=opts)
    mesh = ctx.assign(x, y, z, None, g, scheme, F32).mesh
    sep = ctx.power(mesh, box, opts)
    assert np.array_equal(job["pk"].modes, sep.modes)
    floor = np.abs(sep.shot_noise) * np.ones(nbins)
    assert pk_rel_err(job["pk"].pk, sep.pk, floor) <= 2e-6
    # and with the T-web, where the x pass also writes the spectrum back
    job2 = ctx.job(x, y, z, None, g, scheme, F32, pk=opts, tweb=Context.tweb_opts(8.0, 0.0, 1e-5))
    assert np.array_equal(job2["pk"].pk, job["pk"].pk)
