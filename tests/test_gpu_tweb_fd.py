"""GPU finite-difference T-web -- the reference's default build
(_USE_GFINDIFF_EIGENV_, Headers/def.h:2657) -- with PoissonSolver and
gradfindif, through the C ABI, against the FP64 oracle that restates the
reference loops (Poisson solve, two centred differences per component).

Bars: labels identical except cells with an oracle eigenvalue within the
tie band (1e-5) of lambda_th; eigenvalues within 1e-5 of the largest
|lambda|; the potential within 1e-5 of its largest |phi| (FP32) or 1e-12
(FP64); gradfindif bit-identical to the reference's FP32 arithmetic.
"""
import numpy as np
import pytest

import oracle as orc
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import (CIC, F32, F64, TSC, CamError, Context, Cwclass, JobSpec, Params,
                                  make_grid)

pytestmark = pytest.mark.gpu

BAND = 1e-5
FD = L.TWEB_FD


def label_check(labels, lam_ref, lab_ref, lth):
    near = np.any(np.abs(lam_ref.reshape(-1, 3) - lth) <= BAND, axis=1).reshape(lab_ref.shape)
    return int(((labels != lab_ref) & ~near).sum())


@pytest.mark.parametrize("n,box,R,lth,prec", [
    (64, 1000.0, 8.0, 0.0, F32),     # the small plain config's T-web settings
    (48, 600.0, 20.0, 0.1, F32),     # mixed-radix length, lambda_th > 0
    (128, 1000.0, 3.0, 0.1, F32),    # the large config's R and lambda_th
    (64, 1000.0, 8.0, 0.0, F64),
    (32, 300.0, 0.0, 0.0, F32),      # no smoothing
])
def test_fd_tweb_vs_oracle(ctx, n, box, R, lth, prec):
    x, y, z = synth.clumped(400_000, box, 4_000, 2.0 * box / n, 0.8, seed=n + 7)
    mesh, _ = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))
    mesh = mesh.astype(np.float64 if prec == F64 else np.float32)
    got = ctx.tweb(mesh, box, Context.tweb_opts(R, lth, BAND, method=FD), want_lambdas=True)
    ref = orc.tweb_fd_density(mesh.astype(np.float64), box, R, lth, BAND)
    assert label_check(got.labels, ref.lam, ref.labels, lth) == 0
    assert np.array_equal(np.bincount(got.labels.ravel(), minlength=5)[1:], got.counts)
    lam = np.moveaxis(got.lambdas, 0, -1).astype(np.float64)
    assert np.max(np.abs(lam - ref.lam)) <= 1e-5 * np.abs(ref.lam).max()
    assert abs(got.ties - ref.ties) <= max(2, ref.ties // 10)


def test_fd_tweb_of_a_potential(ctx):
    # EigenValuesTweb(Nft, L, delta, phi, ...): the Hessian of a given potential
    n, box = 48, 400.0
    delta = np.random.default_rng(21).normal(size=(n, n, n)).astype(np.float32)
    phi = orc.poisson_f64(orc.rfft3_f64(delta.astype(np.float64)), n, box, 12.0).astype(np.float32)
    got = ctx.tweb(phi, box, Context.tweb_opts(0.0, 0.0, BAND, input_type=L.INPUT_POTENTIAL, method=FD),
                   want_lambdas=True)
    ref = orc.tweb_fd_potential(phi.astype(np.float64), box, 0.0, BAND)
    assert label_check(got.labels, ref.lam, ref.labels, 0.0) == 0
    lam = np.moveaxis(got.lambdas, 0, -1).astype(np.float64)
    assert np.max(np.abs(lam - ref.lam)) <= 1e-5 * np.abs(ref.lam).max()


def test_potential_input_needs_fd(ctx):
    phi = np.zeros((16, 16, 16), np.float32)
    with pytest.raises(CamError) as e:
        ctx.tweb(phi, 100.0, Context.tweb_opts(0.0, 0.0, BAND, input_type=L.INPUT_POTENTIAL))
    assert e.value.code == L.CAM_E_INVAL
    with pytest.raises(CamError):
        ctx.tweb(phi, 100.0, Context.tweb_opts(0.0, 0.0, BAND, method=7))


@pytest.mark.parametrize("n,R,prec", [(64, 0.0, F32), (48, 15.0, F32), (64, 0.0, F64)])
def test_poisson_vs_oracle(ctx, n, R, prec):
    box = 500.0
    delta = np.random.default_rng(n).normal(size=(n, n, n)).astype(np.float64 if prec == F64 else np.float32)
    got = ctx.poisson(delta, box, R)
    ref = orc.poisson_f64(orc.rfft3_f64(delta.astype(np.float64)), n, box, R)
    tol = 1e-12 if prec == F64 else 1e-5
    assert np.max(np.abs(got - ref)) <= tol * np.abs(ref).max()


def test_gradfindif_bit_exact(ctx):
    import torch
    n, box = 40, 700.0
    f = np.random.default_rng(2).normal(size=(n, n, n)).astype(np.float32) * 3.0
    for dim in (1, 2, 3):
        got = ctx.gradfindif(f, box, dim)
        assert np.array_equal(got, orc.gradfindif_ref_f32(f, dim - 1, box)), dim
        f64 = f.astype(np.float64)
        np.testing.assert_allclose(ctx.gradfindif(f64, box, dim), orc.gradfindif_f64(f64, dim - 1, box),
                                   rtol=0, atol=1e-13 * np.abs(f64).max())
    # device arrays, output over its own input (the reference takes `in` by value)
    t = torch.from_numpy(f).cuda()
    ctx.gradfindif(t, box, 1, out=t)
    ctx.sync()
    assert np.array_equal(t.cpu().numpy(), orc.gradfindif_ref_f32(f, 0, box))


def test_fd_job_and_batch(ctx):
    # a whole mesh job with the FD T-web, its labels against the oracle of its
    # own FP32 mesh, and the same jobs through a captured-graph batch
    n, box, R = 64, 500.0, 8.0
    opts = Context.tweb_opts(R, 0.0, BAND, method=FD)
    jobs = []
    for s in range(3):
        x, y, z = synth.clumped(150_000, box, 1_500, 2.0, 0.7, seed=600 + s)
        jobs.append((x, y, z))
    g = make_grid(n, box)
    x, y, z = jobs[0]
    res = ctx.job(x, y, z, None, g, TSC, F32, pk=Context.pk_opts(TSC, nbins=32), tweb=opts, want_labels=True)
    mesh = ctx.assign(x, y, z, None, g, TSC, F32).mesh
    ref = orc.tweb_fd_density(mesh.astype(np.float64), box, R, 0.0, BAND)
    assert label_check(res["tweb"].labels, ref.lam, ref.labels, 0.0) == 0
    alone = [ctx.job(*j, None, g, TSC, F32, pk=Context.pk_opts(TSC, nbins=32), tweb=opts) for j in jobs]
    for rep in range(2):
        got = ctx.batch([JobSpec(*j, None, grid=g, scheme=TSC, precision=F32, pk=Context.pk_opts(TSC, nbins=32),
                                 tweb=opts) for j in jobs])
        for a, b in zip(got, alone):
            assert np.array_equal(a["tweb"].counts, b["tweb"].counts) and a["tweb"].ties == b["tweb"].ties
    # FFT and FD jobs of the same shape must not share a captured graph
    fft = ctx.batch([JobSpec(*j, None, grid=g, scheme=TSC, precision=F32, pk=Context.pk_opts(TSC, nbins=32),
                             tweb=Context.tweb_opts(R, 0.0, BAND)) for j in jobs])
    want = [ctx.job(*j, None, g, TSC, F32, pk=Context.pk_opts(TSC, nbins=32), tweb=Context.tweb_opts(R, 0.0, BAND))
            for j in jobs]
    for a, b in zip(fft, want):
        assert np.array_equal(a["tweb"].counts, b["tweb"].counts)


def test_cwclass_default_build_variant():
    # Cwclass::get_CWC through the reference-shaped mirror with the FD tensor
    n, box = 32, 250.0
    x, y, z = synth.clumped(100_000, box, 1_000, 3.0, 0.8, seed=71)
    mesh, _ = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))
    mesh = mesh.astype(np.float32)
    cw = Cwclass(Params(Nft=n, Lbox=box, smoothing_R=10.0, lambdath=0.0, tweb_method="fd"))
    cw.get_CWC(mesh.ravel())
    ref = orc.tweb_fd_density(mesh.astype(np.float64), box, 10.0, 0.0, BAND)
    assert label_check(cw.CWClass.reshape(n, n, n), ref.lam, ref.labels, 0.0) == 0
    assert abs(cw.volume_voids - ref.counts[3] / n ** 3) <= (ref.ties + 1) / n ** 3


@pytest.mark.parametrize("method", [L.TWEB_FFT, FD])
def test_tidal_invariants(ctx, method):
    # invariant_field_I/II/III and tidal_anisotropy of the oracle eigenvalues
    n, box, R = 48, 600.0, 15.0
    x, y, z = synth.clumped(300_000, box, 3_000, 4.0, 0.8, seed=81)
    mesh = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))[0].astype(np.float32)
    labels, lam, inv = ctx.tweb_invariants(mesh, box, Context.tweb_opts(R, 0.0, BAND, method=method))
    ref = (orc.tweb_fd_density if method == FD else orc.tweb_density)(mesh.astype(np.float64), box, R, 0.0, BAND)
    want = orc.tidal_invariants(ref.lam)
    scale = np.abs(ref.lam).max()
    assert np.max(np.abs(inv[0] - want[0])) <= 1e-5 * scale
    assert np.max(np.abs(inv[1] - want[1])) <= 1e-5 * scale * scale
    assert np.max(np.abs(inv[2] - want[2])) <= 1e-5 * scale ** 3
    assert np.max(np.abs(inv[3] - want[3])) <= 1e-4 * np.abs(want[3]).max()
    assert label_check(labels, ref.lam, ref.labels, 0.0) == 0
    np.testing.assert_allclose(np.moveaxis(lam, 0, -1), ref.lam, rtol=0, atol=1e-5 * scale)
