"""GPU T-web and whole mesh jobs vs the FP64 oracle (through the C ABI).

Bars: labels identical to the oracle's except cells with an oracle
eigenvalue within the tie band (1e-5) of lambda_th -- those are counted and
reported, every other cell must match; eigenvalues within 1e-5 of the
oracle's, relative to the largest |lambda|; a job equals its stages run one
by one.
"""
import numpy as np
import pytest

import oracle as orc
from conftest import pk_rel_err
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, F64, NGP, TSC, Context, make_grid

pytestmark = pytest.mark.gpu

BAND = 1e-5


def label_check(labels, lam_ref, lab_ref, lth):
    near = np.any(np.abs(lam_ref.reshape(-1, 3) - lth) <= BAND, axis=1).reshape(lab_ref.shape)
    bad = (labels != lab_ref) & ~near
    return int(bad.sum()), int(((labels != lab_ref) & near).sum()), int(near.sum())


@pytest.mark.parametrize("n,box,R,lth,prec", [
    (64, 1000.0, 8.0, 0.0, F32),
    (48, 600.0, 20.0, 0.1, F32),
    (64, 1000.0, 8.0, 0.0, F64),
    (32, 300.0, 0.0, 0.0, F32),
])
def test_tweb_vs_oracle(ctx, n, box, R, lth, prec):
    x, y, z = synth.clumped(400_000, box, 4_000, 2.0 * box / n, 0.8, seed=n)
    mesh, _ = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))
    mesh = mesh.astype(np.float64 if prec == F64 else np.float32)
    got = ctx.tweb(mesh, box, Context.tweb_opts(R, lth, BAND), want_lambdas=True)
    ref = orc.tweb_density(mesh.astype(np.float64), box, R, lth, BAND)
    bad, in_band, near = label_check(got.labels, ref.lam, ref.labels, lth)
    assert bad == 0, (bad, in_band, near)
    assert np.array_equal(np.bincount(got.labels.ravel(), minlength=5)[1:], got.counts)
    lam = np.moveaxis(got.lambdas, 0, -1).astype(np.float64)
    scale = np.abs(ref.lam).max()
    assert np.max(np.abs(lam - ref.lam)) <= 1e-5 * scale
    # tie accounting: the GPU counts cells within the band of its own lambdas
    assert abs(got.ties - ref.ties) <= max(2, ref.ties // 10)


def test_tweb_delta_input(ctx):
    n, box = 32, 200.0
    rng = np.random.default_rng(4)
    delta = rng.normal(size=(n, n, n)).astype(np.float32)
    got = ctx.tweb(delta, box, Context.tweb_opts(5.0, 0.0, BAND, input_type=1), want_lambdas=True)
    ref = orc.tweb_from_spectrum(orc.rfft3_f64(delta.astype(np.float64)), n, box, 5.0, 0.0, BAND)
    bad, _, _ = label_check(got.labels, ref.lam, ref.labels, 0.0)
    assert bad == 0


def oracle_job(x, y, z, w, n, box, scheme, nbins, R, lth, precision):
    mesh, lost = orc.assign_f64(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    if precision == F32:
        mesh = mesh.astype(np.float32).astype(np.float64)
    pk = orc.power_grid(mesh, box, scheme, nbins)
    tw = orc.tweb_density(mesh, box, R, lth, BAND) if R is not None else None
    return mesh, lost, pk, tw


@pytest.mark.parametrize("scheme", [NGP, CIC, TSC])
def test_job_vs_oracle(ctx, scheme):
    n, box, nbins, R, lth = 64, 500.0, 32, 8.0, 0.0
    cfg = synth.config_c5_job(job=scheme)
    x, y, z = cfg["x"], cfg["y"], cfg["z"]
    g = make_grid(n, box)
    res = ctx.job(x, y, z, None, g, scheme, F32, pk=Context.pk_opts(scheme, nbins=nbins),
                  tweb=Context.tweb_opts(R, lth, BAND), want_labels=True)
    mesh, lost, pk, tw = oracle_job(x, y, z, None, n, box, scheme, nbins, R, lth, F32)
    assert res["assign"].n_lost == lost
    floor = pk.shot_noise * pk.sum_sn / np.maximum(pk.modes, 1)
    assert np.array_equal(res["pk"].modes, pk.modes)
    assert pk_rel_err(res["pk"].pk, pk.pk, floor) <= 1e-5
    bad, _, _ = label_check(res["tweb"].labels, tw.lam, tw.labels, lth)
    assert bad == 0


def test_job_equals_stages(ctx):
    n, box = 64, 1000.0
    x, y, z = synth.clumped(300_000, box, 3_000, 2.0, 0.8, seed=31)
    w = synth.halo_masses(x.size, seed=32)
    g = make_grid(n, box)
    res = ctx.job(x, y, z, w, g, TSC, F32, pk=Context.pk_opts(TSC, nbins=32),
                  tweb=Context.tweb_opts(8.0, 0.0, BAND), want_labels=True)
    mesh = ctx.assign(x, y, z, w, g, TSC, F32).mesh
    pk = ctx.power(mesh, box, Context.pk_opts(TSC, nbins=32))
    tw = ctx.tweb(mesh, box, Context.tweb_opts(8.0, 0.0, BAND))
    # the job bins P(k) inside its FFT pass with each mode's power in FP32
    # (FP64 bins), the stage path in FP64 throughout: equal to FP32 rounding
    np.testing.assert_allclose(res["pk"].pk, pk.pk, rtol=2e-6)
    assert np.array_equal(res["tweb"].labels, tw.labels)


def test_job_fp64_mesh_c1_shape(ctx):
    # Config 1 at reduced particle count: CIC onto an FP64 128^3 mesh, 64 bins.
    n, box = 128, 1000.0
    x, y, z = synth.clumped(400_000, box, 4_000, 2.0, 0.8, seed=1)
    g = make_grid(n, box)
    res = ctx.job(x, y, z, None, g, CIC, F64, pk=Context.pk_opts(CIC, nbins=64))
    mesh, lost, pk, _ = oracle_job(x, y, z, None, n, box, CIC, 64, None, 0.0, F64)
    floor = pk.shot_noise * pk.sum_sn / np.maximum(pk.modes, 1)
    # FP64 mesh and FFT; the stencil weights are FP32 products (~1e-7)
    assert pk_rel_err(res["pk"].pk, pk.pk, floor) <= 1e-6


def test_job_payload_estimate_overflow_reruns():
    # Every particle's CIC stencil crosses a brick face along all three axes
    # (home cell 31 ends a brick for every power-of-two brick extent <= 32),
    # so each gives 8 records and one brick receives all 60,000 of its
    # particles: the first job of a fresh context overflows the payload
    # estimate and reruns exactly; the second finds the grown payload, but
    # slabs of the fullest brick too costly, and runs once on the exact path.
    n, box, nbins = 64, 64.0, 24
    rng = np.random.default_rng(41)
    npart = 60_000
    x, y, z = (rng.uniform(31.5, 32.5, npart).astype(np.float32) for _ in range(3))
    w = synth.halo_masses(npart, seed=42)
    g = make_grid(n, box)
    opts = Context.pk_opts(CIC, nbins=nbins)
    c = Context(0)
    try:
        l0 = c.kernel_launches
        r1 = c.job(x, y, z, w, g, CIC, F32, pk=opts)
        l1 = c.kernel_launches
        r2 = c.job(x, y, z, w, g, CIC, F32, pk=opts)
        l2 = c.kernel_launches
        mesh = c.assign(x, y, z, w, g, CIC, F32).mesh
        pk = c.power(mesh, box, opts)
    finally:
        c.close()
    assert l1 - l0 > l2 - l1  # the first job ran twice
    assert r1["assign"].n_lost == 0 and r1["assign"].n_in == npart
    assert np.array_equal(r1["pk"].pk, r2["pk"].pk)
    # fused FP32-per-mode binning against the FP64 stage path
    np.testing.assert_allclose(r1["pk"].pk, pk.pk, rtol=2e-6)
    _, lost, opk, _ = oracle_job(x, y, z, w, n, box, CIC, nbins, None, 0.0, F32)
    assert lost == 0
    floor = opk.shot_noise * opk.sum_sn / np.maximum(opk.modes, 1)
    assert np.array_equal(r1["pk"].modes, opk.modes)
    assert pk_rel_err(r1["pk"].pk, opk.pk, floor) <= 1e-5


def test_job_slabs_measured_overflow_reruns():
    # A context's first job of a mesh shape runs exactly and measures its
    # fullest brick; later jobs write per-brick slabs sized from it (no
    # count pass).  A more concentrated catalogue overflows them: the job
    # reruns exactly, measures again, and the next job fits its slabs.
    # Every result equals a fresh context's exact run bit for bit.
    n, box, nbins = 128, 1000.0, 32
    npart = 400_000
    rng = np.random.default_rng(5)
    ux, uy, uz = (rng.uniform(0.0, box, npart).astype(np.float32) for _ in range(3))
    # density rising towards x = 0: the fullest brick holds 2,942 TSC
    # records against 2,229 of the uniform catalogue (2,101 expected), past
    # the uniform catalogue's slabs of 2,588
    cx = (box * (ux.astype(np.float64) / box) ** 1.2).astype(np.float32)
    w = synth.halo_masses(npart, seed=6)
    g = make_grid(n, box)
    opts = Context.pk_opts(TSC, nbins=nbins)
    c = Context(0)
    try:
        launches = []
        res = []
        for xs in (ux, ux, cx, cx):
            l0 = c.kernel_launches
            res.append(c.job(xs, uy, uz, w, g, TSC, F32, pk=opts))
            launches.append(c.kernel_launches - l0)
    finally:
        c.close()
    exact, slab, rerun, slab2 = launches
    assert slab < exact          # no count pass, scan or brick measure
    assert rerun > exact         # the slab run, then the exact one
    assert slab2 == slab         # the measured slabs hold the new catalogue
    assert np.array_equal(res[0]["pk"].pk, res[1]["pk"].pk)
    assert np.array_equal(res[2]["pk"].pk, res[3]["pk"].pk)
    f = Context(0)
    try:
        fresh = f.job(cx, uy, uz, w, g, TSC, F32, pk=opts)
    finally:
        f.close()
    assert np.array_equal(fresh["pk"].pk, res[3]["pk"].pk)
    assert np.array_equal(fresh["pk"].modes, res[3]["pk"].modes)
    assert res[3]["assign"].n_lost == 0 and res[3]["assign"].n_in == npart
    _, lost, opk, _ = oracle_job(cx, uy, uz, w, n, box, TSC, nbins, None, 0.0, F32)
    floor = opk.shot_noise * opk.sum_sn / np.maximum(opk.modes, 1)
    assert pk_rel_err(res[3]["pk"].pk, opk.pk, floor) <= 1e-5
