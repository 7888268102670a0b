"""GPU BAM kernel steps through the C ABI: the 3D update of Bam::GetKernel
(Source/Bam.cpp:786-910) and Bam::Konvolve (Source/Bam.cpp:1027-1120),
against the oracle.

Bars: the updated kernel and its bins bit-identical to the reference's
real_prec loops; bin means within 1e-12 (FP64 sums of the same values);
Konvolve within 1e-5 of the largest |out| (FP32) or 1e-12 (FP64) of the FP64
oracle.
"""
import numpy as np
import pytest

import oracle as orc
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, Bam, CamError, Context, Params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,box,kmin_u,ndel,nb,prec", [
    (64, 500.0, 0.0, 1.0, 32, np.float32),    # the calibration batch's binning
    (48, 333.0, 0.5, 1.5, 16, np.float32),    # kmin > 0, wide bins, mixed-radix N
    (32, 1000.0, 0.0, 1.0, 16, np.float64),
])
@pytest.mark.parametrize("mode", [L.KERNEL_SET, L.KERNEL_SCALE])
def test_kernel_update_bit_exact(ctx, n, box, kmin_u, ndel, nb, prec, mode):
    rng = np.random.default_rng(n + mode)
    k0 = rng.uniform(0.5, 1.5, size=(n, n, n // 2 + 1)).astype(prec)
    w = rng.uniform(0.8, 1.25, size=nb).astype(np.float32).astype(np.float64)
    got = k0.copy()
    binned, modes = ctx.bam_kernel_update(got, box, w, mode, kmin_u, ndel)
    want, wbinned, wmodes = orc.bam_kernel_update_ref(k0, box, w, mode == L.KERNEL_SCALE, kmin_u, ndel)
    assert np.array_equal(got, want)
    assert np.array_equal(modes, wmodes)
    np.testing.assert_allclose(binned, wbinned, rtol=1e-12)


def test_kernel_update_on_device(ctx):
    import torch
    n, box, nb = 64, 500.0, 32
    k0 = np.ones((n, n, n // 2 + 1), np.float32)
    w = np.linspace(0.9, 1.1, nb)
    t = torch.from_numpy(k0).cuda()
    for _ in range(3):  # repeated rejection-style updates compound on the device
        ctx.bam_kernel_update(t, box, w, L.KERNEL_SCALE)
    want = k0
    for _ in range(3):
        want, _, _ = orc.bam_kernel_update_ref(want, box, w, True)
    assert np.array_equal(t.cpu().numpy(), want)


def test_kernel_update_rejects_bad_arguments(ctx):
    k = np.ones((16, 16, 9), np.float32)
    with pytest.raises(CamError):
        ctx.bam_kernel_update(k, 100.0, np.ones(4))          # bin 0 needs bins 1..4
    with pytest.raises(CamError):
        ctx.bam_kernel_update(k, 100.0, np.ones(8), mode=5)


@pytest.mark.parametrize("n,prec,tol", [(64, np.float32, 1e-5), (48, np.float32, 1e-5), (32, np.float64, 1e-12)])
def test_konvolve_vs_oracle(ctx, n, prec, tol):
    box = 500.0
    rng = np.random.default_rng(n)
    x, y, z = synth.clumped(200_000, box, 2_000, 3.0, 0.7, seed=n)
    mesh, _ = orc.assign_f64(CIC, x, y, z, None, orc.Grid.cubic(n, box))
    delta = (mesh / mesh.mean() - 1.0).astype(prec)
    kern = rng.uniform(0.7, 1.3, size=(n, n, n // 2 + 1)).astype(prec)
    got = ctx.konvolve(delta, box, kern)
    want = orc.konvolve_f64(delta, kern, n)
    assert np.max(np.abs(got - want)) <= tol * np.abs(want).max()


def test_konvolve_in_place_and_nonfinite(ctx):
    import torch
    n, box = 32, 200.0
    rng = np.random.default_rng(3)
    d = rng.normal(size=(n, n, n)).astype(np.float32)
    kern = rng.uniform(0.5, 1.5, size=(n, n, n // 2 + 1)).astype(np.float32)
    t = torch.from_numpy(d).cuda()
    tk = torch.from_numpy(kern).cuda()
    ctx.konvolve(t, box, tk, out=t)  # Konvolve(x, x), as the reference calls it
    ctx.sync()
    want = orc.konvolve_f64(d, kern, n)
    assert np.max(np.abs(t.cpu().numpy() - want)) <= 1e-5 * np.abs(want).max()
    d[3, 4, 5] = np.inf
    with pytest.raises(CamError) as e:
        ctx.konvolve(d, box, kern)
    assert e.value.code == L.CAM_E_NONFINITE


def test_bam_iteration_mirror():
    # GetKernel (no rejection, exponent 0.5) then Konvolve, through the
    # reference-shaped Bam class: P_ref / P_new ratios as weights
    n, box = 64, 500.0
    p = Params(Nft=n, Lbox=box)
    bam = Bam(p)
    nb = bam.kvec.size
    rng = np.random.default_rng(8)
    bam.kvec = (np.arange(nb) + 0.5) * 2 * np.pi / box
    bam.Power_REF = rng.uniform(1e3, 2e3, nb)
    bam.Power_NEW = rng.uniform(1e3, 2e3, nb)
    bam.GetKernel(False, 0.5)
    w = (np.abs(bam.Power_REF / bam.Power_NEW) ** 0.5).astype(np.float32).astype(np.float64)
    want, wbinned, _ = orc.bam_kernel_update_ref(np.ones((n, n, n // 2 + 1), np.float32), box, w, False)
    assert np.array_equal(bam.Kernel.cpu().numpy(), want)
    np.testing.assert_allclose(bam.kernel_updated, wbinned, rtol=1e-12)
    delta = rng.normal(size=(n, n, n)).astype(np.float32)
    out = np.empty_like(delta)
    bam.Konvolve(delta, out)
    ref = orc.konvolve_f64(delta, want, n)
    assert np.max(np.abs(out - ref)) <= 1e-5 * np.abs(ref).max()
    # with rejection: the MT19937 draws of seed 55457 decide per bin
    bam.power_ratio_unsmoothed = np.ones(nb) * 1.05
    k_before = bam.Kernel.cpu().numpy()
    bam.GetKernel(True, 1.0)
    assert np.all(np.isfinite(bam.Kernel.cpu().numpy()))
    changed = np.any(bam.Kernel.cpu().numpy() != k_before)
    assert changed


# ---------------------------------------------------------------- catalogue interpolation
def test_fkp_weights_and_interpolation(ctx):
    # Catalog.cpp's tracer loop: per-object nbar, an extra weight, FKP on
    from cosmicatlas_b200.api import get_interpolated_density_field, make_grid
    n, box, npart = 64, 500.0, 200_000
    x, y, z = synth.clumped(npart, box, 2_000, 3.0, 0.7, seed=91)
    rng = np.random.default_rng(92)
    nbar = rng.uniform(1e-4, 3e-3, npart).astype(np.float32)
    w1 = rng.uniform(0.5, 2.0, npart).astype(np.float32)
    w, sums = ctx.fkp_weights(npart, nbar, 0.0, w1, True, 1e4)
    wref, sref = orc.fkp_weights_f64(nbar, w1, True, 1e4)
    np.testing.assert_allclose(w, wref.astype(np.float32), rtol=1e-7)
    np.testing.assert_allclose(sums, sref, rtol=1e-12)
    mesh, s2 = get_interpolated_density_field(x, y, z, make_grid(n, box), CIC, nbar, 0.0, w1, True, 1e4)
    ref, _ = orc.assign_f64(CIC, x, y, z, wref.astype(np.float32), orc.Grid.cubic(n, box))
    from conftest import rel_err_cells
    assert rel_err_cells(mesh, ref, float(wref.mean())) <= 1e-5
    # constant nbar (no random catalogue), no extra weights, FKP off: unit weights
    w, sums = ctx.fkp_weights(1000, None, 2e-3, None, False, 1e4)
    assert np.all(w == 1.0) and sums[1] == 1000.0 and abs(sums[3] - 2.0) < 1e-12

