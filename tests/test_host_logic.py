"""Host logic of the Python mirror (no GPU): the per-bin weights of
Bam::GetKernel (Source/Bam.cpp:604-723), which stay on the host because they
are one value per bin."""
import numpy as np
import pytest

from cosmicatlas_b200.api import Bam, Params


def make_bam(nb=16, box=500.0):
    b = Bam.__new__(Bam)  # no device kernel: only the host weight loop is exercised
    b.params = Params(Nft=2 * nb, Lbox=box)
    b.kvec = (np.arange(nb) + 0.5) * 2 * np.pi / box
    b.Power_REF = np.linspace(1000.0, 2000.0, nb)
    b.Power_NEW = np.linspace(1500.0, 1000.0, nb)
    b.power_ratio_unsmoothed = np.ones(nb)
    b.shot_noise_ref = 10.0
    return b


def test_weights_without_rejection_are_the_power_ratio():
    b = make_bam()
    w = b.kernel_weights(False, 0.5)
    np.testing.assert_allclose(w, (b.Power_REF / b.Power_NEW) ** 0.5, rtol=1e-7)  # rounded to real_prec
    assert np.array_equal(w, w.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(b.power_ratio_unsmoothed, (b.Power_REF / b.Power_NEW) ** 0.5)
    # exponent >= 1: the plain ratio (Source/Bam.cpp:621-626); P_new = 0 gives 1
    b = make_bam()
    b.Power_NEW[3] = 0.0
    w = b.kernel_weights(False, 1.0)
    assert w[3] == 1.0 and w[4] == pytest.approx(b.Power_REF[4] / b.Power_NEW[4], rel=1e-7)


def test_rejection_accepts_by_the_chi2_ratio():
    # accepted bins take the new ratio, rejected ones keep weight 1; the draw
    # is compared with min(1, chi2_old / chi2_new) (Source/Bam.cpp:700-713)
    b = make_bam()
    b.power_ratio_unsmoothed = np.full(16, 1.02)
    w_all = b.kernel_weights(True, 1.0, uniforms=np.zeros(16))  # every draw below the ratio
    ratio = b.Power_REF / b.Power_NEW
    np.testing.assert_allclose(w_all, ratio, rtol=1e-7)
    b = make_bam()
    b.power_ratio_unsmoothed = np.full(16, 1.02)
    w_none = b.kernel_weights(True, 1.0, uniforms=np.full(16, 1.0 - 1e-12))
    # a draw just below 1 is accepted only where chi2_old >= chi2_new
    dk = 2 * np.pi / 500.0
    sfac = 1.0 / (2 * np.pi * dk * 500.0 ** 3)
    inv = sfac / (b.kvec ** 2 + dk * dk / 12)
    new_h = 0.5 * (b.Power_REF - b.Power_NEW) ** 2 / (inv * b.Power_NEW ** 2)
    p_old = b.Power_REF / 1.02
    old_h = 0.5 * (b.Power_REF - p_old) ** 2 / (inv * (p_old + 10.0) ** 2)
    acc = old_h / new_h > 1.0 - 1e-12
    np.testing.assert_allclose(w_none[acc], ratio[acc], rtol=1e-7)
    assert np.all(w_none[~acc] == 1.0)
    # the unsmoothed ratio is updated in every bin, accepted or not
    np.testing.assert_allclose(b.power_ratio_unsmoothed, ratio)


def test_default_draws_are_mt19937_of_seed_55457():
    # gsl_rng_mt19937 seeded by init_genrand: the reference MT19937 stream
    # (its first output for seed 5489 is 3499211612); one 32-bit output / 2^32 per bin
    rs = np.random.RandomState(5489)
    assert int(rs.randint(0, 2 ** 32, dtype=np.uint64)) == 3499211612
    b = make_bam()
    b.power_ratio_unsmoothed = np.full(16, 1.02)
    w_default = b.kernel_weights(True, 1.0)
    b2 = make_bam()
    b2.power_ratio_unsmoothed = np.full(16, 1.02)
    u = np.random.RandomState(Bam.SEED).randint(0, 2 ** 32, size=16, dtype=np.uint64) / 4294967296.0
    assert np.array_equal(w_default, b2.kernel_weights(True, 1.0, uniforms=u))
