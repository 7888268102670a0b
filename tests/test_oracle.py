"""Pins the CPU oracle (no GPU).

The reference ships no golden vectors, so the oracle is pinned against
known answers derived by hand from the reference source:
  * cell keys at chosen positions, following the float arithmetic of
    getDensity_NGP/CIC/TSC (Source/massFunctions.cpp:57-69, :700-737, :1076-1089);
  * single-particle CIC/TSC weights (massFunctions.cpp:743-769, :1098-1162);
  * the power spectrum of a plane wave (FftwFunctions.cpp:1660-1876);
  * eigenvalues of matrices with known spectra and the label rule
    (Cwclass.cpp:875-890);
and against the reference loops as written (the FP32 restatement).
"""
import numpy as np
import pytest

import oracle as orc


def grid(n, box=1000.0):
    return orc.Grid.cubic(n, box)


# ---------------------------------------------------------------- keys
def test_ngp_keys_known_positions():
    # N = 8, L = 1000, d = 125 (exact in float)
    g = grid(8)
    x = np.array([0.0, 124.99999, 125.0, np.nextafter(np.float32(1000), 0), 1000.0, -1e-3, 500.0], np.float32)
    y = np.full_like(x, 250.0)   # cell 2
    z = np.full_like(x, 0.0)     # cell 0
    k = orc.keys(orc.NGP, x, y, z, g)
    lost = 8 ** 3
    # x: 0 -> 0; 124.99999 -> 0; 125 -> 1; 999.99994 -> 7; 1000 -> lost (x < L);
    # -0.001 -> lost; 500 -> 4.  key = k + N*(j + N*i) with j = 2, k = 0.
    expect = [0 * 64 + 16, 16, 64 + 16, 7 * 64 + 16, lost, lost, 4 * 64 + 16]
    assert k.tolist() == expect


def test_cic_and_tsc_keys_known_positions():
    g = grid(8)
    # CIC: xpos = x - d/2 wrapped once: x = 10 -> -52.5 + 1000 = 947.5 -> cell 7;
    # x = 62.5 -> 0 -> cell 0; x = 1000 -> 937.5 -> cell 7 (accepted after wrap).
    x = np.array([10.0, 62.5, 1000.0, 187.5], np.float32)
    y = np.full_like(x, 62.5)
    z = np.full_like(x, 62.5)
    k = orc.keys(orc.CIC, x, y, z, g)
    assert k.tolist() == [7 * 64, 0, 7 * 64, 1 * 64]
    # TSC accepts x == L (closed interval) and wraps its cell 8 to 0.
    x = np.array([1000.0, 999.0, 0.0], np.float32)
    k = orc.keys(orc.TSC, x, np.zeros_like(x), np.zeros_like(x), g)
    assert k.tolist() == [0, 7 * 64, 0]
    k = orc.keys(orc.TSC, np.array([1000.5], np.float32), np.zeros(1, np.float32), np.zeros(1, np.float32), g)
    assert k.tolist() == [8 ** 3]


def test_keys_follow_float_division_not_double():
    # d = L / N rounded to float (1000/384 is not representable).  Scan many
    # positions and check the key against an explicit float32 recomputation.
    g = orc.Grid.cubic(384, 1000.0)
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 1000, 200_000).astype(np.float32)
    d = np.float32(g.d[0])
    i = np.floor((x - np.float32(0)) / d).astype(np.int64) % 384
    k = orc.keys(orc.NGP, x, np.zeros_like(x), np.zeros_like(x), g)
    assert np.array_equal(k, i * 384 * 384)


# ---------------------------------------------------------------- weights
@pytest.mark.parametrize("t", [0.0, 0.25, 0.5, 0.9375])
def test_single_particle_cic_weights(t):
    n, box = 8, 1000.0
    g = grid(n, box)
    d = box / n
    # node i sits at (i + 1/2) d; a particle at (3 + 1/2 + t) d
    xv = np.float32((3.5 + t) * d)
    mesh, lost = orc.assign_f64(orc.CIC, np.array([xv]), np.array([xv]), np.array([xv]), np.array([2.0], np.float32), g)
    assert lost == 0
    w1 = np.array([1 - t, t])
    expect = np.zeros((n, n, n))
    for a in range(2):
        for b in range(2):
            for c in range(2):
                expect[3 + a, 3 + b, 3 + c] = 2.0 * w1[a] * w1[b] * w1[c]
    np.testing.assert_allclose(mesh, expect, atol=1e-12)


@pytest.mark.parametrize("t", [-0.5, -0.2, 0.0, 0.3])
def test_single_particle_tsc_weights(t):
    n, box = 8, 1000.0
    g = grid(n, box)
    d = box / n
    xv = np.float32((4.5 + t) * d)   # cell 4, offset t from its centre
    mesh, lost = orc.assign_f64(orc.TSC, np.array([xv]), np.array([xv]), np.array([xv]), None, g)
    w1 = np.array([0.5 * (0.5 - t) ** 2, 0.75 - t * t, 0.5 * (0.5 + t) ** 2])
    expect = np.zeros((n, n, n))
    for a in range(3):
        for b in range(3):
            for c in range(3):
                expect[3 + a, 3 + b, 3 + c] = w1[a] * w1[b] * w1[c]
    np.testing.assert_allclose(mesh, expect, atol=1e-12)
    assert abs(mesh.sum() - 1.0) < 1e-12


def test_periodic_wrap_mass_conserved():
    g = grid(4, 100.0)
    x = np.array([0.1, 99.9, 50.0], np.float32)
    for s in (orc.NGP, orc.CIC, orc.TSC):
        mesh, lost = orc.assign_f64(s, x, x, x, None, g)
        assert lost == 0
        assert abs(mesh.sum() - 3.0) < 1e-12


def test_oracle_matches_reference_loop_as_written():
    # The FP32 reference loop computes dx = (xpos - min)/d - i in float, an
    # absolute error of ~ulp(N) ~ 2e-6 cells per weight; so the two agree to
    # that absolute level (relative to the largest cell), not per cell.
    rng = np.random.default_rng(3)
    g = grid(32, 1000.0)
    x, y, z = (rng.uniform(1, 999, 20_000).astype(np.float32) for _ in range(3))
    w = rng.uniform(0.5, 2.0, 20_000).astype(np.float32)
    for s in (orc.NGP, orc.CIC, orc.TSC):
        m64, l64 = orc.assign_f64(s, x, y, z, w, g)
        m32, l32 = orc.assign_ref(s, x, y, z, w, g)
        assert l64 == l32
        err = np.max(np.abs(m64 - m32)) / np.abs(m64).max()
        assert err < 1e-5, (s, err)
        assert abs(m64.sum() - m32.sum()) / m64.sum() < 1e-5


# ---------------------------------------------------------------- P(k)
def test_plane_wave_power():
    # delta(x) = A cos(2 pi m.x / N): |F(m)|^2 = (A N^3 / 2)^2, delta input
    # normal = N^6 / V, so P = A^2 V / 4 in the bin of |m| with one mode.
    n, box, A = 16, 100.0, 0.3
    i = np.arange(n)
    X, Y, Z = np.meshgrid(i, i, i, indexing="ij")
    m = (2, 1, 2)  # |m| = 3
    delta = A * np.cos(2 * np.pi * (m[0] * X + m[1] * Y + m[2] * Z) / n)
    r = orc.power_grid(delta, box, orc.NGP, nbins=8, input_type="delta", mas_corr=False, sn_corr=False)
    expect = np.zeros(8)
    expect[3] = A * A * box ** 3 / 4.0 / r.modes[3]
    np.testing.assert_allclose(r.pk, expect, atol=1e-9 * A * A * box ** 3)


def test_bins_edges_go_up():
    # |k| = 3 k_f exactly (a perfect square) lands in bin 3 with unit bins,
    # and in bin 2 with 1.5 k_f bins (edges 0, 1.5, 3, 4.5 -> 3 is edge of bin 2).
    assert orc.lib().orc_bin(9.0, 0.0, 1.0, 10) == 3
    assert orc.lib().orc_bin(9.0, 0.0, 1.5, 10) == 2
    assert orc.lib().orc_bin(8.99, 0.0, 1.5, 10) == 1
    assert orc.lib().orc_bin(0.25, 1.0, 1.0, 10) == -1
    assert orc.lib().orc_bin(1e6, 0.0, 1.0, 10) == -1


def test_mode_count_is_independent_modes():
    # default binning: every conjugate pair with 0 < |k| < k_Nyq counted once
    n = 16
    spec = np.zeros((n, n, n // 2 + 1), np.complex128)
    r = orc.power_from_spectrum(spec, n, 100.0, orc.NGP, n // 2, 1.0, 1.0)
    f = np.fft.fftfreq(n, 1.0 / n)
    K = np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + f[None, None, :] ** 2)
    full = np.bincount(np.floor(K[K > 0]).astype(int), minlength=64)[: n // 2]
    assert np.array_equal(r.modes * 2, full)


# ---------------------------------------------------------------- eigen / labels
def test_eigen_known_spectra():
    rng = np.random.default_rng(11)
    lam_true = np.array([[3.0, 1.0, -2.0], [0.5, 0.5, 0.5], [1e-3, -1e-3, -5.0], [2.0, 2.0, -1.0]])
    t6 = []
    for l in lam_true:
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        m = q @ np.diag(l) @ q.T
        t6.append([m[0, 0], m[1, 1], m[2, 2], m[0, 1], m[0, 2], m[1, 2]])
    t6 = np.array(t6)
    want = np.sort(lam_true, axis=1)[:, ::-1]
    np.testing.assert_allclose(orc.eig3_f64(t6), want, atol=1e-12)
    np.testing.assert_allclose(orc.eig3_closed(t6), want, atol=1e-7)


def test_label_truth_table():
    lam = np.array([[1.0, 0.5, 0.2], [1.0, 0.5, -0.2], [1.0, -0.5, -0.2], [-1.0, -0.5, -0.2],
                    [0.0, 0.0, 0.0], [0.1 + 1e-6, 0.1, 0.0]])
    labels, counts, ties = orc.classify(lam, 0.0, 1e-5)
    assert labels.tolist() == [1, 2, 3, 4, 4, 2]
    labels, counts, ties = orc.classify(lam[5:], 0.1, 1e-5)
    assert labels.tolist() == [3] and ties == 1


# ---------------------------------------------------------------- finite-difference T-web
def test_gradfindif_known_answer():
    # gradfindif (Source/NumericalMethods.cpp:1123-1218) of sin(2 pi f x / N)
    # along each axis: (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / (12 d) gives
    # (8 sin(t) - sin(2t)) / (6 d) cos(2 pi f x / N), t = 2 pi f / N; the
    # other axes are untouched.
    n, box, f = 16, 160.0, 3
    d = box / n
    t = 2 * np.pi * f / n
    x = np.arange(n)
    wave = np.sin(t * x)
    amp = (8 * np.sin(t) - np.sin(2 * t)) / (6 * d)
    for axis in range(3):
        shape = [1, 1, 1]
        shape[axis] = n
        field = np.broadcast_to(wave.reshape(shape), (n, n, n)).copy()
        want = np.broadcast_to((amp * np.cos(t * x)).reshape(shape), (n, n, n))
        np.testing.assert_allclose(orc.gradfindif_f64(field, axis, box), want, atol=1e-13)
    # five-point weights on a single spike: out[x] = (-in[x+2] + 8 in[x+1] - 8 in[x-1] + in[x-2]) / (12 d)
    spike = np.zeros((n, 1, 1))
    spike[5] = 1.0
    g = orc.gradfindif_f64(spike, 0, box)[:, 0, 0] * 12 * d
    assert np.allclose(g[[3, 4, 6, 7]], [-1.0, 8.0, -8.0, 1.0]) and np.count_nonzero(np.abs(g) > 1e-15) == 4


def test_poisson_inverts_laplacian():
    # PoissonSolver (Source/Miscelanious.cpp:1189-1275): nabla^2 phi = delta for a
    # zero-mean delta, with the spectral Laplacian -k^2.
    n, box = 16, 100.0
    delta = np.random.default_rng(3).normal(size=(n, n, n))
    delta -= delta.mean()
    phi = orc.poisson_f64(orc.rfft3_f64(delta), n, box)
    kf = 2 * np.pi / box
    f = orc.signed_freq(n)
    k2 = (f[:, None, None] ** 2 + f[None, :, None] ** 2 + np.arange(n // 2 + 1)[None, None, :] ** 2) * kf * kf
    np.testing.assert_allclose(orc.irfft3_f64(-k2 * orc.rfft3_f64(phi), n), delta, atol=1e-10)


def test_fd_tidal_tensor_is_a_fourier_multiplier():
    # On a periodic mesh the centred difference is the Fourier multiplier
    # i s(k), s(k) = (8 sin kd - sin 2kd) / (6 d), so the stencil Hessian of
    # phi = c2r(-delta_k / k^2) equals c2r(s_a s_b / k^2 delta_k): the form the
    # GPU T-web computes with its finite-difference method.
    n, box, R = 24, 300.0, 15.0
    delta = np.random.default_rng(5).normal(size=(n, n, n))
    dk = orc.rfft3_f64(delta)
    t_fd = orc.tidal_fd(orc.poisson_f64(dk, n, box, R), box)
    kf, d = 2 * np.pi / box, box / n
    f = orc.signed_freq(n)
    fz = np.arange(n // 2 + 1, dtype=np.float64)
    s = lambda fr: (8 * np.sin(fr * kf * d) - np.sin(2 * fr * kf * d)) / (6 * d)
    sx, sy, sz = s(f)[:, None, None], s(f)[None, :, None], s(fz)[None, None, :]
    k2 = (f[:, None, None] ** 2 + f[None, :, None] ** 2 + fz[None, None, :] ** 2) * kf * kf
    with np.errstate(divide="ignore", invalid="ignore"):
        base = np.where(k2 > 0, dk / k2, 0.0) * np.exp(-0.5 * k2 * R * R)
    pairs = [(sx, sx), (sy, sy), (sz, sz), (sx, sy), (sx, sz), (sy, sz)]
    for c, (a, b) in enumerate(pairs):
        np.testing.assert_allclose(t_fd[..., c], orc.irfft3_f64(base * a * b, n),
                                   atol=1e-12 * np.abs(t_fd[..., c]).max())
    # and it differs from the spectral (FFT) tensor by the stencil's truncation error
    t_fft = orc.tidal_components(dk, n, box, R)
    assert 0 < np.abs(t_fd - t_fft).max() < 0.2 * np.abs(t_fft).max()


def test_gradfindif_as_written_matches_fp64():
    # the FP32 restatement of the reference's arithmetic agrees with the FP64
    # stencil to float rounding
    n, box = 20, 1000.0
    f = np.random.default_rng(9).normal(size=(n, n, n)).astype(np.float32)
    for axis in range(3):
        a = orc.gradfindif_ref_f32(f, axis, box).astype(np.float64)
        b = orc.gradfindif_f64(f.astype(np.float64), axis, box)
        assert np.max(np.abs(a - b)) <= 1e-6 * np.abs(b).max()


# ---------------------------------------------------------------- BAM kernel
def test_bam_kernel_bins_follow_float_modulus():
    # GetKernel's bins (Source/Bam.cpp:829-905) from real_prec arithmetic: the
    # FP64 floor(|k| / DeltaK) except where |k| / DeltaK sits within float
    # rounding of an integer; non-decreasing along every row
    n, box = 32, 700.0
    for kmin_u, ndel in ((0.0, 1.0), (0.5, 1.5)):
        b = orc.bam_kernel_bins(n, box, kmin_u, ndel)
        f = orc.signed_freq(n)
        q = np.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + np.arange(n // 2 + 1)[None, None, :] ** 2)
        x = (q - kmin_u) / ndel
        exact = np.floor(x).astype(np.int64)
        near = np.abs(x - np.round(x)) < 1e-5
        assert np.array_equal(b[~near], exact[~near])
        assert np.all(np.diff(b, axis=2) >= 0)
    # the axis modes k = 1..N/2 of unit bins land on their own index or, at a
    # float rounding below the edge, one lower
    b = orc.bam_kernel_bins(n, box)
    assert np.all((b[0, 0, :] == np.arange(n // 2 + 1)) | (b[0, 0, :] == np.arange(n // 2 + 1) - 1))


def test_bam_kernel_update_known_answers():
    n, box, nb = 16, 200.0, 8
    w = np.linspace(0.5, 2.0, nb)
    k0 = np.full((n, n, n // 2 + 1), 3.0, np.float32)
    k1, binned, modes = orc.bam_kernel_update_ref(k0, box, w, scale=False)
    b = orc.bam_kernel_bins(n, box)
    inb = b < nb
    assert np.array_equal(k1[inb], w.astype(np.float32)[b[inb]]) and np.all(k1[~inb] == 3.0)
    assert modes.sum() == inb.sum()
    np.testing.assert_allclose(binned[1:], w.astype(np.float32)[1:], rtol=1e-7)
    assert binned[0] == (binned[1] + binned[2] + binned[3] + binned[4]) / 4.0
    k2, _, _ = orc.bam_kernel_update_ref(k1, box, w, scale=True)
    assert np.array_equal(k2[inb], k1[inb] * w.astype(np.float32)[b[inb]])


def test_konvolve_with_unit_kernel():
    # K = 1: c2r(r2c(in)) / N^3 = in, then times 2 w / N^3 with w = N^2 (N/2+1)
    n = 12
    m = np.random.default_rng(1).normal(size=(n, n, n))
    out = orc.konvolve_f64(m, np.ones((n, n, n // 2 + 1)), n)
    np.testing.assert_allclose(out, m * 2.0 * (n // 2 + 1) / n, rtol=0, atol=1e-12 * np.abs(m).max())


# ---------------------------------------------------------------- cross P(k)
def test_cross_power_of_a_field_with_itself():
    # X = Y: the cross spectrum is the auto spectrum without shot noise, and
    # the coefficient is 1 in every bin with modes
    n, box = 16, 300.0
    m = np.random.default_rng(4).uniform(0.5, 1.5, size=(n, n, n))
    x = orc.cross_power_grid(m, m, box, orc.CIC, 8)
    auto = orc.power_grid(m, box, orc.CIC, 8, sn_corr=False)
    # the auto spectrum of rho - mean normalised by N_gal^2/V equals that of rho/mean - 1 by N^6/V
    np.testing.assert_allclose(x.pk, auto.pk, rtol=1e-12)
    np.testing.assert_allclose(x.pk_x, x.pk_y, rtol=1e-12)
    c = orc.cross_power_grid(m, m, box, orc.CIC, 8, coeff=True)
    has = c.modes > 0
    np.testing.assert_allclose(c.pk[has], 1.0, rtol=1e-12)
    # -X anticorrelates: coefficient -1
    c = orc.cross_power_grid(m - 1.0, 1.0 - m, box, orc.CIC, 8, "delta", "delta", coeff=True)
    np.testing.assert_allclose(c.pk[has], -1.0, rtol=1e-12)


def test_multipoles_of_an_isotropic_field_vanish_and_rotate():
    # a field made isotropic by averaging over the three lines of sight has
    # sum_los P_2 = 0 (L_2 averages to 0 over the axes: mu_x^2 + mu_y^2 + mu_z^2 = 1);
    # a field stretched along z has P_2 of opposite sign about z and about x
    n, box = 24, 400.0
    rng = np.random.default_rng(6)
    g = rng.normal(size=(n, n, n))
    tot = np.zeros(12)
    for los in range(3):
        p0, p2, p4, md = orc.power_multipoles(g, box, orc.NGP, 12, los, "delta", mas_corr=False, sn_corr=False)
        tot += p2
    np.testing.assert_allclose(tot, 0.0, atol=1e-10 * np.abs(p0.pk).max())
    k = np.fft.fftfreq(n)[None, None, :n // 2 + 1] * 0 + np.arange(n // 2 + 1)[None, None, :]
    aniso = orc.irfft3_f64(orc.rfft3_f64(g) * np.exp(-0.02 * k * k), n)  # suppress high k_z only
    _, p2z, _, _ = orc.power_multipoles(aniso, box, orc.NGP, 12, 2, "delta", mas_corr=False, sn_corr=False)
    _, p2x, _, _ = orc.power_multipoles(aniso, box, orc.NGP, 12, 0, "delta", mas_corr=False, sn_corr=False)
    assert p2z[6] < 0 < p2x[6]
