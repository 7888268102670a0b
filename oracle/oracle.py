"""CPU oracle for the CosmicAtlas/BAM mesh hot path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product library never does.

Parity status: mass assignment PINNED, the rest UNPINNED.  The reference's
own getDensity_NGP/CIC/TSC compile from Source/massFunctions.cpp against
stand-in headers (oracle/Makefile, target ref -> oracle/_ref/); the golden
meshes they write (tests/golden/) pin this module's assignment and keys.
The P(k) estimator and the T-web need FFTW3, GSL and class headers that
cannot be built here, and the reference ships no golden vectors, so this
module restates the reference source text:

* mass assignment, keys, P(k) binning, eigenvalues: ``oracle/cam_oracle.c``
  (each function cites the reference lines it follows);
* FFTs: pocketfft (scipy's, threaded) in FP64 stands in for FFTW3 (unpinned third-party
  boundary: the reference links an unversioned system FFTW,
  Main/Makefile:42-43);
* the tidal tensor follows calc_LapPhiv, Source/NumericalMethods.cpp:2609-2680,
  and the Gaussian filter kernelcomp, Source/NumericalMethods.cpp:2272-2273.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NGP, CIC, TSC = 0, 1, 2
SCHEME_P = {NGP: 0, CIC: 1, TSC: 2}  # window exponent p (Source/Params.cpp:3531-3542)


def build() -> str:
    """Compile ``cam_oracle.c`` with the committed Makefile; returns the .so path."""
    so = os.path.join(_HERE, "_build", "liboracle.so")
    src = os.path.join(_HERE, "cam_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return so


REF_SRC = os.environ.get("CAM_REFERENCE_TREE", "/root/reference")
REF_SO = os.path.join(_HERE, "_ref", "libref_mass.so")
_REF = None


def build_ref() -> str | None:
    """Compile the reference's own getDensity_NGP/CIC/TSC from its source tree
    (oracle/Makefile, target ref) into oracle/_ref/ when the tree is present;
    returns the .so path if it exists (built here, or shipped prebuilt)."""
    src = os.path.join(REF_SRC, "Source", "massFunctions.cpp")
    if os.path.exists(src):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REF_SRC}"], check=True)
    return REF_SO if os.path.exists(REF_SO) else None


def ref_lib():
    """The reference's compiled getDensity_* (None when oracle/_ref is absent)."""
    global _REF
    if _REF is None and os.path.exists(REF_SO):
        _REF = ctypes.CDLL(REF_SO)
        P = ctypes.c_void_p
        _REF.ref_assign.argtypes = [ctypes.c_int, ctypes.c_int64, P, P, P, P, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_int64] + [ctypes.c_float] * 9 + [P, P]
        _REF.ref_assign.restype = ctypes.c_int
    return _REF


def reference_getdensity(scheme, x, y, z, w, grid: "Grid"):
    """The reference's own getDensity_{NGP,CIC,TSC} (Source/massFunctions.cpp,
    compiled from source): its float mesh and the seconds the call took."""
    r = ref_lib()
    if r is None:
        raise FileNotFoundError("oracle/_ref/libref_mass.so is not built")
    x, y, z = _f32(x), _f32(y), _f32(z)
    w = None if w is None else _f32(w)
    n, L, d, mn = grid.n, grid.L, grid.d, grid.mn
    mesh = np.empty(tuple(n), np.float32)
    sec = ctypes.c_double(0.0)
    rc = r.ref_assign(scheme, x.size, _p(x), _p(y), _p(z), _p(w), n[0], n[1], n[2], L[0], L[1], L[2],
                      d[0], d[1], d[2], mn[0], mn[1], mn[2], _p(mesh), ctypes.byref(sec))
    if rc != 0:
        raise ValueError("ref_assign failed")
    return mesh, sec.value


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        P = ctypes.c_void_p
        i64, i32, f64, f32 = ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_float
        _LIB.orc_keys.argtypes = [i32, i64, P, P, P, P, P, P, P, P]
        _LIB.orc_keys.restype = None
        _LIB.orc_assign_f64.argtypes = [i32, i64, P, P, P, P, P, P, P, P, P]
        _LIB.orc_assign_f64.restype = i64
        _LIB.orc_assign_f64_mt.argtypes = [i32, i64, P, P, P, P, P, P, P, P, P]
        _LIB.orc_assign_f64_mt.restype = i64
        _LIB.orc_assign_ref.argtypes = [i32, i64, P, P, P, P, i64, i64, i64,
                                        f32, f32, f32, f32, f32, f32, f32, f32, f32, P]
        _LIB.orc_assign_ref.restype = i64
        _LIB.orc_assign_omp.argtypes = [i32, i64, P, P, P, P, i64, i64, i64,
                                        f32, f32, f32, f32, f32, f32, f32, f32, f32, P, i32]
        _LIB.orc_assign_omp.restype = i64
        _LIB.orc_set_threads.argtypes = [i32]
        _LIB.orc_set_threads.restype = None
        _LIB.orc_power_f64.argtypes = [i64, P, i32, i32, i32, f64, f64, f64, f64, i32, P, P, P, P]
        _LIB.orc_power_f64.restype = None
        _LIB.orc_cross_f64.argtypes = [i64, P, P, i32, i32, f64, f64, i32, P, P, P, P]
        _LIB.orc_cross_f64.restype = None
        _LIB.orc_multipole_f64.argtypes = [i64, P, i32, i32, f64, f64, i32, i32, P, P, P]
        _LIB.orc_multipole_f64.restype = None
        _LIB.orc_power_ref.argtypes = [i64, P, i32, i32, i32, f32, f32, f32, f32, f32, i32, i32, P, P]
        _LIB.orc_power_ref.restype = None
        _LIB.orc_bin.argtypes = [f64, f64, f64, i32]
        _LIB.orc_bin.restype = i64
        _LIB.orc_eig3_f64.argtypes = [i64, P, P]
        _LIB.orc_eig3_f64.restype = None
        _LIB.orc_classify.argtypes = [i64, P, f64, f64, P, P, P]
        _LIB.orc_classify.restype = None
    return _LIB


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Grid:
    """Mesh geometry: cells per axis, box sides, spacing and origin (float32),
    the fields of s_params_box_mas, Headers/Type_structures_def.h:1141-1152."""
    n: tuple
    L: tuple
    d: tuple
    mn: tuple

    @staticmethod
    def cubic(n: int, L: float, mn: float = 0.0) -> "Grid":
        d = float(np.float32(np.float32(L) / np.float32(n)))
        return Grid((n, n, n), (L, L, L), (d, d, d), (mn, mn, mn))

    def arrays(self):
        return (np.asarray(self.n, np.int64), np.asarray(self.L, np.float32),
                np.asarray(self.d, np.float32), np.asarray(self.mn, np.float32))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def keys(scheme, x, y, z, grid: Grid) -> np.ndarray:
    x, y, z = _f32(x), _f32(y), _f32(z)
    n, L, d, mn = grid.arrays()
    out = np.empty(x.size, np.int64)
    lib().orc_keys(scheme, x.size, _p(x), _p(y), _p(z), _p(n), _p(L), _p(d), _p(mn), _p(out))
    return out


def assign_f64(scheme, x, y, z, w, grid: Grid):
    """FP64 mesh with the pinned semantics; returns (mesh[N1,N2,N3], n_lost)."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    w = None if w is None else _f32(w)
    n, L, d, mn = grid.arrays()
    mesh = np.empty(tuple(int(v) for v in n), np.float64)
    lost = lib().orc_assign_f64(scheme, x.size, _p(x), _p(y), _p(z), _p(w),
                                _p(n), _p(L), _p(d), _p(mn), _p(mesh))
    return mesh, int(lost)


def assign_f64_mt(scheme, x, y, z, w, grid: Grid):
    """assign_f64 on all host threads (atomic FP64 adds; only the order of the
    additions differs from the serial loop): for the full-size meshes."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    w = None if w is None else _f32(w)
    n, L, d, mn = grid.arrays()
    mesh = np.empty(tuple(int(v) for v in n), np.float64)
    lost = lib().orc_assign_f64_mt(scheme, x.size, _p(x), _p(y), _p(z), _p(w),
                                   _p(n), _p(L), _p(d), _p(mn), _p(mesh))
    return mesh, int(lost)


def assign_ref(scheme, x, y, z, w, grid: Grid):
    """The reference's FP32 serial loop as written (CPU baseline)."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    w = None if w is None else _f32(w)
    n, L, d, mn = grid.n, grid.L, grid.d, grid.mn
    mesh = np.empty(tuple(n), np.float32)
    lost = lib().orc_assign_ref(scheme, x.size, _p(x), _p(y), _p(z), _p(w), n[0], n[1], n[2],
                                L[0], L[1], L[2], d[0], d[1], d[2], mn[0], mn[1], mn[2], _p(mesh))
    return mesh, int(lost)


def set_threads(n: int = 0):
    """Thread count of the oracle's OpenMP loops (n <= 0: all)."""
    lib().orc_set_threads(int(n))


def assign_omp(scheme, x, y, z, w, grid: Grid, nthreads=0):
    """The Gen-B OpenMP private-grid form of the reference loops, with its
    NTHREADS-fold over-count fixed (CPU baseline)."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    w = None if w is None else _f32(w)
    n, L, d, mn = grid.n, grid.L, grid.d, grid.mn
    mesh = np.empty(tuple(n), np.float32)
    lost = lib().orc_assign_omp(scheme, x.size, _p(x), _p(y), _p(z), _p(w), n[0], n[1], n[2],
                                L[0], L[1], L[2], d[0], d[1], d[2], mn[0], mn[1], mn[2], _p(mesh), int(nthreads))
    return mesh, int(lost)


def rfft3_f64(mesh: np.ndarray) -> np.ndarray:
    """Unnormalised forward r2c (FFTW layout [i][j][k<=N/2]); stands in for
    do_fftw_r2c, Source/NumericalMethods.cpp:1718-1753.  pocketfft in FP64
    (scipy's, on all host threads)."""
    import scipy.fft
    return scipy.fft.rfftn(np.asarray(mesh, np.float64), workers=-1)


def irfft3_f64(spec: np.ndarray, n: int) -> np.ndarray:
    """c2r divided by N^3 as do_fftw_c2r does, Source/NumericalMethods.cpp:1818-1856
    (the inverse transform already divides by N^3)."""
    import scipy.fft
    return scipy.fft.irfftn(spec, s=(n, n, n), axes=(0, 1, 2), workers=-1)


@dataclass
class PkResult:
    pk: np.ndarray
    modes: np.ndarray
    sum_raw: np.ndarray
    sum_sn: np.ndarray
    kcent: np.ndarray
    shot_noise: float
    normal: float
    n_obj: float


def power_from_spectrum(spec, n, L, scheme, nbins, shot_noise, normal,
                        kmin_u=0.0, dk_u=1.0, mas_corr=True, sn_corr=True) -> PkResult:
    spec = np.ascontiguousarray(spec, dtype=np.complex128)
    pk = np.empty(nbins); modes = np.empty(nbins, np.int64)
    sr = np.empty(nbins); ss = np.empty(nbins)
    lib().orc_power_f64(n, _p(spec), SCHEME_P[scheme], int(mas_corr), int(sn_corr),
                        float(shot_noise), float(normal), float(kmin_u), float(dk_u), nbins,
                        _p(pk), _p(modes), _p(sr), _p(ss))
    kf = 2.0 * np.pi / L
    kcent = kf * (kmin_u + (np.arange(nbins) + 0.5) * dk_u)
    return PkResult(pk, modes, sr, ss, kcent, shot_noise, normal, float("nan"))


def power_grid(mesh, L, scheme, nbins, kmin_u=0.0, dk_u=1.0, input_type="density",
               mas_corr=True, sn_corr=True) -> PkResult:
    """PowerSpectrumF::compute_power_spectrum_grid, Source/PowerSpectrumF.cpp:1739-1800,
    in FP64: density input -> data = rho - N_gal/N^3, normal = N_gal^2/V,
    SN = V/N_gal; delta input -> normal = N^6/V, N_gal = 1."""
    n = mesh.shape[0]
    vol = float(L) ** 3
    mesh = np.asarray(mesh, np.float64)
    if input_type == "density":
        ngal = float(mesh.sum())
        data = mesh - ngal / mesh.size
        normal = ngal * ngal / vol
    else:
        ngal = 1.0
        data = mesh
        normal = float(mesh.size) ** 2 / vol
    sn = vol / ngal
    spec = rfft3_f64(data)
    r = power_from_spectrum(spec, n, L, scheme, nbins, sn, normal, kmin_u, dk_u, mas_corr, sn_corr)
    r.n_obj = ngal
    return r


def power_multipoles(mesh, L, scheme, nbins, los=2, input_type="density", kmin_u=0.0, dk_u=1.0,
                     mas_corr=True, sn_corr=True):
    """P(k) (power_grid) and the multipoles of FftwFunctions::power_spectrum_fkp,
    Source/FftwFunctions.cpp:958-1625, for a box with a fixed line of sight:
    P_2 = 5 sum L_2 |F|^2/W^2 / (modes normal), P_4 = 9 sum L_4 |F|^2/W^2 / (...),
    with the normalisation of power_grid and no shot noise for l > 0."""
    n = mesh.shape[0]
    p0 = power_grid(mesh, L, scheme, nbins, kmin_u, dk_u, input_type, mas_corr, sn_corr)
    m = np.asarray(mesh, np.float64)
    data = m - m.sum() / m.size if input_type == "density" else m
    spec = np.ascontiguousarray(rfft3_f64(data), np.complex128)
    s2, s4 = np.empty(nbins), np.empty(nbins)
    md = np.empty(nbins, np.int64)
    lib().orc_multipole_f64(n, _p(spec), SCHEME_P[scheme], int(mas_corr), float(kmin_u), float(dk_u), nbins,
                            int(los), _p(s2), _p(s4), _p(md))
    den = np.maximum(md, 1) * p0.normal
    return p0, np.where(md > 0, 5.0 * s2 / den, 0.0), np.where(md > 0, 9.0 * s4 / den, 0.0), md


@dataclass
class CrossResult:
    pk: np.ndarray      # cross power, or the coefficient with coeff=True
    pk_x: np.ndarray
    pk_y: np.ndarray
    modes: np.ndarray


def cross_power_grid(mx, my, L, scheme, nbins, input_x="density", input_y="density", coeff=False,
                     kmin_u=0.0, dk_u=1.0, mas_corr=True) -> CrossResult:
    """PowerSpectrumF::compute_cross_power_spectrum_grid, Source/PowerSpectrumF.cpp:549-632,
    with FftwFunctions::cross_power_spectrum_fkp, Source/FftwFunctions.cpp:645-893, in
    FP64: density meshes become rho/mean - 1, both normalisations are
    (L^1.5 / N^3)^-2 = N^6 / L^3, P_X = sum Re(F_X F_Y*) / W^2 / (modes N^6/L^3);
    coeff=True divides by sqrt(P_XX P_YY) (:885-893)."""
    n = mx.shape[0]
    def delta(m, kind):
        m = np.asarray(m, np.float64)
        return m / (m.sum() / m.size) - 1.0 if kind == "density" else m
    s1 = np.ascontiguousarray(rfft3_f64(delta(mx, input_x)), np.complex128)
    s2 = np.ascontiguousarray(rfft3_f64(delta(my, input_y)), np.complex128)
    cr, a1, a2 = np.empty(nbins), np.empty(nbins), np.empty(nbins)
    md = np.empty(nbins, np.int64)
    lib().orc_cross_f64(n, _p(s1), _p(s2), SCHEME_P[scheme], int(mas_corr), float(kmin_u), float(dk_u), nbins,
                        _p(cr), _p(a1), _p(a2), _p(md))
    normal = float(n) ** 6 / float(L) ** 3
    with np.errstate(divide="ignore", invalid="ignore"):
        px = np.where(md > 0, cr / (md * normal), 0.0)
        pxx = np.where(md > 0, a1 / (md * normal), 0.0)
        pyy = np.where(md > 0, a2 / (md * normal), 0.0)
        pk = np.where(md > 0, px / np.sqrt(pxx * pyy), 0.0) if coeff else px
    return CrossResult(pk, pxx, pyy, md)


def signed_freq(n: int) -> np.ndarray:
    """coords[i] / deltak = i if i <= N/2 else i - N (NumericalMethods.cpp:2625-2626)."""
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


def tidal_components(delta_k, n, L, R):
    """T_ab = c2r(k_a k_b / k^2 * exp(-k^2 R^2 / 2) * delta_k) / N^3 for the six
    symmetric pairs (xx, yy, zz, xy, xz, yz).  calc_LapPhiv computes all nine,
    Source/Miscelanious.cpp:1792-1828."""
    kf = 2.0 * np.pi / L
    fx = signed_freq(n)[:, None, None] * kf
    fy = signed_freq(n)[None, :, None] * kf
    fz = np.arange(n // 2 + 1, dtype=np.float64)[None, None, :] * kf
    k2 = fx * fx + fy * fy + fz * fz
    with np.errstate(divide="ignore", invalid="ignore"):
        ik2 = np.where(k2 > 0, 1.0 / k2, 0.0)
    g = np.exp(-0.5 * k2 * R * R) if R > 0 else 1.0
    base = delta_k * ik2 * g
    pairs = [(fx, fx), (fy, fy), (fz, fz), (fx, fy), (fx, fz), (fy, fz)]
    out = np.empty((n, n, n, 6))
    for c, (a, b) in enumerate(pairs):
        out[..., c] = irfft3_f64(base * (a * b), n)
    return out


def eig3_f64(t6: np.ndarray) -> np.ndarray:
    """Descending eigenvalues of the (…,6) tensors via LAPACK (numpy eigvalsh)."""
    m = np.empty(t6.shape[:-1] + (3, 3))
    m[..., 0, 0] = t6[..., 0]; m[..., 1, 1] = t6[..., 1]; m[..., 2, 2] = t6[..., 2]
    m[..., 0, 1] = m[..., 1, 0] = t6[..., 3]
    m[..., 0, 2] = m[..., 2, 0] = t6[..., 4]
    m[..., 1, 2] = m[..., 2, 1] = t6[..., 5]
    return np.linalg.eigvalsh(m)[..., ::-1].copy()


def eig3_closed(t6: np.ndarray) -> np.ndarray:
    t6 = np.ascontiguousarray(t6.reshape(-1, 6), np.float64)
    lam = np.empty((t6.shape[0], 3))
    lib().orc_eig3_f64(t6.shape[0], _p(t6), _p(lam))
    return lam


@dataclass
class TwebResult:
    labels: np.ndarray
    lam: np.ndarray
    counts: np.ndarray
    ties: int


def classify(lam, lth, band=1e-5):
    """CWClass = 4 - #{lambda > lambda_th}, Source/Cwclass.cpp:875-890."""
    lam = np.ascontiguousarray(lam.reshape(-1, 3), np.float64)
    labels = np.empty(lam.shape[0], np.uint8)
    counts = np.zeros(4, np.int64)
    ties = np.zeros(1, np.int64)
    lib().orc_classify(lam.shape[0], _p(lam), float(lth), float(band), _p(labels), _p(counts), _p(ties))
    return labels, counts, int(ties[0])


def tidal_invariants(lam: np.ndarray) -> np.ndarray:
    """invariant_field_I/II/III and tidal_anisotropy, Source/Miscelanious.cpp:1460-1492,
    of descending eigenvalues (…,3), in FP64: (4, …)."""
    l1, l2, l3 = lam[..., 0], lam[..., 1], lam[..., 2]
    i1 = l1 + l2 + l3
    i2 = l1 * l2 + l2 * l3 + l1 * l3
    i3 = (l1 * l2) * l3
    ta = np.sqrt(0.5 * ((l3 - l1) ** 2 + (l3 - l2) ** 2 + (l2 - l1) ** 2)) / (2.0 + i1)
    return np.stack([i1, i2, i3, ta])


def tweb_from_spectrum(delta_k, n, L, R, lth, band=1e-5) -> TwebResult:
    t6 = tidal_components(delta_k, n, L, R)
    lam = eig3_f64(t6).reshape(n, n, n, 3)
    labels, counts, ties = classify(lam, lth, band)
    return TwebResult(labels.reshape(n, n, n), lam, counts, ties)


def tidal_planes(delta_k, n, L, R, planes) -> np.ndarray:
    """The six components of tidal_components on the x-planes `planes` only,
    (len(planes), N, N, 6): the inverse transform along x is evaluated at
    those planes as a DFT (T(x_p) = sum_kx F[kx] e^{2 pi i kx x_p / N} / N),
    then the inverse r2c over (y, z).  Equal to tidal_components[planes] up
    to FP64 rounding; memory O(N^2 (N/2+1)) for one component at a time."""
    import scipy.fft
    kf = 2.0 * np.pi / L
    fx = signed_freq(n)[:, None, None] * kf
    fy = signed_freq(n)[None, :, None] * kf
    fz = np.arange(n // 2 + 1, dtype=np.float64)[None, None, :] * kf
    planes = np.asarray(planes, np.int64)
    ex = np.exp(2j * np.pi * np.outer(planes, np.arange(n)) / n) / n  # (P, N)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    out = np.empty((planes.size, n, n, 6))
    chunk = max(1, (1 << 26) // (n * (n // 2 + 1)))
    for c, (a, b) in enumerate(pairs):
        acc = np.zeros((planes.size, n, n // 2 + 1), np.complex128)
        for i0 in range(0, n, chunk):
            i1 = min(n, i0 + chunk)
            k = (fx[i0:i1], fy, fz)
            k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2]
            with np.errstate(divide="ignore", invalid="ignore"):
                m = np.where(k2 > 0, k[a] * k[b] / k2, 0.0)
            if R > 0:
                m = m * np.exp(-0.5 * k2 * R * R)
            blk = delta_k[i0:i1] * m  # (i1-i0, N, N/2+1)
            acc += np.tensordot(ex[:, i0:i1], blk, axes=(1, 0))
        out[..., c] = scipy.fft.irfftn(acc, s=(n, n), axes=(1, 2), workers=-1)
    return out


def tweb_density(mesh, L, R, lth, band=1e-5) -> TwebResult:
    """Cwclass::get_CWC on delta = rho/mean - 1 (Source/Cwclass.cpp:235-890,
    FFT tidal-tensor variant EigenValuesTweb, Source/Miscelanious.cpp:1772)."""
    n = mesh.shape[0]
    mesh = np.asarray(mesh, np.float64)
    nbar = mesh.sum() / mesh.size
    delta_k = rfft3_f64(mesh / nbar - 1.0)
    return tweb_from_spectrum(delta_k, n, L, R, lth, band)


# ---- finite-difference T-web (the reference's default variant) ----------

def poisson_f64(delta_k, n, L, R=0.0) -> np.ndarray:
    """PoissonSolver, Source/Miscelanious.cpp:1189-1275: phi = c2r(-delta_k / k^2)
    / N^3 with k from coords[i] = k_f (i <= N/2 ? i : i - N) and the k = 0 mode
    set to 0 (:1251-1262).  R > 0 also applies the Gaussian filter of
    kernelcomp, Source/NumericalMethods.cpp:2272-2273, to delta_k."""
    kf = 2.0 * np.pi / L
    fx = signed_freq(n)[:, None, None] * kf
    fy = signed_freq(n)[None, :, None] * kf
    fz = np.arange(n // 2 + 1, dtype=np.float64)[None, None, :] * kf
    k2 = fx * fx + fy * fy + fz * fz
    with np.errstate(divide="ignore", invalid="ignore"):
        term = np.where(k2 > 0, -1.0 / k2, 0.0)
    g = np.exp(-0.5 * k2 * R * R) if R > 0 else 1.0
    return irfft3_f64(delta_k * term * g, n)


def gradfindif_f64(f: np.ndarray, axis: int, L: float) -> np.ndarray:
    """gradfindif, Source/NumericalMethods.cpp:1123-1218: the 4th-order centred
    difference (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2]) / (12 L / N) along one
    axis (dim 1 = x = axis 0, the slowest; dim 3 = z = axis 2), periodic."""
    n = f.shape[axis]
    ideltaH = 1.0 / (12.0 * (L / n))
    return (-np.roll(f, -2, axis) + 8.0 * np.roll(f, -1, axis) - 8.0 * np.roll(f, 1, axis)
            + np.roll(f, 2, axis)) * ideltaH


def gradfindif_ref_f32(f: np.ndarray, axis: int, L: float) -> np.ndarray:
    """gradfindif as the reference evaluates it with real_prec = float
    (Source/NumericalMethods.cpp:1126-1127, :1153): deltaH = 12.0 * (L1 / N1)
    from a float quotient, ideltaH = 1.0 / deltaH rounded to float, and
    (-in[rr] + 8.0*in[r] - 8.0*in[l] + in[ll]) * ideltaH evaluated left to
    right in double (8.0 is a double literal), rounded to float on
    assignment."""
    n = f.shape[axis]
    d = np.float32(L) / np.float32(n)
    deltaH = np.float32(12.0 * np.float64(d))
    ideltaH = np.float32(1.0 / np.float64(deltaH))
    a = np.asarray(f, np.float32).astype(np.float64)
    v = ((-np.roll(a, -2, axis) + 8.0 * np.roll(a, -1, axis)) - 8.0 * np.roll(a, 1, axis)) + np.roll(a, 2, axis)
    return (v * np.float64(ideltaH)).astype(np.float32)


def tidal_fd(phi: np.ndarray, L: float) -> np.ndarray:
    """The (…,6) tensors (xx, yy, zz, xy, xz, yz) of EigenValuesTweb's
    _USE_GFINDIFF_EIGENV_ branch, Source/Miscelanious.cpp:1681-1700: the
    first differences of phi along x, y, z, each differenced again.  The
    off-diagonal entries are the ones gsl_eigen_symmv reads (its lower
    triangle, in_matrix[1], [2], [5] at :1733-1738): T_xy = D_x(D_y phi),
    T_xz = D_x(D_z phi), T_yz = D_y(D_z phi)."""
    gx = gradfindif_f64(phi, 0, L)
    gy = gradfindif_f64(phi, 1, L)
    gz = gradfindif_f64(phi, 2, L)
    out = np.empty(phi.shape + (6,))
    out[..., 0] = gradfindif_f64(gx, 0, L)
    out[..., 1] = gradfindif_f64(gy, 1, L)
    out[..., 2] = gradfindif_f64(gz, 2, L)
    out[..., 3] = gradfindif_f64(gy, 0, L)
    out[..., 4] = gradfindif_f64(gz, 0, L)
    out[..., 5] = gradfindif_f64(gz, 1, L)
    return out


def tweb_fd_potential(phi, L, lth, band=1e-5) -> TwebResult:
    """EigenValuesTweb(Nft, L, delta, phi, ...) with finite differences
    (Source/Miscelanious.cpp:1663-1760) and the labels of Cwclass.cpp:875-890."""
    n = phi.shape[0]
    lam = eig3_f64(tidal_fd(np.asarray(phi, np.float64), L)).reshape(n, n, n, 3)
    labels, counts, ties = classify(lam, lth, band)
    return TwebResult(labels.reshape(n, n, n), lam, counts, ties)


def tweb_fd_from_spectrum(delta_k, n, L, R, lth, band=1e-5) -> TwebResult:
    return tweb_fd_potential(poisson_f64(delta_k, n, L, R), L, lth, band)


def tweb_fd_density(mesh, L, R, lth, band=1e-5) -> TwebResult:
    """Cwclass::get_CWC with the reference's default T-web
    (Source/Cwclass.cpp:235-277): PoissonSolver on delta = rho/mean - 1,
    then the finite-difference tidal tensor."""
    n = mesh.shape[0]
    mesh = np.asarray(mesh, np.float64)
    nbar = mesh.sum() / mesh.size
    return tweb_fd_from_spectrum(rfft3_f64(mesh / nbar - 1.0), n, L, R, lth, band)


# ---- catalogue weights -------------------------------------------------------

def fkp_weights_f64(nbar, w_in=None, fkp=True, P_est=0.0):
    """The tracer loop's weights and sums, Source/Catalog.cpp:14140-14165, in
    FP64: w = w_in / (1 + P_est nbar) (FKP on); (n_selected, W_r = sum w,
    S_r = sum w^2, normal = sum nbar w^2)."""
    nbar = np.asarray(nbar, np.float64)
    w = np.ones_like(nbar) if w_in is None else np.asarray(w_in, np.float64).copy()
    if fkp:
        w = w * (1.0 / (1.0 + P_est * nbar))
    return w, np.array([float(nbar.size), w.sum(), (w * w).sum(), (nbar * w * w).sum()])


# ---- BAM kernel (GetKernel's 3D update, Konvolve) ---------------------------

def bam_kernel_bins(n, L, DeltaKmin=0.0, ndel=1.0, dtype=np.float32) -> np.ndarray:
    """The bin of every half-complex element in Bam::GetKernel,
    Source/Bam.cpp:829-905, in the reference's real_prec arithmetic:
    kv = _get_modulo(coords[i]*dk, coords[j]*dk, coords[k]*dk), a macro that
    expands to sqrt(c_i*dk*c_i*dk + c_j*dk*c_j*dk + c_k*dk*c_k*dk)
    (Headers/def.h:695), then floor((kv - kmin) / DeltaK).  dk, kmin and
    DeltaK are Params' double values read through real_prec getters
    (Source/Params.cpp:4092-4103, Headers/Params.h:4326-4363)."""
    t = np.dtype(dtype).type
    deltak = 2.0 * np.pi / np.float64(np.float32(L))
    dk2 = deltak * deltak
    deltak0 = np.sqrt((dk2 + dk2) + dk2) / np.sqrt(3.0)
    dk, kmin, dK = t(deltak), t(DeltaKmin * deltak0), t(ndel * deltak0)
    c = signed_freq(n).astype(dtype)
    ck = np.arange(n // 2 + 1).astype(dtype)
    with np.errstate(over="ignore", invalid="ignore"):
        tx = ((c * dk) * c) * dk
        tz = ((ck * dk) * ck) * dk
        kv = np.sqrt((tx[:, None, None] + tx[None, :, None]) + tz[None, None, :])
        b = np.floor((kv - kmin) / dK)
    return b.astype(np.int64)


def bam_kernel_update_ref(kernel, L, weight, scale: bool, DeltaKmin=0.0, ndel=1.0):
    """GetKernel's 3D loops (Source/Bam.cpp:829-905) on a copy of `kernel`
    (N, N, N/2+1): kernel = weight[b] (no rejection) or kernel *= weight[b]
    (rejection) for 0 <= b < nbins, in the kernel's precision.  Returns the
    updated kernel, the bin means of it (FP64 sums; bin 0 = mean of bins
    1..4, :905-910) and the element counts."""
    k = np.array(kernel, copy=True)
    t = k.dtype.type
    nb = len(weight)
    b = bam_kernel_bins(k.shape[0], L, DeltaKmin, ndel, k.dtype)
    inb = (b >= 0) & (b < nb)
    w = np.asarray(weight, np.float64).astype(k.dtype)
    if scale:
        k[inb] = k[inb] * w[b[inb]]
    else:
        k[inb] = w[b[inb]]
    sums = np.bincount(b[inb], weights=k[inb].astype(np.float64), minlength=nb)[:nb]
    modes = np.bincount(b[inb], minlength=nb)[:nb].astype(np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):
        binned = sums / modes
    binned[0] = (binned[1] + binned[2] + binned[3] + binned[4]) / 4.0
    return k, binned, modes


def konvolve_f64(mesh, kernel, n):
    """Bam::Konvolve, Source/Bam.cpp:1027-1120, in FP64: c2r(K r2c(in)) / N^3,
    divided by N^3 / (2 w) with w the sum of K over the half-complex array."""
    w = np.sum(np.asarray(kernel, np.float64))
    out = irfft3_f64(rfft3_f64(np.asarray(mesh, np.float64)) * np.asarray(kernel, np.float64), n)
    return out / (float(n) ** 3 / (2.0 * w))


def power_ref(spec_c64, n, L, scheme, nbins, shot_noise, normal, ndel=1.0, fix_octant4=True):
    """The reference's FP32 loop as written (CPU baseline)."""
    spec = np.ascontiguousarray(spec_c64, dtype=np.complex64)
    pk = np.empty(nbins, np.float32); md = np.empty(nbins, np.int32)
    dk = np.float32(2.0 * np.pi / L)
    lib().orc_power_ref(n, _p(spec), SCHEME_P[scheme], 1, 1, float(shot_noise), float(normal),
                        float(dk), 0.0, float(ndel * dk), nbins, int(fix_octant4), _p(pk), _p(md))
    return pk, md
