"""Host-side mirror of the reference's hot-path interface over libcam.

Two layers:

* ``Context``: one CUDA device, its stream, cached FFT plans and scratch
  buffers (cam_ctx).  Methods map 1:1 to the C ABI.
* Reference-shaped entry points with the reference's names, argument meaning
  and effects: ``getDensity_NGP/CIC/TSC`` (Headers/massFunctions.h:12-26),
  ``do_fftw_r2c/c2r`` (Source/NumericalMethods.cpp:1718, :1818),
  ``PowerSpectrumF.compute_power_spectrum_grid`` (Source/PowerSpectrumF.cpp:1739)
  and ``Cwclass.get_CWC`` (Source/Cwclass.cpp:235).  Where the reference exits
  on an error these raise ``CamError``.

Arrays may be numpy (host) or torch CUDA tensors (device, same device as the
context); results come back in the same kind of memory.
"""
from __future__ import annotations

import ctypes
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import CamError

NGP, CIC, TSC = L.NGP, L.CIC, L.TSC
F32, F64 = L.F32, L.F64


def make_grid(n, box, d=None, mn=0.0) -> L.Grid:
    n3 = (n, n, n) if np.isscalar(n) else tuple(n)
    b3 = (box, box, box) if np.isscalar(box) else tuple(box)
    m3 = (mn, mn, mn) if np.isscalar(mn) else tuple(mn)
    if d is None:
        d3 = tuple(float(np.float32(np.float32(b) / np.float32(k))) for b, k in zip(b3, n3))
    else:
        d3 = (d, d, d) if np.isscalar(d) else tuple(d)
    g = L.Grid()
    for a in range(3):
        g.n[a], g.L[a], g.d[a], g.min[a] = int(n3[a]), float(b3[a]), float(d3[a]), float(m3[a])
    return g


def _f32(a):
    if a is None or L.is_device(a):
        return a
    return np.ascontiguousarray(a, dtype=np.float32)


@dataclass
class PkResult:
    pk: np.ndarray
    modes: np.ndarray
    kvector: np.ndarray
    n_obj: float
    shot_noise: float
    normal: float


@dataclass
class TwebResult:
    labels: object
    lambdas: object
    counts: np.ndarray
    ties: int
    mean: float


@dataclass
class AssignResult:
    mesh: object
    n_in: int
    n_lost: int
    sum_mesh: float


class Context:
    """A cam_ctx on one device with an optional HBM budget (bytes).

    Device arrays (torch tensors) are read on the context's own stream: ones
    just produced by torch kernels must be complete first
    (torch.cuda.synchronize()), or set_stream(torch.cuda.current_stream().cuda_stream)
    makes the context launch on torch's stream."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.cam_ctx_create(device, hbm_budget, ctypes.byref(h))
        if rc != L.CAM_OK:
            raise CamError(rc, f"cannot create a context on device {device}")
        self.h = h
        self.device = device
        self._lock = threading.Lock()

    def close(self):
        if getattr(self, "h", None):
            self._lib.cam_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != L.CAM_OK:
            raise CamError(rc, self._lib.cam_last_error(self.h).decode())

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.cam_kernel_launches(self.h))

    def profile(self, on: bool = True):
        self._check(self._lib.cam_profile_enable(self.h, int(on)))

    def profile_read(self, reset: bool = True) -> dict:
        """{kernel: (launches, total_ms)} since the last reset."""
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.cam_profile_read(self.h, buf, len(buf), int(reset)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.rsplit(",", 2)
            out[name] = (int(cnt), float(ms))
        return out

    def set_stream(self, stream_handle: int | None):
        self._check(self._lib.cam_ctx_set_stream(self.h, stream_handle))

    def sync(self):
        self._check(self._lib.cam_ctx_sync(self.h))

    # ---------------------------------------------------------------- helpers
    def _particles(self, x, y, z, w):
        dev = L.is_device(x)
        x, y, z, w = _f32(x), _f32(y), _f32(z), _f32(w)
        p = L.Particles()
        p.n = int(x.shape[0])
        p.x, p.y, p.z, p.w = L.ptr(x), L.ptr(y), L.ptr(z), L.ptr(w)
        p.mem = L.MEM_DEVICE if dev else L.MEM_HOST
        return p, (x, y, z, w), dev

    @staticmethod
    def _empty(shape, dtype, dev, like=None):
        if dev:
            import torch
            tdt = {np.float32: torch.float32, np.float64: torch.float64, np.uint32: torch.int32,
                   np.uint8: torch.uint8, np.int64: torch.int64, np.complex64: torch.complex64,
                   np.complex128: torch.complex128}[dtype]
            return torch.empty(shape, dtype=tdt, device=like.device)
        return np.empty(shape, dtype)

    # ---------------------------------------------------------------- assignment
    def assign(self, x, y, z, w, grid: L.Grid, scheme: int, precision: int = F32, out=None) -> AssignResult:
        p, keep, dev = self._particles(x, y, z, w)
        shape = (grid.n[0], grid.n[1], grid.n[2])
        dt = np.float64 if precision == F64 else np.float32
        mesh = out if out is not None else self._empty(shape, dt, dev, x)
        st = L.AssignStats()
        self._check(self._lib.cam_assign(self.h, ctypes.byref(p), ctypes.byref(grid), scheme, precision,
                                         L.ptr(mesh), L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(st)))
        return AssignResult(mesh, st.n_in, st.n_lost, st.sum_mesh)

    def count_ngp(self, x, y, z, grid: L.Grid) -> AssignResult:
        p, keep, dev = self._particles(x, y, z, None)
        shape = (grid.n[0], grid.n[1], grid.n[2])
        out = self._empty(shape, np.uint32, dev, x)
        st = L.AssignStats()
        self._check(self._lib.cam_count_ngp(self.h, ctypes.byref(p), ctypes.byref(grid), L.ptr(out),
                                            L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(st)))
        return AssignResult(out, st.n_in, st.n_lost, st.sum_mesh)

    def cell_keys(self, x, y, z, grid: L.Grid, scheme: int):
        p, keep, dev = self._particles(x, y, z, None)
        out = self._empty((p.n,), np.int64, dev, x)
        self._check(self._lib.cam_cell_keys(self.h, ctypes.byref(p), ctypes.byref(grid), scheme, L.ptr(out),
                                            L.MEM_DEVICE if dev else L.MEM_HOST))
        return out

    # ---------------------------------------------------------------- FFT
    def fft_r2c(self, mesh):
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        cdt = np.complex128 if prec == F64 else np.complex64
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        out = self._empty((n, n, n // 2 + 1), cdt, dev, mesh)
        self._check(self._lib.cam_fft_r2c(self.h, n, prec, L.ptr(mesh), L.ptr(out),
                                          L.MEM_DEVICE if dev else L.MEM_HOST))
        return out

    def fft_c2r(self, spec):
        dev = L.is_device(spec)
        n = spec.shape[0]
        prec = F64 if str(spec.dtype).endswith("complex128") else F32
        rdt = np.float64 if prec == F64 else np.float32
        if not dev:
            spec = np.ascontiguousarray(spec)
        out = self._empty((n, n, n), rdt, dev, spec)
        self._check(self._lib.cam_fft_c2r(self.h, n, prec, L.ptr(spec), L.ptr(out),
                                          L.MEM_DEVICE if dev else L.MEM_HOST))
        return out

    # ---------------------------------------------------------------- P(k)
    @staticmethod
    def pk_opts(scheme=CIC, nbins=0, ndel=1.0, DeltaKmin=0.0, mas_correction=True, sn_correction=True,
                input_type=L.INPUT_DENSITY) -> L.PkOpts:
        o = L.PkOpts()
        o.scheme, o.mas_correction, o.sn_correction = scheme, int(mas_correction), int(sn_correction)
        o.input_type, o.nbins, o.DeltaKmin, o.ndel = input_type, nbins, DeltaKmin, ndel
        return o

    def power(self, mesh, box: float, opts: L.PkOpts) -> PkResult:
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        nb = opts.nbins if opts.nbins > 0 else int(n / opts.ndel / 2)
        pk = np.empty(nb); md = np.empty(nb, np.int64); kv = np.empty(nb)
        info = L.PkInfo()
        g = make_grid(n, box)
        self._check(self._lib.cam_power(self.h, ctypes.byref(g), L.ptr(mesh), prec,
                                        L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(opts),
                                        L.ptr(pk), L.ptr(md), L.ptr(kv), ctypes.byref(info)))
        return PkResult(pk, md, kv, info.n_obj, info.shot_noise, info.normal)

    def power_multipoles(self, mesh, box: float, opts: L.PkOpts, los: int = 2) -> dict:
        """P(k) and its multipoles l = 2, 4 about axis los (0 x, 1 y, 2 z), as
        power_spectrum_fkp forms them (Source/FftwFunctions.cpp:958)."""
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        nb = opts.nbins if opts.nbins > 0 else int(n / opts.ndel / 2)
        p0, p2, p4, kv = np.empty(nb), np.empty(nb), np.empty(nb), np.empty(nb)
        md = np.empty(nb, np.int64)
        info = L.PkInfo()
        g = make_grid(n, box)
        self._check(self._lib.cam_power_multipoles(self.h, ctypes.byref(g), L.ptr(mesh), prec,
                                                   L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(opts), los,
                                                   L.ptr(p0), L.ptr(p2), L.ptr(p4), L.ptr(md), L.ptr(kv),
                                                   ctypes.byref(info)))
        return {"p0": p0, "p2": p2, "p4": p4, "modes": md, "kvector": kv}

    def cross_power(self, mesh_x, mesh_y, box: float, opts: L.PkOpts, input_type_y=L.INPUT_DENSITY,
                    want_coeff=False) -> dict:
        """Cross power spectrum (PowerSpectrumF::compute_cross_power_spectrum_grid,
        Source/PowerSpectrumF.cpp:549): returns pk (cross power or, with
        want_coeff, the cross-correlation coefficient), pk_x, pk_y, modes, kvector."""
        dev = L.is_device(mesh_x)
        if dev != L.is_device(mesh_y):
            raise ValueError("both meshes must be on the host or both on the device")
        n = mesh_x.shape[0]
        prec = F64 if str(mesh_x.dtype).endswith("float64") else F32
        if str(mesh_y.dtype) != str(mesh_x.dtype):
            raise ValueError("both meshes must have one precision")
        if not dev:
            mesh_x, mesh_y = np.ascontiguousarray(mesh_x), np.ascontiguousarray(mesh_y)
        nb = opts.nbins if opts.nbins > 0 else int(n / opts.ndel / 2)
        pk, px, py, kv = np.empty(nb), np.empty(nb), np.empty(nb), np.empty(nb)
        md = np.empty(nb, np.int64)
        g = make_grid(n, box)
        self._check(self._lib.cam_cross_power(self.h, ctypes.byref(g), L.ptr(mesh_x), L.ptr(mesh_y), prec,
                                              L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(opts), input_type_y,
                                              int(want_coeff), L.ptr(pk), L.ptr(px), L.ptr(py), L.ptr(md),
                                              L.ptr(kv)))
        return {"pk": pk, "pk_x": px, "pk_y": py, "modes": md, "kvector": kv}

    # ---------------------------------------------------------------- T-web
    @staticmethod
    def tweb_opts(R=0.0, lambda_th=0.0, tie_band=1e-5, input_type=L.INPUT_DENSITY, method=L.TWEB_FFT) -> L.TwebOpts:
        """method: L.TWEB_FFT (tidal tensor k_a k_b / k^2 delta_k) or L.TWEB_FD
        (finite differences of the potential, the reference's default)."""
        o = L.TwebOpts()
        o.smoothing_R, o.lambda_th, o.tie_band, o.input_type, o.method = R, lambda_th, tie_band, input_type, method
        return o

    def tweb_invariants(self, mesh, box: float, opts: L.TwebOpts):
        """cam_tweb_invariants: (labels, lambdas, invariants) with invariants
        (4, N, N, N) = I, II, III and the tidal anisotropy per cell."""
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        labels = self._empty((n, n, n), np.uint8, dev, mesh)
        lam = self._empty((3, n, n, n), np.float32, dev, mesh)
        inv = self._empty((4, n, n, n), np.float32, dev, mesh)
        st = L.TwebStats()
        g = make_grid(n, box)
        m = L.MEM_DEVICE if dev else L.MEM_HOST
        self._check(self._lib.cam_tweb_invariants(self.h, ctypes.byref(g), L.ptr(mesh), prec, m, ctypes.byref(opts),
                                                  L.ptr(labels), L.ptr(lam), L.ptr(inv), m, ctypes.byref(st)))
        return labels, lam, inv

    def tweb(self, mesh, box: float, opts: L.TwebOpts, want_lambdas=False) -> TwebResult:
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        labels = self._empty((n, n, n), np.uint8, dev, mesh)
        lam = self._empty((3, n, n, n), np.float32, dev, mesh) if want_lambdas else None
        st = L.TwebStats()
        g = make_grid(n, box)
        self._check(self._lib.cam_tweb(self.h, ctypes.byref(g), L.ptr(mesh), prec,
                                       L.MEM_DEVICE if dev else L.MEM_HOST, ctypes.byref(opts),
                                       L.ptr(labels), L.ptr(lam), L.MEM_DEVICE if dev else L.MEM_HOST,
                                       ctypes.byref(st)))
        return TwebResult(labels, lam, np.array(st.counts[:], np.int64), int(st.ties), st.mean)

    # ------------------------------------------------- potential / differences
    def poisson(self, delta, box: float, R: float = 0.0):
        """PoissonSolver (Source/Miscelanious.cpp:1189): phi with nabla^2 phi =
        delta (k = 0 mode dropped), optionally Gaussian-smoothed with radius R."""
        dev = L.is_device(delta)
        n = delta.shape[0]
        prec = F64 if str(delta.dtype).endswith("float64") else F32
        if not dev:
            delta = np.ascontiguousarray(delta)
        out = self._empty((n, n, n), np.float64 if prec == F64 else np.float32, dev, delta)
        g = make_grid(n, box)
        m = L.MEM_DEVICE if dev else L.MEM_HOST
        self._check(self._lib.cam_poisson(self.h, ctypes.byref(g), L.ptr(delta), prec, m, R, L.ptr(out), m))
        return out

    def gradfindif(self, field, box: float, dim: int, out=None):
        """gradfindif (Source/NumericalMethods.cpp:1123): 4th-order centred
        difference along dim (1 = x, the slowest axis; 3 = z)."""
        dev = L.is_device(field)
        n = field.shape[0]
        prec = F64 if str(field.dtype).endswith("float64") else F32
        if not dev:
            field = np.ascontiguousarray(field)
        if out is None:
            out = self._empty((n, n, n), np.float64 if prec == F64 else np.float32, dev, field)
        g = make_grid(n, box)
        m = L.MEM_DEVICE if dev else L.MEM_HOST
        self._check(self._lib.cam_gradfindif(self.h, ctypes.byref(g), L.ptr(field), prec, m, dim, L.ptr(out), m))
        return out

    # ---------------------------------------------------------------- catalogue
    def fkp_weights(self, n, nbar=None, nbar_const=0.0, w_in=None, fkp=True, P_est=0.0):
        """cam_fkp_weights: per-object weights w_in / (1 + P_est nbar) and the sums
        (n_selected, W_r, S_r, normal) of Catalog.cpp:14120-14190.  Arrays on the
        host or the device (all alike); returns (weights, sums)."""
        arrs = [a for a in (nbar, w_in) if a is not None]
        dev = bool(arrs) and L.is_device(arrs[0])
        nbar = nbar if (nbar is None or dev) else np.ascontiguousarray(nbar, np.float32)
        w_in = w_in if (w_in is None or dev) else np.ascontiguousarray(w_in, np.float32)
        out = self._empty((int(n),), np.float32, dev, arrs[0] if dev else None)
        sums = np.zeros(4)
        m = L.MEM_DEVICE if dev else L.MEM_HOST
        self._check(self._lib.cam_fkp_weights(self.h, int(n), L.ptr(nbar), float(nbar_const), L.ptr(w_in), int(fkp),
                                              float(P_est), m, L.ptr(out), m, L.ptr(sums)))
        return out, sums

    # ---------------------------------------------------------------- BAM kernel
    def bam_kernel_update(self, kernel, box: float, weight, mode=L.KERNEL_SET, DeltaKmin=0.0, ndel=1.0):
        """The 3D update of Bam::GetKernel (Source/Bam.cpp:786-910) on the
        half-complex kernel array (N, N, N/2+1), in place.  Returns the bin
        means of the updated kernel (bin 0 = mean of bins 1..4) and the
        element count of each bin."""
        dev = L.is_device(kernel)
        n = kernel.shape[0]
        prec = F64 if str(kernel.dtype).endswith("float64") else F32
        if not dev and not kernel.flags["C_CONTIGUOUS"]:
            raise ValueError("kernel must be C-contiguous (it is updated in place)")
        w = np.ascontiguousarray(weight, np.float64)
        nb = w.size
        binned = np.empty(nb)
        modes = np.empty(nb, np.int64)
        g = make_grid(n, box)
        self._check(self._lib.cam_bam_kernel_update(self.h, ctypes.byref(g), prec, DeltaKmin, ndel, nb, L.ptr(w),
                                                    mode, L.ptr(kernel), L.MEM_DEVICE if dev else L.MEM_HOST,
                                                    L.ptr(binned), L.ptr(modes)))
        return binned, modes

    def konvolve(self, mesh, box: float, kernel, out=None):
        """Bam::Konvolve (Source/Bam.cpp:1027): mesh convolved with the
        half-complex kernel, normalised by 2 sum(kernel) / N^3."""
        dev = L.is_device(mesh)
        n = mesh.shape[0]
        prec = F64 if str(mesh.dtype).endswith("float64") else F32
        if not dev:
            mesh = np.ascontiguousarray(mesh)
        kdev = L.is_device(kernel)
        if not kdev:
            kernel = np.ascontiguousarray(kernel)
        if out is None:
            out = self._empty((n, n, n), np.float64 if prec == F64 else np.float32, dev, mesh)
        g = make_grid(n, box)
        m = L.MEM_DEVICE if dev else L.MEM_HOST
        self._check(self._lib.cam_konvolve(self.h, ctypes.byref(g), L.ptr(mesh), prec, m, L.ptr(kernel),
                                           L.MEM_DEVICE if kdev else L.MEM_HOST, L.ptr(out), m))
        return out

    # ---------------------------------------------------------------- job
    def stage(self, x, y, z, w=None) -> "StagedParticles":
        """One host->device upload of a particle set, reusable by several jobs
        (cam_particles_stage); valid until the next stage() on this context."""
        p, keep, dev = self._particles(x, y, z, w)
        d = L.Particles()
        self._check(self._lib.cam_particles_stage(self.h, ctypes.byref(p), ctypes.byref(d)))
        return StagedParticles(d, keep)

    def job(self, x, y=None, z=None, w=None, grid: L.Grid = None, scheme: int = CIC, precision=F32,
            pk: L.PkOpts | None = None, tweb: L.TwebOpts | None = None, want_labels=False):
        """One mesh job (cam_job_run).  `x` may be a StagedParticles (then y, z,
        w are unused)."""
        j = JobSpec(x, y, z, w, grid=grid, scheme=scheme, precision=precision, pk=pk, tweb=tweb,
                    want_labels=want_labels)
        self._check(self._lib.cam_job_run(self.h, ctypes.byref(j.desc), ctypes.byref(j.res)))
        return j.result()

    def batch(self, jobs: list["JobSpec"]) -> list[dict]:
        """Runs jobs through cam_batch_run: consecutive jobs of one shape are
        packed into captured-graph batches.  Returns one result per job, as
        job() does (labels are not available in batches)."""
        n = len(jobs)
        descs = (L.JobDesc * n)(*[j.desc for j in jobs])
        ress = (L.JobResult * n)(*[j.res for j in jobs])
        rc = self._lib.cam_batch_run(self.h, descs, n, ress)
        for j, r in zip(jobs, ress):
            j.res = r  # filled for every job, also when one of them failed
        self._check(rc)
        return [j.result() for j in jobs]


class JobSpec:
    """A cam_job_desc with its host result arrays (and the particle arrays
    kept alive until the job is done)."""

    def __init__(self, x, y=None, z=None, w=None, grid: L.Grid = None, scheme: int = CIC, precision=F32,
                 pk: L.PkOpts | None = None, tweb: L.TwebOpts | None = None, want_labels=False):
        if isinstance(x, StagedParticles):
            p, self.keep = x.parts, x.keep
        else:
            dev = L.is_device(x)
            xs = tuple(_f32(a) for a in (x, y, z, w))
            p = L.Particles()
            p.n = int(xs[0].shape[0])
            p.x, p.y, p.z, p.w = (L.ptr(a) for a in xs)
            p.mem = L.MEM_DEVICE if dev else L.MEM_HOST
            self.keep = xs
        d = L.JobDesc()
        d.parts, d.grid, d.scheme, d.precision = p, grid, scheme, precision
        if pk is not None:
            d.pk = pk
        d.want_tweb = int(tweb is not None)
        if tweb is not None:
            d.tweb = tweb
        self.desc = d
        self.want_tweb = tweb is not None
        nb = 0
        if pk is not None:
            nb = pk.nbins if pk.nbins > 0 else int(grid.n[0] / pk.ndel / 2)
        self.nb = nb
        self.pk = np.empty(nb)
        self.modes = np.empty(nb, np.int64)
        self.kvector = np.empty(nb)
        n = grid.n[0]
        self.labels = np.empty((n, n, n), np.uint8) if (tweb is not None and want_labels) else None
        r = L.JobResult()
        r.pk, r.modes, r.kvector, r.labels = L.ptr(self.pk), L.ptr(self.modes), L.ptr(self.kvector), \
            L.ptr(self.labels)
        self.res = r

    def result(self) -> dict:
        r = self.res
        return {
            "pk": PkResult(self.pk, self.modes, self.kvector, r.pk_info.n_obj, r.pk_info.shot_noise,
                           r.pk_info.normal) if self.nb else None,
            "assign": AssignResult(None, r.assign.n_in, r.assign.n_lost, r.assign.sum_mesh),
            "tweb": TwebResult(self.labels, None, np.array(r.tweb.counts[:], np.int64), int(r.tweb.ties),
                               r.tweb.mean) if self.want_tweb else None,
        }


class Server:
    """Continuous-batching job server on one device (cam_server_*).

    submit() queues a JobSpec and returns its id; wait(id) returns the job's
    result dict (raising CamError on a failed job).  Jobs start as soon as a
    worker and the HBM budget allow; queued small jobs of one shape are
    packed into captured-graph batches."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, workers: int = 4, max_batch: int = 16):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.cam_server_create(device, hbm_budget, workers, max_batch, ctypes.byref(h))
        if rc != L.CAM_OK:
            raise CamError(rc, "cam_server_create failed")
        self.h = h
        self._jobs: dict[int, JobSpec] = {}

    def submit(self, job: JobSpec) -> int:
        jid = ctypes.c_uint64()
        rc = self._lib.cam_server_submit(self.h, ctypes.byref(job.desc), ctypes.byref(job.res), ctypes.byref(jid))
        if rc != L.CAM_OK:
            raise CamError(rc, "cam_server_submit failed")
        self._jobs[jid.value] = job
        return jid.value

    def wait(self, jid: int, timeout_s: float | None = None) -> dict:
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        job = self._jobs[jid]
        rc = job.status if hasattr(job, "status") else self._lib.cam_server_wait(self.h, jid, us)
        if rc == L.CAM_E_TIMEOUT:
            raise TimeoutError(f"job {jid} still running")
        self._jobs.pop(jid)
        if rc != L.CAM_OK:
            raise CamError(rc, f"job {jid} failed ({self._lib.cam_server_last_error(self.h).decode()})")
        return job.result()

    def poll(self, jid: int) -> bool:
        """True once the job has finished (its status is then kept for wait)."""
        rc = self._lib.cam_server_poll(self.h, jid)
        if rc == L.CAM_E_BUSY:
            return False
        self._jobs[jid].status = rc
        return True

    def stats(self, reset: bool = False) -> dict:
        st = L.ServerStats()
        rc = self._lib.cam_server_stats_get(self.h, ctypes.byref(st), int(reset))
        if rc != L.CAM_OK:
            raise CamError(rc, "cam_server_stats_get failed")
        return {f: getattr(st, f) for f, _ in L.ServerStats._fields_}

    def trace(self, max_records: int = 1 << 20) -> np.ndarray:
        """Completed jobs since the last call: structured array with id,
        submit_ms, start_ms, end_ms, worker, batch, status, big."""
        buf = (L.JobTrace * max_records)()
        cnt = ctypes.c_int()
        rc = self._lib.cam_server_trace(self.h, buf, max_records, ctypes.byref(cnt))
        if rc != L.CAM_OK:
            raise CamError(rc, "cam_server_trace failed")
        dt = np.dtype([(f, np.uint64 if f == "id" else (np.float64 if f.endswith("_ms") else np.int32))
                       for f, _ in L.JobTrace._fields_])
        return np.array([tuple(getattr(r, f) for f, _ in L.JobTrace._fields_) for r in buf[:cnt.value]], dtype=dt)

    def close(self):
        if self.h:
            self._lib.cam_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceLoop:
    """The persistent on-device request loop (cam_devloop_*): one resident
    kernel, one CTA of 1024 threads per SM (max_ctas: fewer, leaving SMs to
    other work), each running whole small jobs
    (FP32 cubic meshes of N = 32, 64, 128; device particles; P(k); no
    T-web) taken from a queue in mapped host memory.  submit() returns an
    id; wait() returns the job's result as Context.job does."""

    def __init__(self, device: int = 0, max_particles: int = 1 << 20, nslots: int = 4096,
                 idle_timeout_s: float = 10.0, max_ctas: int = 0):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.cam_devloop_create(device, int(max_particles), int(nslots), float(idle_timeout_s),
                                          int(max_ctas), ctypes.byref(h))
        if rc != L.CAM_OK:
            raise CamError(rc, "cam_devloop_create")
        self.h = h
        self._jobs: dict[int, JobSpec] = {}

    def _err(self, rc, what):
        msg = self._lib.cam_devloop_last_error(self.h)
        raise CamError(rc, f"{what}: {msg.decode() if msg else ''}")

    def submit(self, job: "JobSpec") -> int:
        jid = ctypes.c_uint64()
        rc = self._lib.cam_devloop_submit(self.h, ctypes.byref(job.desc), ctypes.byref(jid))
        if rc != L.CAM_OK:
            self._err(rc, "cam_devloop_submit")
        self._jobs[jid.value] = job
        return jid.value

    def wait(self, jid: int, timeout_s: float | None = None) -> dict:
        job = self._jobs[jid]
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        rc = self._lib.cam_devloop_wait(self.h, jid, us, ctypes.byref(job.desc), ctypes.byref(job.res))
        if rc != L.CAM_OK:
            self._err(rc, "cam_devloop_wait")
        del self._jobs[jid]
        return job.result()

    def state(self):
        """(status, running): status CAM_E_TIMEOUT once the kernel has ended
        on its idle limit."""
        r = ctypes.c_int()
        rc = self._lib.cam_devloop_state(self.h, ctypes.byref(r))
        return rc, r.value

    def close(self):
        if getattr(self, "h", None):
            self._lib.cam_devloop_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class StagedParticles:
    parts: L.Particles
    keep: tuple


_default: dict[int, Context] = {}
_default_lock = threading.Lock()


def alloc_stats(reset: bool = False) -> dict:
    """The library's device-allocation counters (cam_alloc_stats_get)."""
    st = L.AllocStats()
    rc = L.lib().cam_alloc_stats_get(ctypes.byref(st), int(reset))
    if rc != L.CAM_OK:
        raise CamError(rc, "cam_alloc_stats_get")
    return {"allocs": st.allocs, "failures": st.failures, "bytes": st.bytes, "total_ms": round(st.total_ms, 3),
            "max_ms": round(st.max_ms, 3)}


def default_context(device: int = 0) -> Context:
    with _default_lock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


# ---------------------------------------------------------------------------
# Reference-shaped entry points
# ---------------------------------------------------------------------------

def _getDensity(scheme, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass,
                delta, weightmass):
    g = make_grid((N1, N2, N3), (L1, L2, L3), (d1, d2, d3), (min1, min2, min3))
    w = Par_mass if weightmass else None
    prec = F64 if str(delta.dtype).endswith("float64") else F32
    out = delta.reshape(N1, N2, N3) if hasattr(delta, "reshape") else delta
    ctx = default_context()
    res = ctx.assign(xp, yp, zp, w, g, scheme, prec, out=out)
    return res.n_lost


def getDensity_NGP(N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta,
                   weightmass):
    """Source/massFunctions.cpp:35 -- fills ``delta`` (N1*N2*N3) in place; returns NLOSS."""
    return _getDensity(NGP, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass,
                       delta, weightmass)


def getDensity_CIC(N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta,
                   weightmass):
    """Source/massFunctions.cpp:678 -- fills ``delta`` in place; returns NLOSS."""
    return _getDensity(CIC, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass,
                       delta, weightmass)


def getDensity_TSC(N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass, delta,
                   weightmass):
    """Source/massFunctions.cpp:1050 -- fills ``delta`` in place; returns NLOSS."""
    return _getDensity(TSC, N1, N2, N3, L1, L2, L3, d1, d2, d3, min1, min2, min3, xp, yp, zp, Par_mass,
                       delta, weightmass)


def do_fftw_r2c(Nft, data_in, data_out):
    """Source/NumericalMethods.cpp:1718 -- unnormalised r2c into ``data_out``
    (N, N, N/2+1) complex."""
    res = default_context().fft_r2c(data_in.reshape(Nft, Nft, Nft))
    data_out[...] = res.reshape(data_out.shape)


def do_fftw_c2r(Nft, data_in, data_out):
    """Source/NumericalMethods.cpp:1818 -- c2r divided by N^3 into ``data_out``."""
    res = default_context().fft_c2r(data_in.reshape(Nft, Nft, Nft // 2 + 1))
    data_out[...] = res.reshape(data_out.shape)


def write_array(fname, data):
    """FileOutput::write_array, Source/FileOutput.cpp:858-912: the mesh as raw
    native-endian float32 (no header) into fname + ".dat"."""
    a = data.detach().cpu().numpy() if hasattr(data, "detach") else np.asarray(data)
    np.ascontiguousarray(a, np.float32).tofile(fname + ".dat")


def read_array(fname, out):
    """FileOutput::read_array, Source/FileOutput.cpp:727-752: out.size raw
    float32 values from fname (the name as given), into out."""
    a = np.fromfile(fname, np.float32, count=out.size)
    if a.size != out.size:
        raise CamError(L.CAM_E_INVAL, f"{fname}: {a.size} values, {out.size} expected")
    out.reshape(-1)[...] = a
    return out


def get_interpolated_density_field(x, y, z, grid: L.Grid, scheme: int, nbar=None, nbar_const=0.0, weights=None,
                                   fkp=True, P_est=0.0, precision=F32):
    """The catalogue's tracer loop, Source/Catalog.cpp:14104-14240: each object
    weighted by its other weights times the FKP weight 1 / (1 + P_est nbar),
    assigned with `scheme`; returns (mesh, sums) with sums = (n_selected, W_r,
    S_r, normal_power).  The assignment is the deterministic one of
    getDensity_* (the reference's OpenMP loop races on the mesh)."""
    ctx = default_context()
    w, sums = ctx.fkp_weights(len(x), nbar, nbar_const, weights, fkp, P_est)
    res = ctx.assign(x, y, z, w, grid, scheme, precision)
    return res.mesh, sums


def PoissonSolver(Lbox, Nft, data_in, data_out):
    """Source/Miscelanious.cpp:1189 -- the potential of ``data_in`` into ``data_out``."""
    res = default_context().poisson(data_in.reshape(Nft, Nft, Nft), Lbox)
    data_out[...] = res.reshape(data_out.shape)


def gradfindif(N1, N2, N3, L1, L2, L3, data_in, data_out, dim):
    """Source/NumericalMethods.cpp:1123 -- centred difference along ``dim`` into
    ``data_out`` (cubic meshes)."""
    if not (N1 == N2 == N3):
        raise CamError(L.CAM_E_UNSUPPORTED, "gradfindif: cubic meshes only")
    res = default_context().gradfindif(data_in.reshape(N1, N2, N3), L1, dim)
    data_out[...] = res.reshape(data_out.shape)


def EigenValuesTweb(Nft, L1, delta, *args):
    """Both reference overloads, eigenvalues in descending order into the last
    three arguments:
    EigenValuesTweb(Nft, L1, delta, out1, out2, out3), Source/Miscelanious.cpp:1772
        -- tidal tensor of delta by FFTs;
    EigenValuesTweb(Nft, L1, delta, phi, out1, out2, out3), Source/Miscelanious.cpp:1663
        -- finite-difference Hessian of the potential phi (the default build)."""
    if len(args) == 3:
        mesh, opts = delta, Context.tweb_opts(0.0, 0.0, 0.0, L.INPUT_DELTA, L.TWEB_FFT)
    elif len(args) == 4:
        mesh, opts = args[0], Context.tweb_opts(0.0, 0.0, 0.0, L.INPUT_POTENTIAL, L.TWEB_FD)
        args = args[1:]
    else:
        raise TypeError("EigenValuesTweb(Nft, L1, delta, [phi,] out1, out2, out3)")
    r = default_context().tweb(mesh.reshape(Nft, Nft, Nft), L1, opts, want_lambdas=True)
    for a, out in enumerate(args):
        out[...] = r.lambdas[a].reshape(out.shape)


@dataclass
class Params:
    """The Params getters the hot path reads (Headers/Params.h): _Nft, _Lbox,
    _mass_assignment (0 NGP, 1 CIC, 2 TSC), _MAS_correction, _SN_correction,
    _input_type ("density_grid" | "delta_grid"), _ndel_data, _DeltaKmin,
    _lambdath; smoothing_R is the Gaussian radius applied before the T-web.
    tweb_method picks the tidal tensor, as the reference's compile-time
    switch does (Headers/def.h:2657-2658): "fft" (_USE_GFFT_EIGENV_) or
    "fd" (_USE_GFINDIFF_EIGENV_, the reference's default build)."""
    Nft: int
    Lbox: float
    mass_assignment: int = CIC
    MAS_correction: bool = True
    SN_correction: bool = True
    input_type: str = "density_grid"
    input_type_two: str = "density_grid"
    ndel_data: float = 1.0
    DeltaKmin: float = 0.0
    Nnp_data: int = 0
    lambdath: float = 0.0
    smoothing_R: float = 0.0
    tie_band: float = 1e-5
    tweb_method: str = "fft"
    device: int = 0


class PowerSpectrumF:
    """Source/PowerSpectrumF.cpp:1739 (compute_power_spectrum_grid) with the
    accessors of Headers/PowerSpectrumF.h."""

    def __init__(self, params: Params):
        self.params = params
        self.pk0 = np.zeros(0)
        self.modes_g = np.zeros(0, np.int64)
        self.kvector_data = np.zeros(0)

    def compute_power_spectrum_grid(self, data_in, write_to_file=False):
        p = self.params
        it = L.INPUT_DENSITY if p.input_type == "density_grid" else L.INPUT_DELTA
        o = Context.pk_opts(p.mass_assignment, p.Nnp_data, p.ndel_data, p.DeltaKmin, p.MAS_correction,
                            p.SN_correction, it)
        mesh = data_in.reshape(p.Nft, p.Nft, p.Nft)
        r = default_context(p.device).power(mesh, p.Lbox, o)
        self.pk0, self.modes_g, self.kvector_data = r.pk, r.modes, r.kvector
        self.shot_noise, self.normal_power, self.ngal = r.shot_noise, r.normal, r.n_obj
        if write_to_file:
            raise CamError(L.CAM_E_UNSUPPORTED, "file output is not part of the GPU path")

    def compute_cross_power_spectrum_grid(self, dm, X, Y, get_cross_coeff=False):
        """Source/PowerSpectrumF.cpp:549: X uses input_type, Y input_type_two
        (Params.input_type_two); fills pk0, modes_g, kvector_data."""
        p = self.params
        n = p.Nft
        it = L.INPUT_DENSITY if p.input_type == "density_grid" else L.INPUT_DELTA
        it2 = L.INPUT_DENSITY if p.input_type_two == "density_grid" else L.INPUT_DELTA
        o = Context.pk_opts(p.mass_assignment, p.Nnp_data, p.ndel_data, p.DeltaKmin, p.MAS_correction, False, it)
        r = default_context(p.device).cross_power(X.reshape(n, n, n), Y.reshape(n, n, n), p.Lbox, o, it2,
                                                  get_cross_coeff)
        self.pk0, self.modes_g, self.kvector_data = r["pk"], r["modes"], r["kvector"]

    def _pk0(self, i):
        return self.pk0[i]

    def _nmodes_k(self, i):
        return self.modes_g[i]

    def _kvector_data(self, i):
        return self.kvector_data[i]


I_KNOT, I_FILAMENT, I_SHEET, I_VOID = 1, 2, 3, 4


class Cwclass:
    """Source/Cwclass.cpp:235 (get_CWC) with the public members lambda1..3,
    CWClass and the volume fractions of Headers/Cwclass.h."""

    def __init__(self, params: Params):
        self.params = params

    def get_CWC(self, delta):
        p = self.params
        it = L.INPUT_DELTA if p.input_type == "delta_grid" else L.INPUT_DENSITY
        method = {"fft": L.TWEB_FFT, "fd": L.TWEB_FD}[p.tweb_method]
        o = Context.tweb_opts(p.smoothing_R, p.lambdath, p.tie_band, it, method)
        r = default_context(p.device).tweb(delta.reshape(p.Nft, p.Nft, p.Nft), p.Lbox, o, want_lambdas=True)
        ng = float(p.Nft) ** 3
        self.lambda1, self.lambda2, self.lambda3 = (r.lambdas[0].reshape(-1), r.lambdas[1].reshape(-1),
                                                    r.lambdas[2].reshape(-1))
        self.CWClass = r.labels.reshape(-1)
        self.volume_knots, self.volume_filaments, self.volume_sheets, self.volume_voids = (
            r.counts[0] / ng, r.counts[1] / ng, r.counts[2] / ng, r.counts[3] / ng)
        self.ties = r.ties

    do_CWC = get_CWC


class Bam:
    """The kernel steps of a BAM calibration iteration (Source/Bam.cpp):
    GetKernel (:529) updates the Fourier-space kernel from the ratio of the
    reference to the current power spectrum, Konvolve (:1027) convolves a
    mesh with it.  The kernel lives on the device, (N, N, N/2+1) real_prec,
    initialised to 1 (:243).  Power_REF, Power_NEW, kvec (h/Mpc) and
    shot_noise_ref are set by the caller, as the reference's members are."""

    SEED = 55457  # gsl_rng_default_seed of GetKernel (Source/Bam.cpp:594)

    def __init__(self, params: Params):
        import torch
        self.params = params
        n = params.Nft
        self.Kernel = torch.ones((n, n, n // 2 + 1), dtype=torch.float32, device=f"cuda:{params.device}")
        # filled on torch's stream; the library context launches on its own
        torch.cuda.synchronize(params.device)
        nb = params.Nnp_data if params.Nnp_data > 0 else int(n / params.ndel_data / 2)
        self.kvec = np.zeros(nb)
        self.Power_REF = np.zeros(nb)
        self.Power_NEW = np.zeros(nb)
        self.power_ratio_unsmoothed = np.ones(nb)
        self.shot_noise_ref = 0.0
        self.kernel_updated = np.zeros(nb)
        self.nmodes = np.zeros(nb, np.int64)

    def kernel_weights(self, rejection: bool, exponent: float, uniforms=None):
        """The per-bin weights of GetKernel (Source/Bam.cpp:604-723), host side
        (one value per bin).  With rejection, a bin takes its new ratio when a
        uniform draw is below min(1, chi2_old / chi2_new); `uniforms` are
        those draws (default: MT19937 seeded with init_genrand(55457), the
        stream of gsl_rng_mt19937, one 32-bit output / 2^32 per bin)."""
        nb = self.kvec.size
        p = self.params
        weight = np.ones(nb)
        if rejection and uniforms is None:
            rs = np.random.RandomState(self.SEED)
            uniforms = rs.randint(0, 2 ** 32, size=nb, dtype=np.uint64) / 4294967296.0
        dk = 2.0 * np.pi / p.Lbox
        sfac = 1.0 / (2.0 * np.pi * dk * p.Lbox ** 3)
        for i in range(nb):
            pr, pn = float(self.Power_REF[i]), float(self.Power_NEW[i])
            if 0 <= exponent < 1.0:
                ratio = 1.0 if (pn == 0 or pr == 0) else abs(pr / pn) ** exponent
            else:
                ratio = 1.0 if pn == 0 else pr / pn
            if not rejection:
                weight[i] = ratio
            else:
                k2 = self.kvec[i] ** 2
                inv = sfac / (k2 + dk * dk / 12.0)
                s_new = 1.0 if pr == 0 else inv * pn * pn
                new_h = 0.5 * (pr - pn) ** 2 / s_new
                p_old = pr / self.power_ratio_unsmoothed[i]
                s_old = 1.0 if pr == 0 else inv * (p_old + self.shot_noise_ref) ** 2
                old_h = 0.5 * (pr - p_old) ** 2 / s_old
                with np.errstate(divide="ignore", invalid="ignore"):
                    ratio_diff = np.float64(old_h) / np.float64(new_h)
                if uniforms[i] < min(1.0, ratio_diff):
                    weight[i] = ratio
            self.power_ratio_unsmoothed[i] = ratio
        return weight.astype(np.float32).astype(np.float64)

    def GetKernel(self, rejection: bool, exponent: float, uniforms=None):
        p = self.params
        w = self.kernel_weights(rejection, exponent, uniforms)
        mode = L.KERNEL_SCALE if rejection else L.KERNEL_SET
        self.kernel_updated, self.nmodes = default_context(p.device).bam_kernel_update(
            self.Kernel, p.Lbox, w, mode, p.DeltaKmin, p.ndel_data)

    def Konvolve(self, data_in, data_out):
        p = self.params
        n = p.Nft
        res = default_context(p.device).konvolve(data_in.reshape(n, n, n), p.Lbox, self.Kernel)
        data_out[...] = res.reshape(data_out.shape)

    def get_invariants(self, delta):
        """get_CWC plus the invariant fields of the tidal tensor that BAM's
        bias binning uses (invariant_field_I/II/III, tidal_anisotropy,
        Source/Miscelanious.cpp:1460-1492), as members I, II, III, tidal."""
        p = self.params
        it = L.INPUT_DELTA if p.input_type == "delta_grid" else L.INPUT_DENSITY
        method = {"fft": L.TWEB_FFT, "fd": L.TWEB_FD}[p.tweb_method]
        o = Context.tweb_opts(p.smoothing_R, p.lambdath, p.tie_band, it, method)
        labels, lam, inv = default_context(p.device).tweb_invariants(delta.reshape(p.Nft, p.Nft, p.Nft), p.Lbox, o)
        self.CWClass = labels.reshape(-1)
        self.lambda1, self.lambda2, self.lambda3 = (lam[a].reshape(-1) for a in range(3))
        self.I, self.II, self.III, self.tidal = (inv[a].reshape(-1) for a in range(4))

    def get_Tclassification(self, ig):
        return int(self.CWClass[ig])
