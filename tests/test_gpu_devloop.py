"""The persistent on-device request loop (cam_devloop_*) against cam_job_run.

The loop runs whole jobs inside one resident kernel, one CTA per job.  Its
assignment uses the same device functions and fixed-point scale as
cam_job_run, so the lost count and the mesh sum are bit-identical.  Its
FFT holds 8 points per thread (radix-8 stages; cam_job_run's 16-point
threads take radix-16 stages where that saves a pass) and it bins each
mode's power in FP64 (cam_job_run: FP32 per mode, FP64 bins), so P(k)
agrees to FP32 rounding (2e-6 here), with identical mode counts.  A job's
result does not depend on the jobs that ran beside it, and every
device-side wait is bounded: with no job for the idle limit the kernel
ends, and the next submission relaunches it.  The loops here use half the
SMs, so the cam_job_run references run beside them.
"""
import time

import numpy as np
import pytest

from conftest import pk_rel_err
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, NGP, TSC, CamError, Context, DeviceLoop, JobSpec, make_grid

pytestmark = pytest.mark.gpu


def _parts(npart, box, seed, weighted):
    import torch
    x, y, z = synth.clumped(npart, box, max(1, npart // 100), 2.0, 0.8, seed)
    w = synth.halo_masses(npart, seed=seed + 1) if weighted else None
    return [torch.from_numpy(v).cuda() for v in (x, y, z)] + ([torch.from_numpy(w).cuda()] if weighted else [None])


def _close(a, b):
    assert a["assign"].n_lost == b["assign"].n_lost
    assert a["assign"].sum_mesh == b["assign"].sum_mesh
    assert np.array_equal(a["pk"].modes, b["pk"].modes)
    floor = np.abs(b["pk"].shot_noise) * np.ones(len(b["pk"].pk))
    assert pk_rel_err(a["pk"].pk, b["pk"].pk, floor) <= 2e-6


@pytest.fixture(scope="module")
def loop():
    # half the SMs: the cam_job_run references run beside it
    lp = DeviceLoop(0, max_particles=1 << 20, nslots=1024, idle_timeout_s=20.0, max_ctas=74)
    yield lp
    lp.close()


@pytest.mark.parametrize("n,scheme,weighted,npart", [(32, CIC, False, 50_000), (64, CIC, False, 262_144),
                                                     (64, TSC, True, 200_000), (128, NGP, False, 300_000),
                                                     (128, TSC, False, 500_000), (64, NGP, True, 100_000)])
def test_devloop_matches_job_run(ctx, loop, n, scheme, weighted, npart):
    import torch
    box = 500.0
    x, y, z, w = _parts(npart, box, n + scheme, weighted)
    torch.cuda.synchronize()
    g = make_grid(n, box)
    opts = Context.pk_opts(scheme, nbins=n // 2)
    ref = ctx.job(x, y, z, w, g, scheme, F32, pk=opts)
    got = loop.wait(loop.submit(JobSpec(x, y, z, w, grid=g, scheme=scheme, precision=F32, pk=opts)), 60.0)
    _close(got, ref)


def test_devloop_job_alone_equals_in_mix(loop):
    import torch
    box = 400.0
    jobs = []
    rng = np.random.default_rng(3)
    for k in range(96):
        n = int(rng.choice([32, 64, 128]))
        s = int(rng.integers(0, 3))
        x, y, z, w = _parts(int(rng.integers(20_000, 200_000)), box, 100 + k, bool(k % 2))
        jobs.append(JobSpec(x, y, z, w, grid=make_grid(n, box), scheme=s, precision=F32,
                            pk=Context.pk_opts(s, nbins=n // 2)))
    torch.cuda.synchronize()
    alone = loop.wait(loop.submit(jobs[40]), 60.0)
    ids = [loop.submit(j) for j in jobs]
    res = [loop.wait(i, 60.0) for i in ids]
    mixed = res[40]
    assert mixed["assign"].sum_mesh == alone["assign"].sum_mesh
    assert np.array_equal(mixed["pk"].pk, alone["pk"].pk)
    assert np.array_equal(mixed["pk"].modes, alone["pk"].modes)


def test_devloop_idle_limit_ends_the_kernel_and_a_submission_relaunches_it(ctx):
    import torch
    lp = DeviceLoop(0, max_particles=1 << 18, nslots=16, idle_timeout_s=0.2, max_ctas=74)
    try:
        time.sleep(1.0)  # no job: every CTA's bounded wait runs out
        rc, running = lp.state()
        assert rc == L.CAM_E_TIMEOUT and running == 0
        box = 300.0
        x, y, z, w = _parts(60_000, box, 9, False)
        torch.cuda.synchronize()
        g = make_grid(64, box)
        opts = Context.pk_opts(CIC, nbins=32)
        got = lp.wait(lp.submit(JobSpec(x, y, z, None, grid=g, scheme=CIC, precision=F32, pk=opts)), 60.0)
        _close(got, ctx.job(x, y, z, None, g, CIC, F32, pk=opts))
    finally:
        lp.close()


def test_devloop_rejects_jobs_outside_its_scope(loop):
    import torch
    x, y, z, _ = _parts(1000, 100.0, 5, False)
    for kw in (dict(grid=make_grid(256, 100.0)), dict(grid=make_grid(64, 100.0), precision=1),
               dict(grid=make_grid(64, 100.0), tweb=Context.tweb_opts(2.0, 0.0, 1e-5))):
        spec = JobSpec(x, y, z, None, scheme=CIC, pk=Context.pk_opts(CIC, nbins=16), **{"precision": F32, **kw})
        with pytest.raises(CamError) as e:
            loop.submit(spec)
        assert e.value.code == L.CAM_E_UNSUPPORTED
    hx = x.cpu().numpy()
    spec = JobSpec(hx, hx, hx, None, grid=make_grid(64, 100.0), scheme=CIC, precision=F32,
                   pk=Context.pk_opts(CIC, nbins=16))
    with pytest.raises(CamError):
        loop.submit(spec)
