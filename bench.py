"""Mesh-job throughput of the CosmicAtlas/BAM hot path on B200.

Workload (the scheme-sweep configuration): 16,777,216 float32 particles from
the clumped process (20% uniform, 80% in 200,000 Gaussian clumps of
sigma = 1.5 Mpc/h) in a periodic box L = 1000 Mpc/h, halo-like masses
log10 M ~ N(12.5, 0.5) truncated to [11, 15].  One step = three mesh jobs
(NGP, CIC, TSC), each: mass assignment onto 256^3 FP32 -> r2c FFT -> P(k) in
128 bins with window deconvolution and shot-noise subtraction.

value : jobs/s with the particles resident in HBM (device pointers).
e2e   : jobs/s through the C ABI with pinned host particle buffers: every
        step uploads the step's particles once (cam_particles_stage) and runs
        the three jobs on them; the host->device copy and the device->host
        copies of the P(k) results are inside the timed region.  Two contexts
        on two streams alternate steps, and each step's upload is issued
        before the previous step's jobs (the copy engine overlaps them).
Multi-GPU: one process per GPU, each runs its own jobs (independent meshes,
"weak" scaling, no collective in the data path); time is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PARTICLES = 16_777_216
NMESH = 256
BOX = 1000.0
NBINS = 128
SCHEMES = (0, 1, 2)  # NGP, CIC, TSC
METRIC = "mesh-jobs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--kernels-only", action="store_true",
                    help="profiler runs: the device-resident pass only (no e2e pass, no CPU baseline)")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "single512", "large768", "c1", "calib", "calib_pk",
                                                             "stream", "bam"],
                    help="sweep: the benchmark line (default); single512 / large768 / c1: one-job latency lines; "
                         "calib / stream: served vs plain per-call jobs/s and latency")
    ap.add_argument("--jobs", type=int, default=0, help="calib / stream: number of jobs (0 = the config's)")
    ap.add_argument("--rates", default="50,200,800", help="stream: Poisson arrival rates (jobs/s)")
    ap.add_argument("--held-gb", type=float, default=24.0,
                    help="stream: GB of submitted jobs' inputs the client may hold before it waits")
    ap.add_argument("--serving-jobs", type=int, default=4096,
                    help="sweep: jobs of the calibration batch timed served vs per-call on the same line (0: skip)")
    ap.add_argument("--stream-jobs", type=int, default=2000,
                    help="sweep: jobs of the mixed stream timed served vs per-call on the same line (0: skip)")
    ap.add_argument("--stream-rates", default="200",
                    help="sweep: Poisson arrival rates of the mixed stream on the same line (besides saturation)")
    ap.add_argument("--mesh", type=int, default=0, help="single512 only: override N (profiler runs)")
    ap.add_argument("--tweb-method", default="fft", choices=["fft", "fd"],
                    help="single-job workloads: T-web tidal tensor by FFTs (k_a k_b / k^2) or by the "
                         "reference's default finite differences")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def max_over_ranks(ms, device="cuda"):
    """The slowest rank's time (every rank gets it); one rank: ms itself.
    Jobs are replicas with no collective in their data path, so this is the
    only exchange of a timed region."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(jobs_per_rank, world, ms_max):
    """Throughput of all ranks together: every rank's jobs over the slowest
    rank's time (weak scaling: per-rank work is fixed as ranks are added)."""
    return jobs_per_rank * world / (ms_max / 1e3)


def rank_seed(base, rank):
    """Each rank draws its own catalogue (independent jobs per replica)."""
    return base + 1000 * rank


def config_dict(n_particles, extra=None):
    d = {"workload": "scheme sweep: %d clumped weighted particles, L=1000, NGP+CIC+TSC onto 256^3 FP32, "
                     "r2c FFT, P(k) 128 bins" % n_particles,
         "particles": n_particles, "mesh": NMESH, "box": BOX, "nbins": NBINS,
         "jobs_per_step": len(SCHEMES),
         "l2": "inputs larger than L2 (268 MB particles, 64 MB mesh, 135 MB spectrum per job)"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """SM clock, max clock and clock-event (throttle) reasons of the GPU,
    sampled every `period_s` (5 ms) through NVML while the timed region runs
    (reading only; nvidia-smi -lms 100 if NVML is unavailable)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period_s = period_s
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.proc = None
        self.thread = None
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            p = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        get_r = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), float(mx), int(get_r(h))))
            except Exception:
                pass
            self.stop.wait(self.period_s)

    def _sample_now(self):
        if self.nv is None:
            return
        nv, h = self.nv
        get_r = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        try:
            self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                 float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)), int(get_r(h))))
        except Exception:
            pass

    def __enter__(self):
        self.nv = None
        try:
            nv, h = self._nvml_handle()
            self.nv = (nv, h)
            # one sample at the start (short timed regions), then every 5 ms
            self._sample_now()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            pass
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 3.0:  # first line before the timed region
                time.sleep(0.01)
            self.samples.clear()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read_smi(self):
        bits = [0x8, 0x40, 0x20, 0x4]
        for line in self.proc.stdout:
            f = [v.strip() for v in line.split(",")]
            try:
                r = sum(b for i, b in enumerate(bits) if len(f) > 5 + i and f[5 + i].lower().startswith("active"))
                self.samples.append((float(f[1]), float(f[2]), r))
            except ValueError:
                pass

    def __exit__(self, *a):
        self._sample_now()  # and one at the end
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        reasons = sorted(n for n, b in self.REASONS.items() if any(s[2] & b for s in self.samples))
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml" if self.proc is None else "nvidia-smi"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant stage's kernels from the
    committed ncu summary (profiles/ncu_traffic.json), if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


def cufft_r2c_ms(n, stream, reps=20):
    """Mean time of torch.fft.rfftn (cuFFT) on an n^3 FP32 device mesh."""
    import torch
    m = torch.randn((n, n, n), device="cuda", dtype=torch.float32)
    for _ in range(3):
        torch.fft.rfftn(m)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.current_stream())
    for _ in range(reps):
        torch.fft.rfftn(m)
    e1.record(torch.cuda.current_stream())
    torch.cuda.synchronize()
    del m
    return e0.elapsed_time(e1) / reps


def ours_r2c_ms(ctx, n, reps=20):
    """Mean time of the library's own r2c alone (cam_fft_r2c on an n^3 FP32
    device mesh: no P(k) binning; its FFTW-layout output costs one layout
    copy more than the jobs' internal layout), CUDA events on the launching
    stream: the like-for-like counterpart of cufft_r2c_ms.  The context
    launches on torch's current stream (set by the caller)."""
    import torch
    m = torch.randn((n, n, n), device="cuda", dtype=torch.float32)
    st = torch.cuda.current_stream()
    for _ in range(3):
        ctx.fft_r2c(m)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        ctx.fft_r2c(m)
    e1.record(st)
    torch.cuda.synchronize()
    del m
    return e0.elapsed_time(e1) / reps


def pk_error_vs_oracle(x, y, z, w, pks):
    """max over bins of |P - P_oracle| / max(|P_oracle|, SN C(k)/W^2) for each
    scheme's job: the FP64 oracle assigns the same particles and bins the
    FP64 spectrum (the error metric of the P(k) tests)."""
    orc = _cpu_oracle()
    out = {}
    for s in SCHEMES:
        mesh, _ = orc.assign_f64_mt(s, x, y, z, w, orc.Grid.cubic(NMESH, BOX))
        ref = orc.power_grid(mesh, BOX, s, NBINS)
        floor = np.maximum(np.abs(ref.pk), np.abs(ref.shot_noise * ref.sum_sn / np.maximum(ref.modes, 1)))
        got = np.asarray(pks[s].pk, np.float64)
        has = ref.modes > 0
        out[("ngp", "cic", "tsc")[s]] = float(np.max(np.abs(got - ref.pk)[has] / floor[has]))
    out["max"] = max(out.values())
    out["note"] = "last timed step's three jobs vs the FP64 oracle (oracle/), computed after the timed region"
    return out


# -------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from cosmicatlas_b200 import synth
    from cosmicatlas_b200.api import Context, make_grid

    rank, local, world = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    npart = args.particles
    x, y, z = synth.clumped(npart, BOX, 200_000, 1.5, 0.8, seed=rank_seed(2, rank))
    w = synth.halo_masses(npart, seed=rank_seed(1002, rank))
    dev = [torch.from_numpy(v).cuda() for v in (x, y, z, w)]
    pinned = [torch.from_numpy(v).pin_memory() for v in (x, y, z, w)]
    grid = make_grid(NMESH, BOX)
    ctx = Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    opts = {s: Context.pk_opts(s, nbins=NBINS) for s in SCHEMES}

    last_pk = {}

    def step(arrs, lat=None):
        # host arrays: one upload per step serves the three schemes
        src = arrs if arrs[0].is_cuda else [ctx.stage(*arrs)]
        for s in SCHEMES:
            if lat is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            if len(src) == 1:
                r = ctx.job(src[0], grid=grid, scheme=s, precision=0, pk=opts[s])
            else:
                r = ctx.job(src[0], src[1], src[2], src[3], grid, s, 0, pk=opts[s])
            if lat is not None:
                e1.record(stream)
                lat.append((e0, e1))
            last_pk[s] = r["pk"]
        return r

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # second context for the host-fed pass: step i+1's upload (an
    # asynchronous copy on its stream) runs under step i's jobs
    ctx_b = Context(local)
    stream_b = torch.cuda.Stream()
    ctx_b.set_stream(stream_b.cuda_stream)
    ctxs = (ctx, ctx_b)

    def host_fed(k):
        staged = [None, None]
        staged[0] = ctxs[0].stage(*pinned)
        r = None
        for i in range(k):
            if i + 1 < k:
                staged[(i + 1) % 2] = ctxs[(i + 1) % 2].stage(*pinned)
            c, src = ctxs[i % 2], staged[i % 2]
            for s in SCHEMES:
                r = c.job(src, grid=grid, scheme=s, precision=0, pk=opts[s])
        return r

    def timed_host_fed(k):
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        host_fed(k)
        # every job has returned its P(k) to the host: all work is done
        t1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(t0.elapsed_time(t1))
        barrier()
        return ms

    def timed(arrs, k, lat=None):
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(k):
            step(arrs, lat)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(t0.elapsed_time(t1))
        barrier()
        return ms

    for _ in range(args.warmup):
        step(dev)
        if not args.kernels_only:
            host_fed(2)
    # device-resident inputs: the headline `value`
    lat = []
    launches0 = ctx.kernel_launches
    with ClockSampler(local) as clk:
        ms = timed(dev, args.steps, lat)
    launches = ctx.kernel_launches - launches0
    job_ms = sorted(a.elapsed_time(b) for a, b in lat)
    # per-kernel CUDA-event times from a separate, untimed pass
    prof_steps = min(args.steps, 10)
    ctx.profile(True)
    ctx.profile_read(reset=True)
    for _ in range(prof_steps):
        step(dev)
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    # end to end: pinned host particles in, P(k) out
    ms_e2e = timed_host_fed(args.steps) if not args.kernels_only else float("nan")

    # the FFT stage against cuFFT (torch.fft.rfftn on the device), comparison only
    cufft_ms = cufft_r2c_ms(NMESH, stream) if rank == 0 else None
    plain_fft_ms = ours_r2c_ms(ctx, NMESH) if rank == 0 else None
    # P(k) of the last timed step's three jobs against the FP64 oracle
    # (outside the timed region)
    pk_err = pk_error_vs_oracle(x, y, z, w, last_pk) if rank == 0 and not args.kernels_only else None

    jobs = len(SCHEMES) * args.steps * world
    value = whole_job_rate(len(SCHEMES) * args.steps, world, ms)
    e2e = whole_job_rate(len(SCHEMES) * args.steps, world, ms_e2e)
    h2d = npart * 16
    d2h = len(SCHEMES) * NBINS * 24

    out = None
    if rank == 0:
        hbm, peak_kind = peaks()
        jobs_rank = len(SCHEMES) * prof_steps  # jobs of the profiled pass
        # stage roofline: algorithmic bytes per job (unit = one mesh job)
        nh = NMESH * NMESH * (NMESH // 2 + 1)
        stage_bytes = {
            "assign": npart * (12 + 4) + 4 * NMESH ** 3,
            "fft_r2c": 4 * NMESH ** 3 + 8 * nh,
            "power": 8 * nh,
        }
        stage_kernels = {
            "assign": ["assign_bin_count", "assign_starts", "assign_partition", "tile_sum_kernel", "tile_offsets_kernel",
                       "tile_scan_kernel", "assign_bin_scatter", "assign_deposit", "partial_sum_kernel<double>",
                       "final_sum_kernel"],
            # fft_cols_pk: the x pass that also bins P(k) (the binning adds no traffic)
            "fft_r2c": ["fft_rows_r2c", "fft_cols", "fft_rows_c2c", "fft_cols_pk"],
            "power": ["pk_bin", "pk_final_kernel", "pk_nyq", "pk_final"],
        }
        # kernels on the side stream run beside the stage's main-stream
        # kernels: reported per stage, not added to its time
        side_kernels = {"fft_r2c": ["side.fft_rows_c2c", "side.fft_cols"], "power": ["side.pk_nyq"]}
        # P(k) binned inside the r2c's x pass: its spectrum read is that
        # pass's; the power stage only reduces per-CTA partial sums
        fused_pk = "fft_cols_pk" in prof
        if fused_pk:
            stage_bytes["power"] = None
        stages = {}
        for st, names in stage_kernels.items():
            t = sum(prof.get(nm, (0, 0.0))[1] for nm in names) / jobs_rank
            ach = stage_bytes[st] / (t / 1e3) / 1e9 if t > 0 and stage_bytes[st] else None
            stages[st] = {"ms_per_job": round(t, 4), "algorithmic_bytes": stage_bytes[st],
                          "achieved_gbs": round(ach, 1) if ach else None,
                          "frac": round(ach / hbm, 4) if ach else None}
            if st == "power" and fused_pk:
                stages[st]["note"] = ("the spectrum is binned inside the r2c's x pass (fft_r2c stage); these "
                                      "kernels reduce the per-CTA partial sums")
            ov = sum(prof.get(nm, (0, 0.0))[1] for nm in side_kernels.get(st, [])) / jobs_rank
            if ov > 0:
                stages[st]["overlapped_ms_per_job"] = round(ov, 4)
                stages[st]["overlapped_note"] = ("the Nyquist plane's kernels, on a side stream beside the "
                                                 "main-stream kernels above")
        dom = max(stages, key=lambda s: stages[s]["ms_per_job"])
        traffic = ncu_traffic()
        dom_traffic = traffic.get(dom) if isinstance(traffic, dict) else None
        # the single kernel with the most time, with its ncu DRAM bytes
        kname, (kl, kms) = max(prof.items(), key=lambda t: t[1][1])
        kbytes = (traffic or {}).get("kernels", {}).get(kname)
        dominant_kernel = {"name": kname, "ms_per_launch": round(kms / max(kl, 1), 4),
                           "dram_bytes_per_launch": kbytes,
                           "dram_gbs": round(kbytes / (kms / max(kl, 1) / 1e3) / 1e9, 1) if kbytes else None}
        kernels = {k: {"launches": v[0], "ms_total": round(v[1], 3)} for k, v in sorted(prof.items())}
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "jobs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded clumped process, halo-like masses)",
            "config": config_dict(npart, {"parallelism": f"job replicas x{world}"}),
            "latency_ms": {"p50": round(float(np.percentile(job_ms, 50)), 3),
                           "p99": round(float(np.percentile(job_ms, 99)), 3)},
            "e2e": {"value": round(e2e, 3), "unit": "jobs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "cam_particles_stage + 3 x cam_job_run per step; two contexts alternate steps, "
                            "each upload issued before the previous step's jobs"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "stage": dom, "achieved": stages[dom]["achieved_gbs"],
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": stages[dom]["frac"], "traffic": dom_traffic,
                         "note": "stage = the kernels that implement one assignment (algorithmic bytes "
                                 "N_p*16 + 4*N^3 per job); traffic = their ncu DRAM bytes per job",
                         "traffic_path": (traffic or {}).get("path"),
                         "dominant_kernel": dominant_kernel},
            "stages": stages,
            "kernels": kernels,
            "clocks": clk.summary(),
        }
        if cufft_ms is not None:
            out["stages"]["fft_r2c"]["cufft_ms"] = round(cufft_ms, 4)
            out["stages"]["fft_r2c"]["cufft_note"] = ("torch.fft.rfftn of a 256^3 FP32 device mesh (cuFFT), CUDA "
                                                      "events, comparison only: not on the product path")
            out["stages"]["fft_r2c"]["plain_ms"] = round(plain_fft_ms, 4)
            out["stages"]["fft_r2c"]["plain_note"] = ("cam_fft_r2c alone on the same mesh (no P(k) binning, "
                                                      "FFTW-layout output), CUDA events; ms_per_job above is the "
                                                      "jobs' r2c with P(k) binned in its last pass")
        if pk_err is not None:
            out["pk_rel_err"] = pk_err["max"]
            out["pk_rel_err_detail"] = pk_err
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out, (x, y, z, w)


def _cpu_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    return orc


def cpu_job(orc, scheme, x, y, z, w, assign="reference", threads=0):
    """One scheme-sweep job on the host, as the reference runs it:
    assign = "reference": the reference's own getDensity_* compiled from its
    source (oracle/_ref; Gen A, serial particle loop, as Main/Makefile links
    it), or its FP32 restatement when oracle/_ref is absent ("port");
    assign = "omp": the Gen-B private-grid OpenMP form (NTHREADS-fold count
    fixed) on `threads` threads.  Then the threaded r2c (scipy's pocketfft
    in FP32 standing in for FFTW3, absent here) and the OpenMP P(k) loop as
    written (octant-4 |delta|^2 fixed).  Returns seconds per stage."""
    import scipy.fft
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    orc.set_threads(cores)
    g = orc.Grid.cubic(NMESH, BOX)
    t0 = time.perf_counter()
    if assign == "omp":
        mesh, _ = orc.assign_omp(scheme, x, y, z, w, g, cores)
        t_assign = time.perf_counter() - t0
    elif orc.ref_lib() is not None:
        mesh, t_assign = orc.reference_getdensity(scheme, x, y, z, w, g)
    else:
        mesh, _ = orc.assign_ref(scheme, x, y, z, w, g)
        t_assign = time.perf_counter() - t0
    t1 = time.perf_counter()
    ngal = float(mesh.sum(dtype=np.float64))
    data = mesh - np.float32(ngal / mesh.size)
    spec = scipy.fft.rfftn(data, workers=cores)
    t2 = time.perf_counter()
    vol = BOX ** 3
    orc.power_ref(spec, NMESH, BOX, scheme, NBINS, vol / ngal, ngal * ngal / vol)
    t3 = time.perf_counter()
    orc.set_threads(0)
    return {"assign": t_assign, "fft": t2 - t1, "power": t3 - t2}


def cpu_baseline_block(x, y, z, w):
    """The CPU baseline on this host, one full-size job per scheme (no
    sampling): the reference's Gen-A loops (compiled from its source when
    oracle/_ref is present) with FFT and P(k) on all cores, plus the Gen-B
    OpenMP assignment on all cores and on the reference's 12 threads
    (_NTHREADS_, Headers/def.h:278)."""
    orc = _cpu_oracle()
    cores = os.cpu_count() or 1
    kind = "reference" if orc.ref_lib() is not None else "port"
    per = [cpu_job(orc, s, x, y, z, w) for s in SCHEMES]
    job_s = sum(sum(t.values()) for t in per) / len(SCHEMES)
    omp_all = [cpu_job(orc, s, x, y, z, w, "omp", cores) for s in SCHEMES]
    omp12 = [cpu_job(orc, s, x, y, z, w, "omp", 12) for s in SCHEMES]

    def rate(ts):
        return round(len(ts) / sum(sum(t.values()) for t in ts), 4)
    return {
        "value": round(1.0 / job_s, 4), "unit": "jobs/s", "cores": cores, "kind": kind,
        "sample": "one full-size job per scheme (16,777,216 particles, 256^3, 128 bins): "
                  + ("the reference's getDensity_* compiled from its source (Gen A, serial scatter)"
                     if kind == "reference" else "the oracle's restatement of getDensity_* (Gen A, serial)")
                  + f", scipy pocketfft r2c on {cores} threads standing in for FFTW3, the OpenMP P(k) loop",
        "stage_s_per_job": {k: round(sum(t[k] for t in per) / len(per), 3) for k in per[0]},
        "gen_b_omp_all_cores": {"value": rate(omp_all), "unit": "jobs/s", "threads": cores, "kind": "port",
                                "note": "Gen-B private-grid OpenMP assignment (NTHREADS-fold count fixed)"},
        "gen_b_omp_12_threads": {"value": rate(omp12), "unit": "jobs/s", "threads": 12, "kind": "port",
                                 "note": "the reference's _NTHREADS_ = 12 (Headers/def.h:278); FFT and P(k) "
                                         "on 12 threads too"},
    }


def run_reference(args):
    """The reference's own CPU implementation of the path on this host, on
    the sweep's config: every step is one full-size job (schemes in turn),
    assignment by the reference's getDensity_* compiled from its source (Gen
    A, serial, as its Makefile links it; the FP32 restatement if oracle/_ref
    is absent), r2c on all cores, the OpenMP P(k) loop.  Rank 0 only."""
    rank, local, world = dist_env()
    if rank != 0:
        return None
    from cosmicatlas_b200 import synth
    orc = _cpu_oracle()
    cores = os.cpu_count() or 1
    npart = args.particles
    x, y, z = synth.clumped(npart, BOX, 200_000, 1.5, 0.8, seed=2)
    w = synth.halo_masses(npart, seed=1002)
    for i in range(min(args.warmup, 1)):
        cpu_job(orc, SCHEMES[i % 3], x, y, z, w)
    t_jobs = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        t = cpu_job(orc, SCHEMES[i % 3], x, y, z, w)
        t_jobs.append(sum(t.values()))
    wall = time.perf_counter() - t0
    value = len(t_jobs) / sum(t_jobs)
    kind = "reference" if orc.ref_lib() is not None else "port"
    sample = (f"one full-size job per step, schemes NGP/CIC/TSC in turn ({npart} particles, 256^3, 128 bins); "
              + ("getDensity_* compiled from the reference source (Gen A, serial scatter)" if kind == "reference"
                 else "the oracle's restatement of getDensity_* (Gen A, serial scatter)")
              + f"; scipy pocketfft r2c on {cores} threads standing in for FFTW3; OpenMP P(k) loop")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "jobs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded clumped process, halo-like masses)",
        "config": config_dict(npart, {"parallelism": f"job replicas x{world}"}),
        "cpu_baseline": {"value": round(value, 4), "unit": "jobs/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "jobs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_single(args):
    """One-job latency lines (not the benchmark line): single512 = 512^3 CIC,
    134,217,728 clumped unit-mass particles, L = 1000, P(k) 256 bins, T-web
    R = 2 cells, lambda_th = 0; large768 = 768^3 TSC of a Zel'dovich-displaced
    lattice (452,984,832 particles, L = 1500), P(k) 256 bins of 1.5 k_f,
    T-web R = 3, lambda_th = 0.1."""
    import torch

    from cosmicatlas_b200 import synth
    from cosmicatlas_b200.api import CIC, TSC, Context, make_grid

    torch.cuda.set_device(0)
    prec = 0
    if args.workload == "c1":
        # config 1: 2,000,000 particles (20% uniform, 80% in 20,000 clumps of
        # sigma 2), CIC onto 128^3 FP64, P(k) 64 bins, T-web R = 8, lambda_th 0
        n, box, scheme, nb, ndel, R, lth, prec = 128, 1000.0, CIC, 64, 1.0, 8.0, 0.0, 1
        x, y, z = synth.clumped(2_000_000, box, 20_000, 2.0, 0.8, seed=1)
        arrs = [torch.from_numpy(v).cuda() for v in (x, y, z)]
    elif args.workload == "single512":
        n = args.mesh or 512
        box, scheme, nb, ndel, R, lth = 1000.0, CIC, n // 2, 1.0, 2.0 * 1000.0 / n, 0.0
        x, y, z = synth.clumped(n ** 3, box, max(1, 2_000_000 * n ** 3 // 512 ** 3), 1.5, 0.8, seed=7)
        arrs = [torch.from_numpy(v).cuda() for v in (x, y, z)]
        del x, y, z
    else:
        n, box, scheme, nb, ndel, R, lth = 768, 1500.0, TSC, 256, 1.5, 3.0, 0.1
        gx, gy, gz, _ = synth.zeldovich_lattice(n, box, device="cuda")
        arrs = [gx, gy, gz]
    npart = int(arrs[0].numel())
    grid = make_grid(n, box)
    ctx = Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    pko = Context.pk_opts(scheme, nbins=nb, ndel=ndel)
    from cosmicatlas_b200 import _lib as CL
    two = Context.tweb_opts(R, lth, 1e-5, method=CL.TWEB_FD if args.tweb_method == "fd" else CL.TWEB_FFT)
    for _ in range(args.warmup):
        ctx.job(arrs[0], arrs[1], arrs[2], None, grid, scheme, prec, pk=pko, tweb=two)
    times = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = ctx.job(arrs[0], arrs[1], arrs[2], None, grid, scheme, prec, pk=pko, tweb=two)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    # per-kernel CUDA-event times from a separate pass of the same jobs
    ctx.profile(True)
    ctx.profile_read(reset=True)
    for _ in range(args.steps):
        ctx.job(arrs[0], arrs[1], arrs[2], None, grid, scheme, prec, pk=pko, tweb=two)
    torch.cuda.synchronize()
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    hbm, kind = peaks()
    nh = n * n * (n // 2 + 1)
    stage_bytes = {"assign": npart * 12 + 4 * n ** 3, "fft_r2c": 4 * n ** 3 + 8 * nh, "power": 8 * nh,
                   "tweb": 8 * nh + n ** 3}
    stage_kernels = {
        "assign": ["assign_bin_count", "assign_scan", "assign_partition", "assign_bin_scatter", "assign_deposit",
                   "partial_sum_kernel<double>", "final_sum_kernel", "assign_starts", "tile_sum_kernel",
                   "tile_offsets_kernel", "tile_scan_kernel"],
        "fft_r2c": ["fft_rows_r2c", "fft_cols", "fft_rows_c2c", "fft_cols_pk"],
        "power": ["pk_bin", "pk_final_kernel", "pk_nyq", "pk_final"],
        "tweb": ["tweb_tidal_x", "tweb_tidal_x_nyq", "tweb_tidal_y", "tweb_tidal_y_nyq", "tweb_tidal_z_eigen",
                 "fd_table_kernel"],
    }
    k = args.steps
    side_kernels = {"fft_r2c": ["side.fft_rows_c2c", "side.fft_cols"], "power": ["side.pk_nyq"]}
    if "fft_cols_pk" in prof:
        stage_bytes["power"] = None  # binned inside the r2c's x pass
    stages = {}
    for st, names in stage_kernels.items():
        t = sum(prof.get(nm, (0, 0.0))[1] for nm in names) / k
        stages[st] = {"ms": round(t, 3), "algorithmic_bytes": stage_bytes[st],
                      "achieved_gbs": round(stage_bytes[st] / (t / 1e3) / 1e9, 1) if t > 0 and stage_bytes[st]
                      else None}
        ov = sum(prof.get(nm, (0, 0.0))[1] for nm in side_kernels.get(st, [])) / k
        if ov > 0:
            stages[st]["overlapped_ms"] = round(ov, 3)
    # the T-web's y-pass runs through fft_cols too: attribute by launch counts is not possible
    # from totals, so report the raw kernel table alongside
    out = {"workload": args.workload, "tweb_method": args.tweb_method, "mesh": n, "particles": npart,
           "ms_per_job": round(float(np.median(times)), 3),
           "ms_min": round(min(times), 3), "steps": k, "warmup": args.warmup, "peak_gbs": hbm, "peak_kind": kind,
           "stages": stages, "kernels": {a: {"launches": b[0], "ms_total": round(b[1], 3)} for a, b in sorted(prof.items())},
           "tweb_counts": [int(v) for v in r["tweb"].counts], "n_lost": r["assign"].n_lost,
           "clocks": clk.summary(),
           "timing": "per job: CUDA events around cam_job_run on the launching stream, synchronised on both "
                     "sides; the per-kernel profile runs on the same jobs"}
    for st in stages.values():
        if st["achieved_gbs"]:
            st["frac"] = round(st["achieved_gbs"] / hbm, 4)
    if args.workload == "single512":
        out["stages"]["fft_r2c"]["cufft_ms"] = round(cufft_r2c_ms(n, stream), 4)
        out["stages"]["fft_r2c"]["plain_ms"] = round(ours_r2c_ms(ctx, n), 4)
    ctx.close()
    if args.workload == "c1":
        out["cpu_ref"] = c1_cpu_reference(x, y, z, n, box, scheme, nb, R, lth)
    return out


def run_bam(args):
    """The kernel steps of one BAM calibration iteration at N^3 (default 512):
    the 3D update of GetKernel (rejection form, kernel *= weight per bin,
    N/2 bins) and Konvolve of an FP32 N^3 mesh, all resident on the device.
    Algorithmic bytes: update 8 N^2 (N/2+1) (kernel read and written);
    Konvolve 4 N^3 (in) + 4 N^2 (N/2+1) (kernel) + 4 N^3 (out)."""
    import torch

    from cosmicatlas_b200 import _lib as CL
    from cosmicatlas_b200.api import Context

    torch.cuda.set_device(0)
    n = args.mesh or 512
    box = 1000.0
    nb = n // 2
    gen = torch.Generator(device="cuda").manual_seed(5)
    delta = torch.randn((n, n, n), device="cuda", generator=gen)
    kern = torch.ones((n, n, n // 2 + 1), device="cuda")
    out = torch.empty_like(delta)
    w = np.random.default_rng(5).uniform(0.99, 1.01, nb)
    ctx = Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    for _ in range(args.warmup):
        ctx.bam_kernel_update(kern, box, w, CL.KERNEL_SCALE)
        ctx.konvolve(delta, box, kern, out=out)
    ctx.profile(True)
    ctx.profile_read(reset=True)
    tu, tk = [], []
    for _ in range(args.steps):
        for dst, fn in ((tu, lambda: ctx.bam_kernel_update(kern, box, w, CL.KERNEL_SCALE)),
                        (tk, lambda: ctx.konvolve(delta, box, kern, out=out))):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            dst.append(e0.elapsed_time(e1))
    prof = ctx.profile_read(reset=True)
    ctx.close()
    hbm, kind = peaks()
    nh = n * n * (n // 2 + 1)
    bu, bk = 8 * nh, 8 * n ** 3 + 4 * nh
    mu, mk = float(np.median(tu)), float(np.median(tk))
    return {"workload": "bam", "mesh": n, "nbins": nb,
            "kernel_update": {"ms": round(mu, 3), "algorithmic_bytes": bu, "achieved_gbs": round(bu / mu / 1e6, 1),
                              "frac": round(bu / mu / 1e6 / hbm, 4)},
            "konvolve": {"ms": round(mk, 3), "algorithmic_bytes": bk, "achieved_gbs": round(bk / mk / 1e6, 1),
                         "frac": round(bk / mk / 1e6 / hbm, 4)},
            "peak_gbs": hbm, "peak_kind": kind, "steps": args.steps, "warmup": args.warmup,
            "note": "host round trip included: each call reads its bin sums back",
            "kernels": {a: {"launches": b[0], "ms_total": round(b[1], 3)} for a, b in sorted(prof.items())}}


def c1_cpu_reference(x, y, z, n, box, scheme, nbins, R, lth):
    """Config 1 through the oracle port of the reference path on the host:
    the serial FP32 scatter as written, scipy rfftn on all cores (standing in
    for threaded FFTW), the OpenMP P(k) loop, and the T-web (FFT tidal
    tensor, per-cell eigenvalues)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import scipy.fft
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    g = orc.Grid.cubic(n, box)
    t0 = time.perf_counter()
    mesh, _ = orc.assign_ref(scheme, x, y, z, None, g)
    t1 = time.perf_counter()
    ngal = float(mesh.sum(dtype=np.float64))
    spec = scipy.fft.rfftn(mesh.astype(np.float64) - ngal / mesh.size, workers=cores)
    orc.power_ref(spec, n, box, scheme, nbins, box ** 3 / ngal, ngal * ngal / box ** 3)
    t2 = time.perf_counter()
    orc.tweb_density(mesh.astype(np.float64), box, R, lth)
    t3 = time.perf_counter()
    return {"ms_per_job": round(1e3 * (t3 - t0), 1), "assign_ms": round(1e3 * (t1 - t0), 1),
            "fft_pk_ms": round(1e3 * (t2 - t1), 1), "tweb_ms": round(1e3 * (t3 - t2), 1), "cores": cores,
            "kind": "port"}


# ------------------------------------------------------------------ serving
def _latency(v):
    v = np.sort(np.asarray(v, np.float64))
    return {"p50": round(float(np.percentile(v, 50)), 3), "p99": round(float(np.percentile(v, 99)), 3),
            "mean": round(float(v.mean()), 3), "max": round(float(v.max()), 3)}


def calib_jobs(njobs):
    """The calibration batch: njobs independent seeds, 262,144 clumped
    particles each (clump fraction U[0.5, 0.9], sigma U[1, 4], 2,000
    clumps), L = 500, CIC onto 64^3 FP32, P(k) in 32 bins, T-web label
    counts with R = 8, lambda_th = 0.  Particles are drawn on the GPU."""
    from cosmicatlas_b200 import synth
    from cosmicatlas_b200.api import CIC, Context, JobSpec, make_grid
    grid = make_grid(64, 500.0)
    pk = Context.pk_opts(CIC, nbins=32)
    tw = Context.tweb_opts(8.0, 0.0, 1e-5)
    parts = []
    for j in range(njobs):
        rng = np.random.default_rng(5 + j)
        frac, sig = rng.uniform(0.5, 0.9), rng.uniform(1.0, 4.0)
        parts.append(synth.clumped_torch(262_144, 500.0, 2_000, sig, frac, seed=100_000 + j))

    def specs():
        return [JobSpec(x, y, z, None, grid=grid, scheme=CIC, precision=0, pk=pk, tweb=tw) for x, y, z in parts]
    return parts, grid, pk, tw, specs


def _events_ms(fn, stream):
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def run_calib(args):
    """Served vs plain per-call throughput on the calibration batch."""
    import torch

    from cosmicatlas_b200.api import CIC, Context, Server
    torch.cuda.set_device(0)
    njobs = args.jobs or 4096
    parts, grid, pk, tw, specs = calib_jobs(njobs)
    stream = torch.cuda.current_stream()
    ctx = Context(0)
    ctx.set_stream(stream.cuda_stream)

    # plain per-call path: one cam_job_run per job
    def plain(k):
        lat = []
        for x, y, z in parts[:k]:
            t0 = time.perf_counter()
            ctx.job(x, y, z, None, grid, CIC, 0, pk=pk, tweb=tw)
            lat.append(1e3 * (time.perf_counter() - t0))
        return lat
    plain(min(njobs, 64))
    ms_plain, lat_plain = _events_ms(lambda: plain(njobs), stream)

    # graph-packed batches through cam_batch_run
    ctx.batch(specs()[:64])
    sp = specs()
    ms_batch, _ = _events_ms(lambda: ctx.batch(sp), stream)

    # the continuous-batching server: every job submitted at t = 0
    with Server(0, workers=4, max_batch=32) as srv:
        warm = specs()[:256]
        for i in [srv.submit(s) for s in warm]:
            srv.wait(i)
        srv.stats(reset=True)
        sp = specs()

        def serve():
            ids = [srv.submit(s) for s in sp]
            for i in ids:
                srv.wait(i)
        with ClockSampler(0) as clk:
            ms_srv, _ = _events_ms(serve, stream)
        st = srv.stats()
    ctx.close()
    return {
        "workload": f"calibration batch: {njobs} jobs x 262,144 clumped particles, L=500, CIC 64^3 FP32, "
                    "P(k) 32 bins, T-web counts R=8",
        "metric": "mesh-jobs/s", "unit": "jobs/s",
        "plain": {"value": round(njobs / (ms_plain / 1e3), 1), "latency_ms": _latency(lat_plain),
                  "path": "cam_job_run per job, one context"},
        "batch": {"value": round(njobs / (ms_batch / 1e3), 1), "path": "cam_batch_run, 32 jobs per graph"},
        "served": {"value": round(njobs / (ms_srv / 1e3), 1), "path": "cam_server: 4 workers, batches of 32",
                   "latency_ms": {"p50": round(st["p50_ms"], 3), "p99": round(st["p99_ms"], 3),
                                  "note": "submit -> result with all jobs submitted at t = 0"},
                   "batches": st["batches"], "graph_replays": st["graph_replays"]},
        "speedup_served_vs_plain": round(ms_plain / ms_srv, 2),
        "speedup_batch_vs_plain": round(ms_plain / ms_batch, 2),
        "clocks": clk.summary(),
    }


def run_calib_pk(args):
    """The calibration batch without the T-web (4,096 jobs: 64^3 CIC FP32,
    262,144 clumped particles each, L = 500, P(k) in 32 bins), through the
    per-call path, graph-packed batches, the job server and the persistent
    on-device request loop (one CTA per job, no launch per job)."""
    import torch

    from cosmicatlas_b200 import synth
    from cosmicatlas_b200.api import CIC, Context, DeviceLoop, JobSpec, Server, make_grid
    torch.cuda.set_device(0)
    njobs = args.jobs or 4096
    grid = make_grid(64, 500.0)
    pk = Context.pk_opts(CIC, nbins=32)
    parts = []
    for j in range(njobs):
        rng = np.random.default_rng(5 + j)
        frac, sig = rng.uniform(0.5, 0.9), rng.uniform(1.0, 4.0)
        parts.append(synth.clumped_torch(262_144, 500.0, 2_000, sig, frac, seed=100_000 + j))
    torch.cuda.synchronize()

    def specs():
        return [JobSpec(x, y, z, None, grid=grid, scheme=CIC, precision=0, pk=pk) for x, y, z in parts]
    stream = torch.cuda.current_stream()
    ctx = Context(0)
    ctx.set_stream(stream.cuda_stream)

    def plain():
        lat = []
        for x, y, z in parts:
            t0 = time.perf_counter()
            ctx.job(x, y, z, None, grid, CIC, 0, pk=pk)
            lat.append(1e3 * (time.perf_counter() - t0))
        return lat
    for x, y, z in parts[:64]:
        ctx.job(x, y, z, None, grid, CIC, 0, pk=pk)
    ms_plain, lat_plain = _events_ms(plain, stream)
    ctx.batch(specs()[:64])
    sp = specs()
    ms_batch, _ = _events_ms(lambda: ctx.batch(sp), stream)
    ctx.close()
    with Server(0, workers=4, max_batch=32) as srv:
        for i in [srv.submit(s) for s in specs()[:256]]:
            srv.wait(i)
        srv.stats(reset=True)
        sp = specs()

        def serve():
            for i in [srv.submit(s) for s in sp]:
                srv.wait(i)
        ms_srv, _ = _events_ms(serve, stream)
        st = srv.stats()
    with DeviceLoop(0, max_particles=262_144, nslots=njobs, idle_timeout_s=10.0) as lp:
        for i in [lp.submit(s) for s in specs()[:256]]:
            lp.wait(i)
        sp = specs()
        lat_dl = []

        def devloop():
            t_sub = {}
            ids = []
            for s in sp:
                t_sub[len(ids)] = time.perf_counter()
                ids.append(lp.submit(s))
            for k, i in enumerate(ids):
                lp.wait(i)
                lat_dl.append(1e3 * (time.perf_counter() - t_sub[k]))
        with ClockSampler(0) as clk:
            ms_dl, _ = _events_ms(devloop, stream)
    return {
        "workload": f"calibration batch without the T-web: {njobs} jobs x 262,144 clumped particles, L=500, "
                    "CIC 64^3 FP32, P(k) 32 bins",
        "metric": "mesh-jobs/s", "unit": "jobs/s",
        "plain": {"value": round(njobs / (ms_plain / 1e3), 1), "latency_ms": _latency(lat_plain),
                  "path": "cam_job_run per job, one context"},
        "batch": {"value": round(njobs / (ms_batch / 1e3), 1), "path": "cam_batch_run, 32 jobs per graph"},
        "served": {"value": round(njobs / (ms_srv / 1e3), 1), "path": "cam_server: 4 workers, batches of 32",
                   "latency_ms": {"p50": round(st["p50_ms"], 3), "p99": round(st["p99_ms"], 3)}},
        "device_loop": {"value": round(njobs / (ms_dl / 1e3), 1),
                        "path": "cam_devloop: one resident kernel, one CTA per job, queue in mapped host memory",
                        "latency_ms": _latency(lat_dl),
                        "latency_note": "submit -> result with all jobs submitted at t = 0 (queueing included)"},
        "speedup_device_loop_vs_plain": round(ms_plain / ms_dl, 2),
        "speedup_served_vs_plain": round(ms_plain / ms_srv, 2),
        "clocks": clk.summary(),
    }


def stream_jobs(njobs, seed=4):
    """The served mixed stream: N from {64..512} (weights .30/.25/.15/.15/.10
    /.05), N_p log-uniform [1e5, 5e7], L log-uniform [250, 2000], scheme
    uniform, half the jobs want the T-web (R = 2 cells, lambda_th = 0);
    P(k) in N/2 bins of width k_f."""
    rng = np.random.default_rng(seed)
    ns = rng.choice([64, 128, 192, 256, 384, 512], size=njobs, p=[0.30, 0.25, 0.15, 0.15, 0.10, 0.05])
    nps = np.exp(rng.uniform(np.log(1e5), np.log(5e7), size=njobs)).astype(np.int64)
    boxes = np.exp(rng.uniform(np.log(250.0), np.log(2000.0), size=njobs))
    schemes = rng.integers(0, 3, size=njobs)
    tweb = rng.uniform(size=njobs) < 0.5
    return [dict(n=int(a), np=int(b), box=float(c), scheme=int(d), tweb=bool(e))
            for a, b, c, d, e in zip(ns, nps, boxes, schemes, tweb)]


def run_stream(args):
    """Served vs plain per-call path on the mixed stream, open-loop Poisson
    arrivals at each rate plus a closed-loop saturation pass.  Particles
    come from four shuffled 5e7-particle pools of the clumped process in the
    unit box (200,000 clumps, sigma = 1.5e-3), scaled by each job's L on the
    GPU just before submission."""
    import torch

    from cosmicatlas_b200 import synth
    from cosmicatlas_b200.api import Context, JobSpec, Server, make_grid
    torch.cuda.set_device(0)
    njobs = args.jobs or 2000
    jobs = stream_jobs(njobs)
    pools = []
    for p in range(4):
        x, y, z = synth.clumped_torch(50_000_000, 1.0, 200_000, 1.5e-3, 0.8, seed=40 + p)
        perm = torch.randperm(x.numel(), device="cuda", generator=torch.Generator("cuda").manual_seed(p))
        pools.append(torch.stack([x[perm], y[perm], z[perm]]))
        del x, y, z, perm
    prep = torch.cuda.Stream()
    budget = 150 << 30

    def make(j, i):
        with torch.cuda.stream(prep):
            xyz = pools[i % 4][:, :j["np"]] * j["box"]
            xyz = torch.where(xyz >= j["box"], torch.zeros_like(xyz), xyz)
        prep.synchronize()
        n = j["n"]
        return JobSpec(xyz[0], xyz[1], xyz[2], None, grid=make_grid(n, j["box"]), scheme=j["scheme"], precision=0,
                       pk=Context.pk_opts(j["scheme"], nbins=n // 2),
                       tweb=Context.tweb_opts(2.0 * j["box"] / n, 0.0, 1e-5) if j["tweb"] else None)

    from cosmicatlas_b200.api import alloc_stats

    def one_pass(workers, max_batch, rate, held_gb=None):
        held_gb = args.held_gb if held_gb is None else held_gb
        rng = np.random.default_rng(99)
        gaps = rng.exponential(1.0 / rate, size=njobs) if rate else np.zeros(njobs)
        with Server(0, hbm_budget=budget, workers=workers, max_batch=max_batch) as srv:
            # warm-up: the first 100 jobs of the stream, all at once, so the
            # contexts' buffers and plans are sized as a running server's are
            for i in [srv.submit(make(j, k)) for k, j in enumerate(jobs[:100])]:
                srv.wait(i)
            srv.stats(reset=True)
            srv.trace()
            alloc_stats(reset=True)
            retries0 = torch.cuda.memory_stats().get("num_alloc_retries", 0)
            pending = []  # (id, bytes): inputs the client holds until done
            held = 0.0
            t_start = time.perf_counter()
            t_next = t_start
            for k, j in enumerate(jobs):
                t_next += gaps[k]
                now = time.perf_counter()
                if t_next > now:
                    time.sleep(t_next - now)
                while pending and held > held_gb * 1e9:  # client back-pressure
                    jid, b = pending.pop(0)
                    srv.wait(jid)
                    held -= b
                jid = srv.submit(make(j, k))
                pending.append((jid, 12.0 * j["np"]))
                held += 12.0 * j["np"]
            for jid, _ in pending:
                srv.wait(jid)
            wall = time.perf_counter() - t_start
            st = srv.stats()
            tr = srv.trace()
            al = alloc_stats()
            torch_retries = torch.cuda.memory_stats().get("num_alloc_retries", 0) - retries0
        tr = tr[-njobs:]
        wait = tr["start_ms"] - tr["submit_ms"]
        run = tr["end_ms"] - tr["start_ms"]
        big = tr["big"] == 1
        free_gb = torch.cuda.mem_get_info()[0] / 1e9

        def pct(v):
            return [round(float(np.percentile(v, q)), 2) for q in (50, 99)] if len(v) else None
        return {"jobs_per_s": round(njobs / wall, 1), "p50_ms": round(st["p50_ms"], 2),
                "p99_ms": round(st["p99_ms"], 2), "batches": st["batches"], "batched_jobs": st["batched_jobs"],
                "graph_replays": st["graph_replays"], "peak_reserved_gb": round(st["peak_bytes_reserved"] / 1e9, 1),
                "trace": {"queue_wait_p50_p99": pct(wait), "run_big_p50_p99": pct(run[big]),
                          "run_small_p50_p99": pct(run[~big]), "big_jobs": int(big.sum()),
                          "worker_busy_s": round(float(np.sum(np.unique(np.stack([tr["worker"], tr["start_ms"],
                                                                                  tr["end_ms"]], 1), axis=0)[:, 2]
                                                             - np.unique(np.stack([tr["worker"], tr["start_ms"],
                                                                                   tr["end_ms"]], 1), axis=0)[:, 1])
                                                  / 1e3), 2),
                          "device_free_gb_after": round(free_gb, 1),
                          "slowest_ms": round(float(np.max(run)), 2) if len(run) else None},
                "allocations": {"library": al, "torch_alloc_retries": int(torch_retries), "held_gb": held_gb}}

    rates = [float(r) for r in args.rates.split(",") if r]
    out = {"workload": f"served mixed stream: {njobs} jobs, N in 64..512, N_p log-uniform [1e5, 5e7], "
                       "L log-uniform [250, 2000], NGP/CIC/TSC, half with T-web; HBM budget 150 GB",
           "metric": "mesh-jobs/s", "unit": "jobs/s", "rates": {}}
    with ClockSampler(0, period_s=0.05) as clk:  # minutes long: 20 samples/s
        out["saturation"] = {"served": one_pass(4, 16, 0), "plain": one_pass(1, 1, 0)}
        for r in rates:
            out["rates"][str(r)] = {"served": one_pass(4, 16, r), "plain": one_pass(1, 1, r)}
    s, p = out["saturation"]["served"], out["saturation"]["plain"]
    out["speedup_served_vs_plain"] = round(s["jobs_per_s"] / p["jobs_per_s"], 2)
    out["clocks"] = clk.summary()
    return out


def main():
    args = parse()
    if args.workload in ("calib", "calib_pk", "stream"):
        fn = {"calib": run_calib, "calib_pk": run_calib_pk, "stream": run_stream}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return
    if args.workload == "bam":
        print(json.dumps(run_bam(args)), flush=True)
        return
    if args.workload != "sweep":
        print(json.dumps(run_single(args)), flush=True)
        return
    if args.impl == "reference":
        out = run_reference(args)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    out, parts = run_ours(args)
    if out is None:
        return
    rank, local, world = dist_env()
    if world == 1 and not args.kernels_only:
        out["cpu_baseline"] = cpu_baseline_block(*parts)
        if args.serving_jobs > 0:
            # the metric's "vs plain path" part: the same jobs through the
            # per-call path and through the serving loop, on this GPU
            args.jobs = args.serving_jobs
            out["serving"] = run_calib(args)
        if args.serving_jobs > 0:
            # the same batch without the T-web, beside the on-device loop
            args.jobs = args.serving_jobs
            out["serving_pk"] = run_calib_pk(args)
        if args.stream_jobs > 0:
            # the mixed stream (2,000 jobs, N 64..512): saturation and a
            # Poisson arrival rate, served against the per-call path
            args.jobs = args.stream_jobs
            args.rates = args.stream_rates
            out["serving_stream"] = run_stream(args)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
