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
        copies of the P(k) results are inside the timed region.
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
    ap.add_argument("--workload", default="sweep", choices=["sweep", "single512", "large768"],
                    help="sweep: the benchmark line (default); single512 / large768: one-job latency lines")
    ap.add_argument("--mesh", type=int, default=0, help="single512 only: override N (profiler runs)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


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
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, nme in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(nme)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


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
    x, y, z = synth.clumped(npart, BOX, 200_000, 1.5, 0.8, seed=2 + 1000 * rank)
    w = synth.halo_masses(npart, seed=1002 + 1000 * rank)
    dev = [torch.from_numpy(v).cuda() for v in (x, y, z, w)]
    pinned = [torch.from_numpy(v).pin_memory() for v in (x, y, z, w)]
    grid = make_grid(NMESH, BOX)
    ctx = Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    opts = {s: Context.pk_opts(s, nbins=NBINS) for s in SCHEMES}

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
        return r

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(arrs, k, lat=None):
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(k):
            step(arrs, lat)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        barrier()
        return ms

    for _ in range(args.warmup):
        step(dev)
        if not args.kernels_only:
            step(pinned)
    # device-resident inputs: the headline `value`
    lat = []
    launches0 = ctx.kernel_launches
    ctx.profile(True)
    ctx.profile_read(reset=True)
    with ClockSampler(local) as clk:
        ms = timed(dev, args.steps, lat)
    prof = ctx.profile_read(reset=True)
    ctx.profile(False)
    launches = ctx.kernel_launches - launches0
    job_ms = sorted(a.elapsed_time(b) for a, b in lat)
    # end to end: pinned host particles in, P(k) out
    ms_e2e = timed(pinned, args.steps) if not args.kernels_only else float("nan")

    jobs = len(SCHEMES) * args.steps * world
    value = jobs / (ms / 1e3)
    e2e = jobs / (ms_e2e / 1e3)
    h2d = npart * 16
    d2h = len(SCHEMES) * NBINS * 24

    out = None
    if rank == 0:
        hbm, peak_kind = peaks()
        jobs_rank = len(SCHEMES) * args.steps
        # stage roofline: algorithmic bytes per job (unit = one mesh job)
        nh = NMESH * NMESH * (NMESH // 2 + 1)
        stage_bytes = {
            "assign": npart * (12 + 4) + 4 * NMESH ** 3,
            "fft_r2c": 4 * NMESH ** 3 + 8 * nh,
            "power": 8 * nh,
        }
        stage_kernels = {
            "assign": ["assign_bin_count", "assign_scan", "assign_bin_scatter", "assign_deposit",
                       "partial_sum_kernel<double>", "final_sum_kernel"],
            "fft_r2c": ["fft_rows_r2c", "fft_cols", "fft_rows_c2c"],
            "power": ["pk_bin", "pk_final_kernel"],
        }
        stages = {}
        for st, names in stage_kernels.items():
            t = sum(prof.get(nm, (0, 0.0))[1] for nm in names) / jobs_rank
            ach = stage_bytes[st] / (t / 1e3) / 1e9 if t > 0 else 0.0
            stages[st] = {"ms_per_job": round(t, 4), "algorithmic_bytes": stage_bytes[st],
                          "achieved_gbs": round(ach, 1), "frac": round(ach / hbm, 4)}
        dom = max(stages, key=lambda s: stages[s]["ms_per_job"])
        traffic = ncu_traffic()
        dom_traffic = traffic.get(dom) if isinstance(traffic, dict) else None
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
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "stage": dom, "achieved": stages[dom]["achieved_gbs"],
                         "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": stages[dom]["frac"], "traffic": dom_traffic},
            "stages": stages,
            "kernels": kernels,
            "clocks": clk.summary(),
        }
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out, (x, y, z, w)


def cpu_baseline_sample(x, y, z, w, nsample, cores):
    """The reference path as written on the host (oracle port): serial FP32
    scatter, threaded FP32 r2c (scipy pocketfft), the OpenMP P(k) loop."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import scipy.fft

    g = orc.Grid.cubic(NMESH, BOX)
    t_assign = 0.0
    t_rest = 0.0
    for s in SCHEMES:
        t0 = time.perf_counter()
        mesh, _ = orc.assign_ref(s, x[:nsample], y[:nsample], z[:nsample], w[:nsample], g)
        t_assign += time.perf_counter() - t0
        t0 = time.perf_counter()
        ngal = float(mesh.sum(dtype=np.float64))
        data = mesh - np.float32(ngal / mesh.size)
        spec = scipy.fft.rfftn(data, workers=cores)
        vol = BOX ** 3
        orc.power_ref(spec, NMESH, BOX, s, NBINS, vol / ngal, ngal * ngal / vol)
        t_rest += time.perf_counter() - t0
    scale = x.size / nsample
    per_job = (t_assign * scale + t_rest) / len(SCHEMES)
    return 1.0 / per_job, per_job


def run_reference(args):
    rank, local, world = dist_env()
    if rank != 0:
        return None
    from cosmicatlas_b200 import synth
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    npart = args.particles
    x, y, z = synth.clumped(npart, BOX, 200_000, 1.5, 0.8, seed=2)
    w = synth.halo_masses(npart, seed=1002)
    nsample = min(npart, 1 << 20)
    for _ in range(min(args.warmup, 1)):
        cpu_baseline_sample(x, y, z, w, nsample, cores)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, _ = cpu_baseline_sample(x, y, z, w, nsample, cores)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = float(np.median(vals))
    sample = (f"{nsample} of {npart} particles per scheme (serial scatter time scaled by {npart / nsample:g}), "
              f"full 256^3 FFT and P(k)")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "jobs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded clumped process, halo-like masses)", "config": config_dict(npart),
        "cpu_baseline": {"value": round(value, 4), "unit": "jobs/s", "cores": cores, "kind": "port",
                         "sample": sample},
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
    if args.workload == "single512":
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
    two = Context.tweb_opts(R, lth, 1e-5)
    for _ in range(args.warmup):
        ctx.job(arrs[0], arrs[1], arrs[2], None, grid, scheme, 0, pk=pko, tweb=two)
    ctx.profile(True)
    ctx.profile_read(reset=True)
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = ctx.job(arrs[0], arrs[1], arrs[2], None, grid, scheme, 0, pk=pko, tweb=two)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    prof = ctx.profile_read(reset=True)
    hbm, kind = peaks()
    nh = n * n * (n // 2 + 1)
    stage_bytes = {"assign": npart * 12 + 4 * n ** 3, "fft_r2c": 4 * n ** 3 + 8 * nh, "power": 8 * nh,
                   "tweb": 8 * nh + n ** 3}
    stage_kernels = {
        "assign": ["assign_bin_count", "assign_scan", "assign_bin_scatter", "assign_deposit",
                   "partial_sum_kernel<double>", "final_sum_kernel", "assign_starts", "tile_sum_kernel",
                   "tile_offsets_kernel", "tile_scan_kernel"],
        "fft_r2c": ["fft_rows_r2c", "fft_cols", "fft_rows_c2c"],
        "power": ["pk_bin", "pk_final_kernel"],
        "tweb": ["tweb_tidal_x", "tweb_tidal_x_nyq", "tweb_tidal_z_eigen"],
    }
    k = args.steps
    stages = {}
    for st, names in stage_kernels.items():
        t = sum(prof.get(nm, (0, 0.0))[1] for nm in names) / k
        stages[st] = {"ms": round(t, 3), "algorithmic_bytes": stage_bytes[st],
                      "achieved_gbs": round(stage_bytes[st] / (t / 1e3) / 1e9, 1) if t > 0 else None}
    # the T-web's y-pass runs through fft_cols too: attribute by launch counts is not possible
    # from totals, so report the raw kernel table alongside
    out = {"workload": args.workload, "mesh": n, "particles": npart, "ms_per_job": round(float(np.median(times)), 3),
           "ms_min": round(min(times), 3), "steps": k, "warmup": args.warmup, "peak_gbs": hbm, "peak_kind": kind,
           "stages": stages, "kernels": {a: {"launches": b[0], "ms_total": round(b[1], 3)} for a, b in sorted(prof.items())},
           "tweb_counts": [int(v) for v in r["tweb"].counts], "n_lost": r["assign"].n_lost}
    ctx.close()
    return out


def main():
    args = parse()
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
        cores = os.cpu_count() or 1
        nsample = min(args.particles, 1 << 20)
        v, per_job = cpu_baseline_sample(*parts, nsample, cores)
        out["cpu_baseline"] = {"value": round(v, 4), "unit": "jobs/s", "cores": cores, "kind": "port",
                               "sample": f"{nsample} of {args.particles} particles per scheme (serial scatter "
                                         f"scaled by {args.particles / nsample:g}), full 256^3 FFT and P(k), "
                                         f"FFT on {cores} threads"}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
