"""GPU serving: graph-packed batches (cam_batch_run) and the continuous-
batching server (cam_server_*) return for every job exactly what the plain
per-call path (cam_job_run) returns for it alone -- bit for bit: the same
deterministic kernels run on per-slot buffers -- and the plain path is
itself checked against the FP64 oracle (P(k) within 1e-5 relative).
"""
import ctypes

import numpy as np
import pytest

import oracle as orc
from conftest import pk_rel_err
from cosmicatlas_b200 import _lib as L
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, F64, NGP, TSC, CamError, Context, JobSpec, Server, make_grid

pytestmark = pytest.mark.gpu

BAND = 1e-5


def make_job(seed, n=64, box=500.0, npart=100_000, scheme=CIC, prec=F32, weights=False, tweb=True, nbins=32,
             labels=False, R=8.0):
    x, y, z = synth.clumped(npart, box, 1_000, 2.0, 0.7, seed=seed)
    w = synth.halo_masses(npart, seed=seed + 1) if weights else None
    return dict(x=x, y=y, z=z, w=w, grid=make_grid(n, box), scheme=scheme, precision=prec,
                pk=Context.pk_opts(scheme, nbins=nbins), tweb=Context.tweb_opts(R, 0.0, BAND) if tweb else None,
                want_labels=labels)


def spec(j):
    return JobSpec(j["x"], j["y"], j["z"], j["w"], grid=j["grid"], scheme=j["scheme"], precision=j["precision"],
                   pk=j["pk"], tweb=j["tweb"], want_labels=j["want_labels"])


def plain(ctx, j):
    return ctx.job(j["x"], j["y"], j["z"], j["w"], j["grid"], j["scheme"], j["precision"], pk=j["pk"],
                   tweb=j["tweb"], want_labels=j["want_labels"])


def assert_same(a, b):
    assert a["assign"].n_in == b["assign"].n_in and a["assign"].n_lost == b["assign"].n_lost
    assert a["assign"].sum_mesh == b["assign"].sum_mesh
    assert np.array_equal(a["pk"].pk, b["pk"].pk, equal_nan=True)
    assert np.array_equal(a["pk"].modes, b["pk"].modes)
    assert np.array_equal(a["pk"].kvector, b["pk"].kvector)
    assert a["pk"].shot_noise == b["pk"].shot_noise
    if a["tweb"] is not None:
        assert np.array_equal(a["tweb"].counts, b["tweb"].counts)
        assert a["tweb"].ties == b["tweb"].ties and a["tweb"].mean == b["tweb"].mean
        if a["tweb"].labels is not None and b["tweb"].labels is not None:
            assert np.array_equal(a["tweb"].labels, b["tweb"].labels)


def test_batch_equals_plain_and_replays(ctx):
    # 34 jobs of one shape (a full batch of 32 + 2), 5 of a second shape
    # (weighted TSC, 48^3), 3 more of the first: three batch keys, each
    # captured after its first run; the second call replays the graphs.
    jobs = [make_job(100 + i) for i in range(34)]
    jobs += [make_job(200 + i, n=48, box=300.0, scheme=TSC, weights=True, nbins=24) for i in range(5)]
    jobs += [make_job(300 + i) for i in range(3)]
    want = [plain(ctx, j) for j in jobs]
    for rep in range(3):
        got = ctx.batch([spec(j) for j in jobs])
        for g, w in zip(got, want):
            assert_same(g, w)


def test_batch_job_vs_oracle(ctx):
    j = make_job(7, npart=200_000)
    got = ctx.batch([spec(j), spec(make_job(8, npart=200_000))])[0]
    mesh, lost = orc.assign_f64(CIC, j["x"], j["y"], j["z"], None, orc.Grid.cubic(64, 500.0))
    pk = orc.power_grid(mesh.astype(np.float32).astype(np.float64), 500.0, CIC, 32)
    floor = pk.shot_noise * pk.sum_sn / np.maximum(pk.modes, 1)
    assert got["assign"].n_lost == lost
    assert np.array_equal(got["pk"].modes, pk.modes)
    assert pk_rel_err(got["pk"].pk, pk.pk, floor) <= 1e-5
    tw = orc.tweb_density(mesh.astype(np.float32).astype(np.float64), 500.0, 8.0, 0.0, BAND)
    # label counts: equal except for cells within the tie band of lambda_th
    diff = got["tweb"].counts - np.bincount(tw.labels.ravel(), minlength=5)[1:]
    assert np.abs(diff).sum() <= 2 * tw.ties


def test_batch_nonfinite_weight_fails_only_that_job(ctx):
    jobs = [make_job(400 + i, weights=True, tweb=False) for i in range(4)]
    jobs[2]["w"] = jobs[2]["w"].copy()
    jobs[2]["w"][17] = np.nan
    specs = [spec(j) for j in jobs]
    with pytest.raises(CamError) as e:
        ctx.batch(specs)
    assert e.value.code == L.CAM_E_NONFINITE
    for i in (0, 1, 3):
        assert_same(specs[i].result(), plain(ctx, jobs[i]))


def test_batch_rejects_labels(ctx):
    with pytest.raises(CamError):
        ctx.batch([spec(make_job(1, labels=True)), spec(make_job(2, labels=True))])


def mixed_stream(seed, count):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        box = float(rng.uniform(250.0, 1000.0))
        scheme = int(rng.integers(0, 3))
        jobs.append(make_job(1000 + i, n=n, box=box, npart=int(rng.integers(20_000, 300_000)), scheme=scheme,
                             prec=F64 if i % 7 == 3 else F32, weights=bool(i % 3 == 0), tweb=bool(i % 2 == 0),
                             labels=bool(i % 5 == 0), nbins=int(n // 4), R=2.0 * box / n))
    # a run of same-shaped small jobs that the server packs into batches
    jobs += [make_job(2000 + i, npart=50_000) for i in range(24)]
    return jobs


def test_server_mix_equals_alone(ctx):
    jobs = mixed_stream(11, 36)
    alone = [plain(ctx, j) for j in jobs]
    with Server(0, workers=4, max_batch=8) as srv:
        specs = [spec(j) for j in jobs]
        ids = [srv.submit(s) for s in specs]
        got = [srv.wait(i, timeout_s=300) for i in ids]
        st = srv.stats()
    for g, a in zip(got, alone):
        assert_same(g, a)
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert st["peak_bytes_reserved"] <= st["budget"]


def test_server_replays_graphs_for_packed_jobs(ctx):
    jobs = [make_job(3000 + i, npart=50_000) for i in range(40)]
    alone = [plain(ctx, j) for j in jobs]
    with Server(0, workers=1, max_batch=8) as srv:
        ids = [srv.submit(spec(j)) for j in jobs]
        got = [srv.wait(i, timeout_s=300) for i in ids]
        st = srv.stats()
        tr = srv.trace()
    for g, a in zip(got, alone):
        assert_same(g, a)
    assert st["batches"] >= 3 and st["graph_replays"] >= 1, st
    # per-job trace: every job once, times ordered, batch sizes add up
    assert sorted(tr["id"].tolist()) == sorted(ids)
    assert np.all(tr["start_ms"] >= tr["submit_ms"]) and np.all(tr["end_ms"] >= tr["start_ms"])
    assert np.all(tr["status"] == 0) and np.all(tr["worker"] == 0)
    assert int((tr["batch"] > 1).sum()) == st["batched_jobs"]


def test_server_budget_admission(ctx):
    # A budget that holds one of these jobs at a time: the workers take
    # turns, dropping their cached buffers when the next job would not fit.
    jobs = [make_job(4000 + i, npart=100_000) for i in range(6)]
    alone = [plain(ctx, j) for j in jobs]
    budget = 100 << 20
    with Server(0, hbm_budget=budget, workers=3, max_batch=1) as srv:
        ids = [srv.submit(spec(j)) for j in jobs]
        got = [srv.wait(i, timeout_s=300) for i in ids]
        st = srv.stats()
        big = make_job(5000, n=256, box=1000.0, npart=2_000_000, tweb=False)
        with pytest.raises(CamError) as e:
            srv.submit(spec(big))
        assert e.value.code == L.CAM_E_NOMEM
    for g, a in zip(got, alone):
        assert_same(g, a)
    assert st["peak_bytes_reserved"] <= budget


def test_server_failed_job_and_poll(ctx):
    jobs = [make_job(6000 + i, weights=True, tweb=False) for i in range(3)]
    jobs[1]["w"] = jobs[1]["w"].copy()
    jobs[1]["w"][5] = np.inf
    with Server(0, workers=2, max_batch=4) as srv:
        specs = [spec(j) for j in jobs]
        ids = [srv.submit(s) for s in specs]
        with pytest.raises(CamError) as e:
            srv.wait(ids[1], timeout_s=300)
        assert e.value.code == L.CAM_E_NONFINITE
        for i in (0, 2):
            assert_same(srv.wait(ids[i], timeout_s=300), plain(ctx, jobs[i]))
        lib = L.lib()
        assert lib.cam_server_poll(srv.h, ids[0]) == L.CAM_E_NOTFOUND  # status already collected
        assert lib.cam_server_poll(srv.h, 10_000) == L.CAM_E_NOTFOUND
        bad = make_job(1)
        bad["grid"] = make_grid((64, 64, 32), 500.0)
        with pytest.raises(CamError):
            srv.submit(spec(bad))
        st = srv.stats(reset=True)
        assert st["failed"] == 1
        assert srv.stats()["completed"] == 0
