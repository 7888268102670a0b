"""GPU mass assignment vs the oracle (through the C ABI).

Bar: sort keys and NGP counts bit-exact; CIC/TSC (and weighted NGP) meshes
within 1e-5 per cell relative to the FP64 oracle (cells below one
particle's mass judged against one particle's mass); bitwise determinism
across runs and particle orders.
"""
import numpy as np
import pytest

import oracle as orc
from conftest import rel_err_cells
from cosmicatlas_b200 import synth
from cosmicatlas_b200.api import CIC, F32, F64, NGP, TSC, CamError, make_grid

pytestmark = pytest.mark.gpu

SCHEMES = [NGP, CIC, TSC]


def edge_positions(box, n):
    """Positions on and around cell edges and box faces."""
    f = np.float32
    d = f(box) / f(n)
    base = [0.0, np.nextafter(f(box), f(0)), box, -1e-4, box + 1e-3, d, np.nextafter(d, f(0)),
            0.5 * d, np.nextafter(f(0.5) * d, f(0)), box - 0.5 * d, 3 * d, np.nan]
    return np.array(base, np.float32)


def mixed_inputs(n, box, npart, seed):
    x, y, z = synth.clumped(npart, box, max(npart // 50, 1), 1.0 * box / n, 0.8, seed)
    e = edge_positions(box, n)
    k = len(e)
    x[:k] = e
    y[k:2 * k] = e
    z[2 * k:3 * k] = e
    x[3 * k:4 * k] = e
    y[3 * k:4 * k] = e[::-1]
    return x, y, z


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("n,box", [(64, 1000.0), (48, 777.7), (17, 100.0)])
def test_keys_bit_exact(ctx, scheme, n, box):
    x, y, z = mixed_inputs(n, box, 100_000, seed=n)
    g = make_grid(n, box)
    got = ctx.cell_keys(x, y, z, g, scheme)
    want = orc.keys(scheme, x, y, z, orc.Grid.cubic(n, box))
    assert np.array_equal(got, want)


def test_keys_non_cubic_with_origin(ctx):
    rng = np.random.default_rng(5)
    n, L, mn = (32, 48, 20), (300.0, 450.0, 200.0), (-10.0, 5.0, 100.0)
    x = rng.uniform(mn[0] - 5, mn[0] + L[0] + 5, 50_000).astype(np.float32)
    y = rng.uniform(mn[1] - 5, mn[1] + L[1] + 5, 50_000).astype(np.float32)
    z = rng.uniform(mn[2] - 5, mn[2] + L[2] + 5, 50_000).astype(np.float32)
    g = make_grid(n, L, None, mn)
    og = orc.Grid(n, L, tuple(g.d), mn)
    for s in SCHEMES:
        assert np.array_equal(ctx.cell_keys(x, y, z, g, s), orc.keys(s, x, y, z, og))


@pytest.mark.parametrize("n,box", [(128, 1000.0), (192, 1500.0)])
def test_ngp_counts_bit_exact(ctx, n, box):
    x, y, z = mixed_inputs(n, box, 400_000, seed=7)
    g = make_grid(n, box)
    r = ctx.count_ngp(x, y, z, g)
    k = orc.keys(NGP, x, y, z, orc.Grid.cubic(n, box))
    want = np.bincount(k[k < n ** 3], minlength=n ** 3).reshape(n, n, n).astype(np.uint32)
    assert np.array_equal(r.mesh, want)
    assert r.n_lost == int((k == n ** 3).sum())
    assert r.n_in + r.n_lost == x.size


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("precision", [F32, F64])
def test_mesh_vs_oracle(ctx, scheme, weighted, precision):
    n, box = 64, 1000.0
    x, y, z = mixed_inputs(n, box, 300_000, seed=11)
    w = synth.halo_masses(x.size, seed=3) if weighted else None
    g = make_grid(n, box)
    r = ctx.assign(x, y, z, w, g, scheme, precision)
    ref, lost = orc.assign_f64(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    assert r.n_lost == lost
    err = rel_err_cells(r.mesh, ref, 1.0 if w is None else float(np.mean(w)))
    assert err <= 1e-5, err
    assert abs(r.sum_mesh - ref.sum()) <= 1e-9 * ref.sum()


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("n", [2, 3, 4, 5, 7, 33, 35])
def test_small_and_ragged_meshes(ctx, scheme, n):
    # meshes smaller than a brick, and meshes whose last brick is partial
    box = 10.0 * n
    x, y, z = mixed_inputs(n, box, 20_000, seed=n)
    g = make_grid(n, box)
    r = ctx.assign(x, y, z, None, g, scheme, F64)
    ref, lost = orc.assign_f64(scheme, x, y, z, None, orc.Grid.cubic(n, box))
    assert r.n_lost == lost
    assert rel_err_cells(r.mesh, ref, 1.0) <= 1e-5


def test_non_cubic_mesh(ctx):
    rng = np.random.default_rng(9)
    n, L, mn = (40, 24, 56), (400.0, 240.0, 560.0), (0.0, 0.0, 0.0)
    x = rng.uniform(0, L[0], 80_000).astype(np.float32)
    y = rng.uniform(0, L[1], 80_000).astype(np.float32)
    z = rng.uniform(0, L[2], 80_000).astype(np.float32)
    g = make_grid(n, L, None, mn)
    for s in SCHEMES:
        r = ctx.assign(x, y, z, None, g, s, F32)
        ref, lost = orc.assign_f64(s, x, y, z, None, orc.Grid(n, L, tuple(g.d), mn))
        assert rel_err_cells(r.mesh, ref, 1.0) <= 1e-5


def test_empty_and_all_lost(ctx):
    g = make_grid(32, 100.0)
    e = np.zeros(0, np.float32)
    r = ctx.assign(e, e, e, None, g, CIC, F32)
    assert r.n_in == 0 and r.n_lost == 0 and not np.any(r.mesh)
    far = np.full(1000, 1e6, np.float32)
    r = ctx.assign(far, far, far, None, g, TSC, F32)
    assert r.n_lost == 1000 and not np.any(r.mesh)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_bitwise_deterministic(ctx, scheme):
    n, box = 96, 1000.0
    x, y, z = synth.clumped(500_000, box, 2_000, 3.0, 0.8, seed=21)
    w = synth.halo_masses(x.size, seed=22)
    g = make_grid(n, box)
    a = ctx.assign(x, y, z, w, g, scheme, F32).mesh
    b = ctx.assign(x, y, z, w, g, scheme, F32).mesh
    # same particles in a different order: same integer sums, same bits
    p = np.random.default_rng(1).permutation(x.size)
    c = ctx.assign(x[p], y[p], z[p], w[p], g, scheme, F32).mesh
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), c.view(np.uint32))


@pytest.mark.parametrize("scheme", SCHEMES)
def test_signed_weights_vs_oracle(ctx, scheme):
    # some negative weights: the deposit's signed fixed-point path
    n, box = 64, 1000.0
    x, y, z = mixed_inputs(n, box, 300_000, seed=41)
    w = synth.halo_masses(x.size, seed=42)
    w[np.random.default_rng(43).random(x.size) < 0.2] *= -1.0
    g = make_grid(n, box)
    r = ctx.assign(x, y, z, w, g, scheme, F64)
    ref, lost = orc.assign_f64(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    assert r.n_lost == lost
    err = rel_err_cells(r.mesh, ref, float(np.mean(np.abs(w))))
    assert err <= 1e-5, err


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("n", [96, 32])
def test_many_particles_vs_oracle(ctx, scheme, n):
    # 4.5 M weighted particles (clumped, plus the edge positions).  At n = 32
    # the bricks shrink to 4 x 4 x 32 cells, so TSC stencils cross brick
    # faces for most particles (several payload records per particle).
    box = 1000.0
    x, y, z = mixed_inputs(n, box, 4_500_000, seed=31 + n)
    w = synth.halo_masses(x.size, seed=32)
    g = make_grid(n, box)
    r = ctx.assign(x, y, z, w, g, scheme, F32)
    ref, lost = orc.assign_f64(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    assert r.n_lost == lost
    err = rel_err_cells(r.mesh, ref, float(np.mean(w)))
    assert err <= 1e-5, err
    p = np.random.default_rng(2).permutation(x.size)
    c = ctx.assign(x[p], y[p], z[p], w[p], g, scheme, F32).mesh
    assert np.array_equal(r.mesh.view(np.uint32), c.view(np.uint32))


def test_device_arrays_roundtrip(ctx):
    import torch
    n, box = 64, 500.0
    x, y, z = synth.clumped(100_000, box, 500, 2.0, 0.8, seed=4)
    g = make_grid(n, box)
    host = ctx.assign(x, y, z, None, g, CIC, F32).mesh
    dx, dy, dz = (torch.from_numpy(v).cuda() for v in (x, y, z))
    dev = ctx.assign(dx, dy, dz, None, g, CIC, F32).mesh
    assert dev.is_cuda
    assert np.array_equal(dev.cpu().numpy(), host)


def test_nonfinite_weight_rejected(ctx):
    x = np.array([1.0, 2.0], np.float32)
    w = np.array([1.0, np.inf], np.float32)
    with pytest.raises(CamError) as e:
        ctx.assign(x, x, x, w, make_grid(8, 10.0), CIC, F32)
    assert e.value.code == -8


def test_invalid_arguments(ctx):
    x = np.ones(4, np.float32)
    with pytest.raises(CamError) as e:
        ctx.assign(x, x, x, None, make_grid(8, 10.0), 7, F32)
    assert e.value.code == -1
    g = make_grid(8, 10.0)
    g.L[0] = -1.0
    with pytest.raises(CamError) as e:
        ctx.assign(x, x, x, None, g, CIC, F32)
    assert e.value.code == -1


# ---- against the reference's own getDensity_* (golden fixture) ------------
def _golden():
    import os
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "getdensity_ref.npz"))


@pytest.mark.parametrize("case", ["bulk", "shift", "edges"])
def test_ngp_counts_equal_reference_getdensity(ctx, case):
    # counts bit-exact against the meshes the reference's getDensity_NGP wrote
    G = _golden()
    n, L, mn = G[f"{case}_grid"]
    n = int(n)
    g = make_grid(n, float(L), None, float(mn))
    got = ctx.count_ngp(G[f"{case}_x"], G[f"{case}_y"], G[f"{case}_z"], g).mesh
    assert np.array_equal(np.asarray(got).astype(np.float32), G[f"{case}_ngp_unit"])


@pytest.mark.parametrize("case", ["bulk", "shift"])
@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("weighted", [False, True])
def test_mesh_vs_reference_getdensity(ctx, case, scheme, weighted):
    # within 1e-5 per cell of the reference's own float meshes
    G = _golden()
    n, L, mn = G[f"{case}_grid"]
    g = make_grid(int(n), float(L), None, float(mn))
    w = G[f"{case}_w"] if weighted else None
    got = ctx.assign(G[f"{case}_x"], G[f"{case}_y"], G[f"{case}_z"], w, g, scheme, F32).mesh
    want = G[f"{case}_{('ngp', 'cic', 'tsc')[scheme]}_{'mass' if weighted else 'unit'}"]
    unit = float(np.mean(w, dtype=np.float64)) if weighted else 1.0
    assert rel_err_cells(got, want, unit) <= 1e-5


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("n", [96, 384])
def test_unaligned_arrays_and_lost_particles_vs_oracle(ctx, scheme, n):
    # device arrays off the 16-byte boundary (scalar loads instead of
    # float4) and particles outside the box (counted as lost, never
    # written): the scatter takes exactly the particles its count pass
    # counted
    import torch
    box = 500.0
    rng = np.random.default_rng(n + scheme)
    npart = 400_001
    buf = rng.uniform(0.0, box, size=(4, npart + 1)).astype(np.float32)
    # every tenth particle anywhere in [-1.5 L, 2.5 L): outside the box even
    # after CIC's one periodic wrap
    buf[:3, ::10] = rng.uniform(-1.5 * box, 2.5 * box, size=(3, buf[:, ::10].shape[1])).astype(np.float32)
    buf[3] = rng.lognormal(0.0, 1.0, npart + 1).astype(np.float32)
    dbuf = torch.from_numpy(buf).cuda()
    xd, yd, zd, wd = dbuf[0, 1:], dbuf[1, 1:], dbuf[2, 1:], dbuf[3, 1:]
    assert xd.data_ptr() % 16 != 0
    x, y, z, w = buf[0, 1:], buf[1, 1:], buf[2, 1:], buf[3, 1:]
    a = ctx.assign(xd, yd, zd, wd, make_grid(n, box), scheme, F32)
    am = a.mesh.cpu().numpy()
    ref, lost = orc.assign_f64_mt(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    assert a.n_lost == lost and lost > 0
    assert rel_err_cells(am, ref, float(np.mean(w, dtype=np.float64))) <= 1e-5


@pytest.mark.parametrize("scheme", [CIC, TSC])
def test_mesh_384_vs_oracle(ctx, scheme):
    # 384^3 (6,912 bricks: the count histogram and scan of a larger mesh)
    n, box = 384, 1000.0
    x, y, z = synth.clumped(3_000_000, box, 30_000, 2.0, 0.8, seed=77 + scheme)
    w = synth.halo_masses(x.size, seed=78)
    got = ctx.assign(x, y, z, w, make_grid(n, box), scheme, F32)
    ref, lost = orc.assign_f64_mt(scheme, x, y, z, w, orc.Grid.cubic(n, box))
    assert got.n_lost == lost
    assert rel_err_cells(got.mesh, ref, float(np.mean(w, dtype=np.float64))) <= 1e-5
