"""The oracle pinned against the reference's own mass assignment.

tests/golden/getdensity_ref.npz holds meshes computed by the reference's
getDensity_NGP / getDensity_CIC / getDensity_TSC (Source/massFunctions.cpp:
35-98, :678-790, :1050-1165), compiled from the reference source
(oracle/Makefile, target ref) by tests/golden/make_golden.py.  Checked here:
  * the oracle's FP32 restatement of those loops (orc_assign_ref) reproduces
    them bit for bit, unit and halo-like weights, with and without an origin
    offset;
  * the FP64 oracle with the pinned semantics agrees per cell within 1e-5 of
    max(|cell|, one mean particle weight) (the reference accumulates in float);
  * the oracle's cell keys give the reference's NGP counts exactly, on
    positions at and next to every cell face and the box faces;
  * where oracle/_ref is built, the live reference still writes the fixture.
"""
import os

import numpy as np
import pytest

import oracle as orc
from conftest import rel_err_cells

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "getdensity_ref.npz"))
NAMES = {0: "ngp", 1: "cic", 2: "tsc"}


def _case(case):
    n, L, mn = G[f"{case}_grid"]
    x, y, z = G[f"{case}_x"], G[f"{case}_y"], G[f"{case}_z"]
    w = G[f"{case}_w"] if f"{case}_w" in G else None
    return x, y, z, w, orc.Grid.cubic(int(n), float(L), float(mn))


@pytest.mark.parametrize("case", ["bulk", "shift"])
@pytest.mark.parametrize("scheme", [0, 1, 2])
@pytest.mark.parametrize("weighted", [False, True])
def test_restatement_bit_exact_vs_reference(case, scheme, weighted):
    x, y, z, w, g = _case(case)
    got, _ = orc.assign_ref(scheme, x, y, z, w if weighted else None, g)
    want = G[f"{case}_{NAMES[scheme]}_{'mass' if weighted else 'unit'}"]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", ["bulk", "shift"])
@pytest.mark.parametrize("scheme", [0, 1, 2])
@pytest.mark.parametrize("weighted", [False, True])
def test_fp64_oracle_vs_reference(case, scheme, weighted):
    x, y, z, w, g = _case(case)
    got, _ = orc.assign_f64(scheme, x, y, z, w if weighted else None, g)
    want = G[f"{case}_{NAMES[scheme]}_{'mass' if weighted else 'unit'}"]
    unit = float(np.mean(w, dtype=np.float64)) if weighted else 1.0
    assert rel_err_cells(got, want, unit) <= 1e-5


@pytest.mark.parametrize("case", ["bulk", "shift", "edges"])
def test_keys_give_reference_ngp_counts(case):
    x, y, z, _, g = _case(case)
    keys = orc.keys(0, x, y, z, g)
    ncell = int(np.prod(g.n))
    counts = np.bincount(keys, minlength=ncell + 1)[:ncell].reshape(g.n)
    assert np.array_equal(counts.astype(np.float32), G[f"{case}_ngp_unit"])


def test_live_reference_writes_the_fixture():
    if orc.ref_lib() is None:
        pytest.skip("oracle/_ref not built (the reference tree is absent)")
    for case in ("bulk", "shift"):
        x, y, z, w, g = _case(case)
        for s, name in NAMES.items():
            assert np.array_equal(orc.reference_getdensity(s, x, y, z, w, g)[0], G[f"{case}_{name}_mass"])
