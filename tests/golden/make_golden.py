"""Writes tests/golden/getdensity_ref.npz: meshes computed by the reference's
own getDensity_NGP / getDensity_CIC / getDensity_TSC (Source/massFunctions.cpp,
compiled from the reference source by oracle/Makefile, target ref) on small
seeded catalogues, for the tests to pin the oracle and the GPU path against
where the reference tree is not available.

    python tests/golden/make_golden.py      (needs oracle/_ref/libref_mass.so)

Cases (unit and halo-like weights for each scheme):
  bulk  : 4,000 clumped particles, 16^3 cells, L = 100, origin 0;
  shift : 2,000 clumped particles, 12^3 cells, L = 50, origin -25 (the box
          spans [-25, 25));
  edges : positions on and next to cell faces and the box faces, NGP only
          (counts = the reference's cell keys).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as orc  # noqa: E402
from cosmicatlas_b200 import synth  # noqa: E402


def edge_positions(n, L, seed):
    rng = np.random.default_rng(seed)
    d = np.float32(np.float32(L) / np.float32(n))
    faces = (np.arange(n + 1, dtype=np.float32) * d).astype(np.float32)
    cand = np.concatenate([faces, np.nextafter(faces, np.float32(-1)), np.nextafter(faces, np.float32(2 * L)),
                           np.float32([0.0, L, np.nextafter(np.float32(L), np.float32(0)), -1e-3, L + 1e-3])])
    cand = cand.astype(np.float32)
    m = 1500
    return [cand[rng.integers(0, cand.size, m)] for _ in range(3)]


def main():
    if orc.build_ref() is None:
        raise SystemExit("oracle/_ref/libref_mass.so is not available")
    out = {}
    for case, (npart, n, L, mn, seed) in {"bulk": (4000, 16, 100.0, 0.0, 71),
                                          "shift": (2000, 12, 50.0, -25.0, 72)}.items():
        x, y, z = synth.clumped(npart, L, npart // 60, 1.5, 0.8, seed)
        x, y, z = [(np.float32(mn) + v).astype(np.float32) for v in (x, y, z)]
        w = synth.halo_masses(npart, seed=seed + 100)
        g = orc.Grid.cubic(n, L, mn)
        out[f"{case}_x"], out[f"{case}_y"], out[f"{case}_z"], out[f"{case}_w"] = x, y, z, w
        out[f"{case}_grid"] = np.array([n, L, mn], np.float64)
        for s, name in ((0, "ngp"), (1, "cic"), (2, "tsc")):
            out[f"{case}_{name}_unit"] = orc.reference_getdensity(s, x, y, z, None, g)[0]
            out[f"{case}_{name}_mass"] = orc.reference_getdensity(s, x, y, z, w, g)[0]
    n, L = 8, 40.0
    x, y, z = edge_positions(n, L, 73)
    out["edges_x"], out["edges_y"], out["edges_z"] = x, y, z
    out["edges_grid"] = np.array([n, L, 0.0], np.float64)
    out["edges_ngp_unit"] = orc.reference_getdensity(0, x, y, z, None, orc.Grid.cubic(n, L))[0]
    np.savez_compressed(os.path.join(HERE, "getdensity_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "getdensity_ref.npz"))


if __name__ == "__main__":
    main()
