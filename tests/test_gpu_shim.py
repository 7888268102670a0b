"""The reference-signature shim (libcam_refapi.so) called from C++ the way
the reference's translation units call getDensity_CIC, do_fftw_r2c/c2r,
EigenValuesTweb (both overloads), PoissonSolver and gradfindif, checked
against the oracle."""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle as orc
from conftest import rel_err_cells
from cosmicatlas_b200 import build as B
from cosmicatlas_b200 import synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_shim_from_cpp(tmp_path):
    shim = B.build_shim()
    exe = tmp_path / "shim_check"
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([gxx, "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "shim_check.cpp"),
                    "-L" + os.path.dirname(shim), "-lcam_refapi", "-Wl,-rpath," + os.path.dirname(shim)],
                   check=True)
    n, box = 48, 600.0
    x, y, z = synth.clumped(200_000, box, 2_000, 4.0, 0.8, seed=17)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(struct.pack("<qqf", x.size, n, box))
        for a in (x, y, z):
            f.write(a.astype(np.float32).tobytes())
    subprocess.run([str(exe), str(tmp_path)], check=True)
    mesh = np.fromfile(tmp_path / "mesh.bin", np.float32).reshape(n, n, n)
    ref, _ = orc.assign_f64(1, x, y, z, None, orc.Grid.cubic(n, box))
    assert rel_err_cells(mesh, ref, 1.0) <= 1e-5
    spec = np.fromfile(tmp_path / "spec.bin", np.complex64).reshape(n, n, n // 2 + 1)
    want = np.fft.rfftn(mesh.astype(np.float64))
    assert np.sqrt(np.mean(np.abs(spec - want) ** 2) / np.mean(np.abs(want) ** 2)) <= 2e-6
    back = np.fromfile(tmp_path / "back.bin", np.float32).reshape(n, n, n)
    assert np.max(np.abs(back - mesh)) <= 1e-5 * np.abs(mesh).max()
    delta = mesh.astype(np.float64) / mesh.astype(np.float64).mean() - 1.0
    tw = orc.tweb_from_spectrum(np.fft.rfftn(delta), n, box, 0.0, 0.0)
    l1 = np.fromfile(tmp_path / "l1.bin", np.float32).reshape(n, n, n)
    l3 = np.fromfile(tmp_path / "l3.bin", np.float32).reshape(n, n, n)
    scale = np.abs(tw.lam).max()
    assert np.max(np.abs(l1 - tw.lam[..., 0])) <= 1e-5 * scale
    assert np.max(np.abs(l3 - tw.lam[..., 2])) <= 1e-5 * scale
    # PoissonSolver, gradfindif and the finite-difference EigenValuesTweb on
    # the FP32 delta the program formed
    d32 = delta.astype(np.float32)
    phi = np.fromfile(tmp_path / "phi.bin", np.float32).reshape(n, n, n)
    phi_ref = orc.poisson_f64(np.fft.rfftn(d32.astype(np.float64)), n, box)
    assert np.max(np.abs(phi - phi_ref)) <= 1e-5 * np.abs(phi_ref).max()
    gx = np.fromfile(tmp_path / "gx.bin", np.float32).reshape(n, n, n)
    assert np.array_equal(gx, orc.gradfindif_ref_f32(phi, 0, box))
    fd = orc.tweb_fd_potential(phi.astype(np.float64), box, 0.0)
    l1 = np.fromfile(tmp_path / "fd_l1.bin", np.float32).reshape(n, n, n)
    l3 = np.fromfile(tmp_path / "fd_l3.bin", np.float32).reshape(n, n, n)
    scale = np.abs(fd.lam).max()
    assert np.max(np.abs(l1 - fd.lam[..., 0])) <= 1e-5 * scale
    assert np.max(np.abs(l3 - fd.lam[..., 2])) <= 1e-5 * scale
