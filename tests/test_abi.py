"""The C-ABI library loads and exports every function include/cam.h declares
(no GPU: nothing is called that touches the device)."""
import os
import re

from cosmicatlas_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header="cam.h", prefix="cam_"):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*:<>]*?\b(" + prefix + r"\w*)\s*\(", src, flags=re.M))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    decl = declared_functions()
    assert "cam_assign" in decl and "cam_job_run" in decl
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert declared_functions() <= set(L.SIGNATURES)


def test_reference_shim_exports_reference_signatures():
    import subprocess
    from cosmicatlas_b200 import build as B
    so = B.SHIM_LIB
    if not os.path.exists(so):
        B.build_shim()
    out = subprocess.run(["nm", "-DC", so], capture_output=True, text=True, check=True).stdout
    names = declared_functions("cam_reference_api.h", "")
    names = {n for n in names if n in ("getDensity_NGP", "getDensity_CIC", "getDensity_TSC", "do_fftw_r2c",
                                       "do_fftw_c2r", "EigenValuesTweb", "PoissonSolver", "gradfindif",
                                       "cam_refapi_last_status")}
    assert len(names) == 9
    for n in names:
        assert any((" T " + n + "(") in line for line in out.splitlines()), n
    # both EigenValuesTweb overloads (FFT tensor of delta; FD Hessian of phi)
    assert sum(1 for line in out.splitlines() if " T EigenValuesTweb(" in line) == 2


def test_version_string():
    assert b"sm_100a" in L.lib().cam_version()


def test_no_device_means_invalid_context():
    # On a host without a GPU, context creation fails with a status code
    # instead of crashing; on a GPU host it succeeds.
    import ctypes
    h = ctypes.c_void_p()
    rc = L.lib().cam_ctx_create(0, 0, ctypes.byref(h))
    if rc == L.CAM_OK:
        assert L.lib().cam_ctx_destroy(h) == L.CAM_OK
    else:
        assert rc in (L.CAM_E_INVAL, L.CAM_E_CUDA)


def test_server_and_batch_reject_bad_arguments_without_device():
    # Host-side argument checks of the serving entry points; no device work.
    import ctypes
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.cam_server_create(0, 0, 0, 8, ctypes.byref(h)) == L.CAM_E_INVAL   # no workers
    assert lib.cam_server_create(0, 0, 2, 0, ctypes.byref(h)) == L.CAM_E_INVAL   # no batch
    assert lib.cam_server_create(0, 0, 2, 33, ctypes.byref(h)) == L.CAM_E_INVAL  # batch > 32
    assert lib.cam_server_create(-1, 0, 2, 8, ctypes.byref(h)) == L.CAM_E_INVAL  # no such device
    assert lib.cam_batch_run(None, None, 0, None) == L.CAM_E_INVAL
    assert lib.cam_server_submit(None, None, None, None) == L.CAM_E_INVAL
    assert lib.cam_server_poll(None, 1) == L.CAM_E_INVAL
    assert lib.cam_server_wait(None, 1, 0) == L.CAM_E_INVAL
    assert lib.cam_server_stats_get(None, None, 0) == L.CAM_E_INVAL
    assert lib.cam_server_destroy(None) == L.CAM_E_INVAL


def test_alloc_stats_without_device():
    # host-side counters: readable (and zero) before any device allocation
    import ctypes
    st = L.AllocStats()
    assert L.lib().cam_alloc_stats_get(ctypes.byref(st), 1) == L.CAM_OK
    assert st.allocs >= 0 and st.failures >= 0
    assert L.lib().cam_alloc_stats_get(None, 0) == L.CAM_E_INVAL


def test_new_entry_points_reject_null_context_without_device():
    # host-side guards of the finite-difference, BAM-kernel, cross-spectrum,
    # multipole, invariant and catalogue-weight entry points: no device work
    lib = L.lib()
    assert lib.cam_poisson(None, None, None, 0, 0, 0.0, None, 0) == L.CAM_E_INVAL
    assert lib.cam_gradfindif(None, None, None, 0, 0, 1, None, 0) == L.CAM_E_INVAL
    assert lib.cam_bam_kernel_update(None, None, 0, 0.0, 1.0, 8, None, 0, None, 0, None, None) == L.CAM_E_INVAL
    assert lib.cam_konvolve(None, None, None, 0, 0, None, 0, None, 0) == L.CAM_E_INVAL
    assert lib.cam_cross_power(None, None, None, None, 0, 0, None, 0, 0, None, None, None, None, None) == L.CAM_E_INVAL
    assert lib.cam_power_multipoles(None, None, None, 0, 0, None, 2, None, None, None, None, None, None) == L.CAM_E_INVAL
    assert lib.cam_tweb_invariants(None, None, None, 0, 0, None, None, None, None, 0, None) == L.CAM_E_INVAL
    assert lib.cam_fkp_weights(None, 10, None, 1.0, None, 1, 1e4, 0, None, 0, None) == L.CAM_E_INVAL
