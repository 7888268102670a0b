"""The C-ABI library loads and exports every function include/cam.h declares
(no GPU: nothing is called that touches the device)."""
import os
import re

from cosmicatlas_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cam_\w+)\s*\(", src, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    decl = declared_functions()
    assert "cam_assign" in decl and "cam_job_run" in decl
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert declared_functions() <= set(L.SIGNATURES)


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
