import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcam.so")


@pytest.fixture(scope="session")
def ctx():
    """A libcam context on cuda:0 (GPU tests only)."""
    from cosmicatlas_b200.api import Context
    c = Context(0)
    yield c
    c.close()


def rel_err_cells(a, b, unit):
    """max over cells |a - b| / max(|b|, unit): per-cell relative error, where
    a cell holding less than one particle's mass (`unit` = mean particle
    weight, 1 for unit masses) is judged against one particle's mass.  Cells
    that only receive a stencil tail of ~1e-8 of a particle cannot carry a
    relative error: the fractional offsets themselves are exact only to
    ~1e-7 cells in FP32."""
    import numpy as np
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), unit)))


def pk_rel_err(pk, pk_ref, floor):
    """|dP| / max(|P_oracle|, SN C(k)/W^2) per bin (the shot-noise level is the
    floor where shot-noise-subtracted bins approach zero)."""
    import numpy as np
    pk = np.asarray(pk, np.float64)
    pk_ref = np.asarray(pk_ref, np.float64)
    den = np.maximum(np.abs(pk_ref), np.abs(np.asarray(floor, np.float64)))
    den = np.where(den > 0, den, 1.0)
    return float(np.max(np.abs(pk - pk_ref) / den))
