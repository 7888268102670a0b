"""Host-side formats either side of the path (no GPU): the raw float32 mesh
files of FileOutput::write_array / read_array (Source/FileOutput.cpp:727-912)."""
import numpy as np
import pytest

from cosmicatlas_b200.api import CamError, read_array, write_array


def test_mesh_file_round_trip(tmp_path):
    m = np.random.default_rng(5).normal(size=(16, 16, 16)).astype(np.float32)
    write_array(str(tmp_path / "mesh"), m)
    assert (tmp_path / "mesh.dat").stat().st_size == m.nbytes  # raw float32, no header
    out = np.empty(m.size, np.float32)
    read_array(str(tmp_path / "mesh.dat"), out)
    assert np.array_equal(out.reshape(m.shape), m)


def test_short_mesh_file_is_an_error(tmp_path):
    np.zeros(10, np.float32).tofile(tmp_path / "short.dat")
    with pytest.raises(CamError):
        read_array(str(tmp_path / "short.dat"), np.empty(64, np.float32))
