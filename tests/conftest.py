import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built_lib():
    """libpgmpm.so built in-tree (nvcc cross-compiles without a GPU)."""
    from physgrad_b200 import build

    return build.build()


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    if not os.path.exists(pyoracle.LIB_PATH):
        pyoracle.build(with_ref=False)
    return pyoracle


@pytest.fixture(scope="session")
def gpu(built_lib):
    if not _cuda_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    import physgrad_b200

    physgrad_b200.lib()
    return physgrad_b200


def _read_vtk(path):
    """Parse the legacy binary VTK particle files of pgmpm_vtk_write_particles:
    returns {"header": str, "x": [n,3], "velocity": [n,3] | None, "J": [n] | None,
    "material": [n] | None, "vertices": [n,2]}."""
    import numpy as np

    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    def block(n, dt):
        nonlocal pos
        a = np.frombuffer(data, dtype=np.dtype(dt).newbyteorder(">"), count=n, offset=pos)
        pos += a.nbytes
        return a.astype(dt)

    out = {"velocity": None, "J": None, "material": None}
    assert line().startswith("# vtk DataFile")
    out["header"] = line()
    assert line() == "BINARY" and line() == "DATASET POLYDATA"
    kw, n, _ = line().split()
    n = int(n)
    out["x"] = block(3 * n, np.float32).reshape(n, 3)
    while pos < len(data):
        s = line()
        if not s:
            continue
        f = s.split()
        if f[0] == "VERTICES":
            out["vertices"] = block(int(f[2]), np.int32).reshape(-1, 2)
        elif f[0] == "POINT_DATA":
            assert int(f[1]) == n
        elif f[0] == "VECTORS":
            out[f[1]] = block(3 * n, np.float32).reshape(n, 3)
        elif f[0] == "SCALARS":
            assert line() == "LOOKUP_TABLE default"
            out[f[1]] = block(n, np.float32 if f[2] == "float" else np.int32)
    return out


@pytest.fixture(scope="session")
def read_vtk():
    return _read_vtk
