import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("gb")


@pytest.fixture(scope="session")
def su2_paths(workdir):
    """SU2 files of the golden-fixture meshes, written once per session."""
    import cases

    cache = {}

    def get(name):
        if name not in cache:
            path = str(workdir / f"{name}.su2")
            cases.MESHES[name]().write_su2(path)
            cache[name] = path
        return cache[name]

    return get
