import gzip
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ncpaprop-release_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("ncpa")


@pytest.fixture(scope="session")
def canonical_profile(workdir):
    """The reference's NCPA canonical profile (samples/), from the fixture."""
    path = os.path.join(str(workdir), "NCPA_canonical_profile_zuvwtdp.dat")
    with gzip.open(os.path.join(GOLDEN, "canonical_profile.dat.gz"), "rb") as fi, open(path, "wb") as fo:
        fo.write(fi.read())
    return path


@pytest.fixture(scope="session")
def analytic_profile(workdir):
    """The analytic 0-150 km profile of the benchmark workloads."""
    import workloads

    return workloads.write_profile(os.path.join(str(workdir), "analytic_150km.dat"))


@pytest.fixture(scope="session")
def gpu():
    import ncpa_gpu

    ctx = ncpa_gpu.Context(0)
    yield ctx
    ctx.close()
