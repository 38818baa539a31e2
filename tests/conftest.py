import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
SCENES = os.path.join(GOLDEN, "scenes")
sys.path.insert(0, REPO)

# The reference project's tree (for the tests that read it directly: the
# reference loader's own bunny load, the adapter compile check).  Named by
# PCR_REFERENCE_ROOT, else looked for beside this repository; absent on
# machines that only carry the repository, where those tests skip.  The
# bunny and every scene the GPU tests use are committed under tests/golden.
REFERENCE_ROOT = os.environ.get("PCR_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO), "reference")
BUNNY_SCENE = os.path.join(SCENES, "cornell-bunny.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def scene_path(name: str) -> str:
    return os.path.join(SCENES, name + ".json")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle


def have_bunny() -> bool:
    return os.path.exists(os.path.join(GOLDEN, "models", "stanford-bunny.obj"))


def have_reference() -> bool:
    return os.path.exists(os.path.join(REFERENCE_ROOT, "code", "Renderer.cpp"))
