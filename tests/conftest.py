import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
SCENES = os.path.join(GOLDEN, "scenes")
sys.path.insert(0, REPO)

# The reference tree exists only in the build container; tests that need
# files that are not committed (the Stanford bunny OBJ) skip elsewhere.
REFERENCE_ROOT = os.environ.get("PCR_REFERENCE_ROOT", "/root/reference")
BUNNY_SCENE = os.path.join(REFERENCE_ROOT, "Scenes", "cornell-bunny.json")


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
    return os.path.exists(os.path.join(REFERENCE_ROOT, "models", "stanford-bunny.obj"))
