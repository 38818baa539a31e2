"""bench.py's reference arm: the reference CPU renderer (oracle/_ref, built
from the reference sources) timed on the host cores, printed as the same
JSON line as the CUDA arm with "impl": "reference".  Under a multi-rank
launch only rank 0 runs it; the other ranks print nothing and exit 0.
A two-render batch keeps the run to a few seconds."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

REF_LIB = os.path.join(REPO, "oracle", "_ref", "libpcrref.so")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--renders", "2",
                           "--steps", "1", "--warmup", "0"], cwd=REPO, env=env, capture_output=True, text=True,
                          timeout=600)


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref not built (needs the reference sources)")
def test_reference_arm_prints_the_contract_line():
    p = _run({"RANK": "0"})
    assert p.returncode == 0, p.stderr[-2000:]
    d = json.loads(p.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference"
    assert d["unit"] == "paths/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "batch2-uneven"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert "spread evenly" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
