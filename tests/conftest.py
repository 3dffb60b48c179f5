import json
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def gat():
    import graphautotune_b200 as g
    from graphautotune_b200 import _lib

    if not _lib.LIB_PATH.exists():
        from graphautotune_b200 import build

        build.build()
    return g


@pytest.fixture(scope="session")
def oracle():
    import pyoracle

    return pyoracle


@pytest.fixture(scope="session")
def golden_schedules():
    out = {}
    for line in (GOLDEN / "ref_schedules.jsonl").read_text().splitlines():
        if line.strip():
            d = json.loads(line)
            out[d["pattern"]] = d
    return out


@pytest.fixture(scope="session")
def golden_naive():
    return json.loads((GOLDEN / "naive_counts.json").read_text())


@pytest.fixture(scope="session")
def golden_patterns():
    return json.loads((GOLDEN / "patterns.json").read_text())


@pytest.fixture(scope="session")
def golden_graphs(gat):
    out = {}
    for p in sorted((GOLDEN / "graphs").glob("*.bin")):
        out[p.stem] = gat.Graph.load(str(p))
    return out


@pytest.fixture(scope="session")
def golden_ref_engine():
    """Answers of the reference engine itself (its target/pm.cu built for
    sm_100a and run on a B200) on the golden graphs."""
    return json.loads((GOLDEN / "ref_engine_counts.json").read_text())
