"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (str(ROOT), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

from __graft_entry__ import load_oracle, load_package  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 machine)")


@pytest.fixture(scope="session")
def mm():
    return load_package()


@pytest.fixture(scope="session")
def orc():
    return load_oracle()


class Golden:
    """tests/golden/golden.npz, produced by tests/golden/make_golden.py from the reference's own code."""

    def __init__(self, path: Path):
        self.z = np.load(path)
        self.index = json.loads(bytes(self.z["index_json"]).decode())

    def cases(self, types=(6, 7, 8, 9)):
        return [c for c in self.index if c["type"] in types]

    def match(self, key):
        return self.z[key] if key in self.z.files else None

    def graph(self, mm, name):
        if name.startswith("adv_"):
            from graphs_small import SmallGraph

            r = self.z[f"{name}/ranges"]
            return SmallGraph(r.shape[0], r, self.z[f"{name}/nbrs"], self.z[f"{name}/weights"])
        kind = name.split("_")[0]
        if kind == "grid":
            w, h = name.split("_")[1].split("x")
            return mm.Graph.grid(int(w), int(h))
        if kind == "rgg":
            _, n, s = name.split("_")
            return mm.Graph.rgg(int(n), 13.0, seed=int(s[1:]))
        if kind == "rmat":
            _, sc, s = name.split("_")
            return mm.Graph.rmat(int(sc), 16, seed=int(s[1:]))
        if kind == "er":
            _, n, s = name.split("_")
            return mm.Graph.er(int(n), 8.0, seed=int(s[1:]))
        raise KeyError(name)


@pytest.fixture(scope="session")
def golden():
    return Golden(ROOT / "tests" / "golden" / "golden.npz")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
