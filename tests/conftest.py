"""Shared pytest configuration: the ``gpu`` marker, paths and fixture access."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
PKG = ROOT / "stl-dev-mpi_b200"
for p in (ROOT / "oracle", PKG):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine library")


class Case:
    """One golden case: tests/golden/<suite>/<name>/*.npy plus its metadata."""

    def __init__(self, suite, meta):
        self.meta = meta
        self.dir = GOLDEN / suite / meta["name"]

    @property
    def name(self):
        return self.meta["name"]

    def __getitem__(self, key):
        return self.meta[key]

    def has(self, array):
        return (self.dir / f"{array}.npy").exists()

    def npy(self, array):
        return np.load(self.dir / f"{array}.npy")

    def complex(self, name):
        return self.npy(f"{name}_re") + 1j * self.npy(f"{name}_im")


def cases(suite, kind=None):
    index = json.loads((GOLDEN / suite / "index.json").read_text())
    return [Case(suite, m) for m in index if kind is None or m["kind"] == kind]


def close_ratio(a, b, atol, rtol):
    """Worst ratio of |a - b| to atol + rtol |b| (crates/stl-core/tests/stats.rs:40-44)."""
    a, b = np.asarray(a).ravel(), np.asarray(b).ravel()
    assert a.shape == b.shape
    return float(np.max(np.abs(a - b) / (atol + rtol * np.abs(b)))) if a.size else 0.0
