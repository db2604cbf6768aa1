"""Shared test setup: import paths, the `gpu` marker and small helpers."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "litter-physics_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


def load_request(name: str) -> dict:
    return json.loads((GOLDEN / f"{name}.request.json").read_text())


def reference_values() -> dict:
    return json.loads((GOLDEN / "reference_values.json").read_text())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle
