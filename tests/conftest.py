"""Shared pytest configuration: the ``gpu`` marker and golden-fixture loaders."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a) and the built libcib200.so")


def load_case(name: str) -> tuple[dict[str, np.ndarray], dict]:
    """Arrays and metadata of one golden case produced by tests/golden/make_golden.py."""
    manifest = json.loads((GOLDEN / "manifest.json").read_text())
    with np.load(GOLDEN / f"{name}.npz") as data:
        arrays = {key: data[key] for key in data.files}
    return arrays, manifest[name]


def golden_names(prefix: str) -> list[str]:
    manifest = json.loads((GOLDEN / "manifest.json").read_text())
    return sorted(name for name in manifest if name.startswith(prefix))


def load_failures() -> dict:
    return json.loads((GOLDEN / "j2_failures.json").read_text())
