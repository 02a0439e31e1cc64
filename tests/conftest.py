"""Shared fixtures. Tests marked ``gpu`` need an sm_100 device; the rest run
on the CPU (oracle, host logic, ABI surface)."""

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "reference_unit_tests.json"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) device")


@pytest.fixture(scope="session")
def golden_cases():
    return json.loads(GOLDEN.read_text())["cases"]


def gray(rows):
    return np.array(rows, dtype=np.uint8).reshape(len(rows), -1) if rows and rows[0] else \
        np.zeros((len(rows), 0), np.uint8)


def f32_bits(rows):
    return np.array(rows, dtype=np.uint32).view(np.float32)
