"""Shared pytest configuration.

Markers: ``gpu`` -- needs a CUDA device (the B200); everything else runs on the CPU.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _mesh(x, y, z, i0, i1, i2) -> dict:
    return {"x": np.array(x, np.float32), "y": np.array(y, np.float32), "z": np.array(z, np.float32),
            "i0": np.array(i0, np.uint32), "i1": np.array(i1, np.uint32), "i2": np.array(i2, np.uint32)}


# Analytic meshes of smallgwn's tests (tests/test_meshes.hpp:13-53, tests/test_fixtures.cuh:14-21,
# tests/unit_gwn_query_winding.cu:23-30), restated.
def octahedron() -> dict:
    return _mesh([1, -1, 0, 0, 0, 0], [0, 0, 1, -1, 0, 0], [0, 0, 0, 0, 1, -1],
                 [0, 2, 1, 3, 2, 1, 3, 0], [2, 1, 3, 0, 0, 2, 1, 3], [4, 4, 4, 4, 5, 5, 5, 5])


def asym_octahedron() -> dict:
    return _mesh([1.7, -0.8, 0.15, -0.1, 0.2, -0.2], [0.1, -0.2, 1.2, -0.7, 0.1, -0.1],
                 [0, 0.1, -0.1, 0.15, 1.5, -0.9],
                 [0, 2, 1, 3, 2, 1, 3, 0], [2, 1, 3, 0, 0, 2, 1, 3], [4, 4, 4, 4, 5, 5, 5, 5])


def cube() -> dict:
    return _mesh([-1, 1, 1, -1, -1, 1, 1, -1], [-1, -1, 1, 1, -1, -1, 1, 1], [-1, -1, -1, -1, 1, 1, 1, 1],
                 [0, 0, 4, 4, 0, 0, 1, 1, 0, 0, 3, 3], [2, 3, 5, 6, 4, 7, 2, 6, 1, 5, 7, 6],
                 [1, 2, 6, 7, 7, 3, 6, 5, 5, 4, 6, 2])


def open_cube() -> dict:
    return _mesh([-1, 1, 1, -1, -1, 1, 1, -1], [-1, -1, 1, 1, -1, -1, 1, 1], [-1, -1, -1, -1, 1, 1, 1, 1],
                 [0, 0, 0, 0, 1, 1, 0, 0, 3, 3], [2, 3, 4, 7, 2, 6, 1, 5, 7, 6], [1, 2, 7, 3, 6, 5, 5, 4, 6, 2])


def single_triangle() -> dict:
    return _mesh([0, 1, 0], [0, 0, 1], [0, 0, 0], [0], [1], [2])


def equal_bounds(count: int) -> dict:
    return _mesh([0, 1, 0], [0, 0, 1], [0, 0, 0], [0] * count, [1] * count, [2] * count)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    torch.cuda.set_device(0)
    return torch


def golden_files() -> list[Path]:
    return sorted(GOLDEN.glob("*.npz"))
