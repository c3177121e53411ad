"""Shared pytest setup: the `gpu` marker, repo paths and golden fixtures.

Tests marked ``gpu`` need a CUDA device and the in-tree library
(atkdsp_b200/lib/libatkdsp_b200.so); everything else runs on a CPU-only host.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / name) as z:
        return {k: z[k] for k in z.files}


def pfb_case_names(data: dict) -> list:
    return sorted({k.split("/")[0] for k in data if k.endswith("/out")})


def run_blocks(p, xs, pattern):
    """Feed element arrays xs through p.process_n in a cycling block pattern
    (the reference tests' uneven-block feeding, test_channelizer.py:74-89)."""
    n = xs[0].size
    nel = len(xs)
    outs, pos, bi = [], 0, 0
    while pos < n:
        b = min(int(pattern[bi % len(pattern)]), n - pos)
        bi += 1
        o = np.asarray(p.process_n([x[pos:pos + b] for x in xs], nel))
        if o.shape[-1]:
            outs.append(o)
        pos += b
    return np.concatenate(outs, axis=-1)


@pytest.fixture(scope="session")
def golden_pfb():
    return load_golden("pfb_cases.npz")


@pytest.fixture(scope="session")
def golden_twin():
    return load_golden("pfb_twin.npz")


@pytest.fixture(scope="session")
def golden_w12():
    return load_golden("w12.npz")


@pytest.fixture(scope="session")
def golden_unpack():
    return load_golden("unpack.npz")


@pytest.fixture(scope="session")
def golden_proto():
    return load_golden("proto.npz")


@pytest.fixture(scope="session")
def golden_osx():
    return load_golden("osx.npz")


@pytest.fixture(scope="session")
def golden_spectrum():
    return load_golden("spectrum.npz")


@pytest.fixture(scope="session")
def golden_cfar():
    return load_golden("cfar.npz")


def spectrum_case_names(data: dict) -> list:
    return sorted({k.split("/")[0] for k in data if k.endswith("/line")})
