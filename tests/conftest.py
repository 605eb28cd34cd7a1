import json
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def built_oracle():
    """The CPU oracle library is test infrastructure; build it on first use."""
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), str(ROOT / "oracle" / "liboracle.so")], check=True)


@pytest.fixture(scope="session")
def golden():
    return {
        "sphere": json.loads((GOLDEN / "beat_sphere_512.json").read_text()),
        "tetra": json.loads((GOLDEN / "beat_tetra_singular12.json").read_text()),
        "rules": json.loads((GOLDEN / "reference_rules.json").read_text()),
        "plans": np.load(GOLDEN / "reference_plans.npz"),
    }


def analytic_sphere(frequency, radius, density=1.21, c=343.0, a=0.1, v=1.0):
    """Pulsating sphere, exp(+iwt): p(r) = rho c v ika/(1+ika) (a/r) exp(-ik(r-a))
    (reference tests/bem_cuda_tests.cpp:135-140)."""
    k = 2 * np.pi * frequency / c
    return density * c * v * (1j * k * a) / (1 + 1j * k * a) * (a / radius) * np.exp(-1j * k * (radius - a))


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
