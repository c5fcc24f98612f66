"""Shared test setup: import paths, the gpu marker and golden-fixture loaders."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


def known_answers() -> dict:
    return json.loads((GOLDEN / "known_answers.json").read_text())


def golden_circuits():
    """Yields (circuit, initial_state, dense_final_state) from dense_random.npz."""
    from circuits import circuit_from_arrays
    d = np.load(GOLDEN / "dense_random.npz")
    for i in range(int(d["count"])):
        arrays = {k: d[f"c{i}_{k}"] for k in ("kind", "target", "control", "second", "angle", "unitary")}
        yield circuit_from_arrays(int(d[f"c{i}_qubits"]), arrays), d[f"c{i}_initial"], d[f"c{i}_final"]


def golden_hamiltonians():
    """Yields (PauliHamiltonian, state, dense_energy, dense_per_term) from hamiltonians.npz."""
    from quantummatter_b200.observables import PauliHamiltonian, PauliString, PauliTerm
    d = np.load(GOLDEN / "hamiltonians.npz")
    for i in range(int(d["count"])):
        n = int(d[f"h{i}_qubits"])
        terms = [PauliTerm(float(c), PauliString(str(lab))) for c, lab in zip(d[f"h{i}_coeffs"], d[f"h{i}_labels"])]
        yield PauliHamiltonian(n, terms), d[f"h{i}_state"], float(d[f"h{i}_energy"]), d[f"h{i}_per_term"]


@pytest.fixture(scope="session")
def gpu_context():
    """One B200 context for the GPU tests (fails, never skips, when the library or device is missing)."""
    from quantummatter_b200.backend import B200BackendOptions, B200Context
    ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=64 << 30, StagingMemoryBudgetBytes=64 << 30))
    yield ctx
    ctx.Dispose()
