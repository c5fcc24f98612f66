"""Diagonal Pauli terms evaluated through the tile's Walsh-Hadamard transform, against the oracle.

Masks cover every kind of local bit (register, lane and warp bits of the tile) and qubits outside
it, on single states and on batches."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from circuits import random_state
from quantummatter_b200.backend import FP32, FP64, DeviceState
from quantummatter_b200.observables import PauliString

pytestmark = pytest.mark.gpu


def diagonal_terms(n: int, seed: int, count: int) -> list[PauliString]:
    rng = np.random.default_rng(seed)
    out = [PauliString("I" * n)]
    out += [PauliString("".join("Z" if q == i else "I" for q in reversed(range(n)))) for i in range(n)]
    while len(out) < count:
        out.append(PauliString("".join(rng.choice(["I", "Z"], size=n))))
    # a few with flips in between, to mix both paths
    out += [PauliString("".join(rng.choice(list("IXYZ"), size=n))) for _ in range(5)]
    return out


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
@pytest.mark.parametrize("n", [9, 13, 18])
def test_many_diagonal_terms(gpu_context, n, precision, tol):
    psi = random_state(n, 100 + n) * 0.7
    obs = diagonal_terms(n, n, 40)
    with DeviceState(gpu_context, n, precision) as st:
        st.Upload(psi)
        vals, mass = st.ExpectationValues(obs)
    want = np.array([orc.expectation(psi, o) for o in obs])
    assert abs(mass - np.vdot(psi, psi).real) <= tol * mass
    assert np.max(np.abs(vals - want)) <= tol


def test_batched_diagonal_terms(gpu_context):
    from quantummatter_b200._lib import load
    from quantummatter_b200.backend import FP64
    from quantummatter_b200.trajectories import B200NoisySimulator
    from quantummatter_b200.noise import NoisyCircuit
    from quantummatter_b200.workloads import brick_circuit
    n = 14
    nc = NoisyCircuit(n).Append(brick_circuit(n, 6, seed=4))
    obs = diagonal_terms(n, 2, 30)
    res = B200NoisySimulator(gpu_context, precision=FP64).RunBatch(nc, np.zeros((3, 0)), obs)
    psi = orc.execute(brick_circuit(n, 6, seed=4))
    want = np.array([orc.expectation(psi, o) for o in obs])
    for t in range(3):
        assert np.max(np.abs(res.values[t] - want)) <= 1e-12
