"""Algorithm builders (QFT, Grover, Deutsch-Jozsa): the circuits against independent models on
the oracle, the planner's pass counts on their diagonal-heavy parts, and plans on the GPU."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle as orc
from circuits import random_state
from quantummatter_b200._lib import check, load
from quantummatter_b200.algorithms import DeutschJozsa, GroverSearch, QuantumFourierTransform
from quantummatter_b200.backend import FP64, DeviceState, Plan
from quantummatter_b200.circuit import prepare
from quantummatter_b200.errors import ArgumentError, ArgumentOutOfRangeError


def test_qft_is_the_discrete_fourier_transform():
    n = 5
    N = 1 << n
    psi = random_state(n, 3)
    want = np.array([sum(np.exp(2j * np.pi * x * y / N) * psi[x] for x in range(N)) for y in range(N)]) / math.sqrt(N)
    got = orc.execute(QuantumFourierTransform.CreateCircuit(n), psi)
    assert np.max(np.abs(got - want)) <= 1e-12
    back = orc.execute(QuantumFourierTransform.CreateCircuit(n, inverse=True), got)
    assert np.max(np.abs(back - psi)) <= 1e-12


def test_grover_amplifies_the_marked_state():
    for n, marked in ((3, 5), (5, 19), (6, 0)):
        c = GroverSearch.CreateCircuit(n, marked)
        psi = orc.execute(c)
        total = c.QubitCount
        # scratch qubits return to zero; the marked input value carries most of the mass
        probs = np.abs(psi) ** 2
        assert probs[marked] > 0.9
        assert probs[(np.arange(1 << total) >> n) != 0].sum() < 1e-24
    assert GroverSearch.RecommendedIterations(4) == round(math.pi / (4 * math.asin(0.25)) - 0.5)
    with pytest.raises(ArgumentOutOfRangeError):
        GroverSearch.CreateCircuit(3, 8)


def test_deutsch_jozsa_distinguishes_constant_and_balanced():
    n = 4
    constant = [True] * (1 << n)
    balanced = [bool((x >> 2) & 1) for x in range(1 << n)]
    for table, zero_prob in ((constant, 1.0), ([False] * (1 << n), 1.0), (balanced, 0.0)):
        psi = orc.execute(DeutschJozsa.CreateCircuit(table))
        assert abs(np.abs(psi[0]) ** 2 - zero_prob) <= 1e-12
    with pytest.raises(ArgumentError):
        DeutschJozsa.CreateCircuit([True, False, False, False, True, False, False, False])


def passes_of(circuit) -> int:
    g, n = prepare(circuit)
    P, O, pb = C.c_int32(), C.c_int32(), C.c_int64()
    check(load().qm_plan_program(circuit.QubitCount, FP64, g, n, 0, C.byref(P), None, 0, C.byref(O), None, 0,
                                 C.byref(pb)))
    return P.value


def test_qft_phase_chains_fuse():
    """A 24-qubit QFT has 24 H, 276 controlled phases and 12 SWAPs; the planner runs it in a
    handful of passes because each chain of controlled phases is a diagonal group."""
    c = QuantumFourierTransform.CreateCircuit(24)
    assert len(c.Operations) == 24 + 276 + 12
    assert passes_of(c) <= 8


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["qft", "iqft", "grover", "dj"])
def test_algorithm_plans_match_the_oracle(gpu_context, which):
    if which == "qft":
        c = QuantumFourierTransform.CreateCircuit(18)
        psi = random_state(18, 1)
    elif which == "iqft":
        c = QuantumFourierTransform.CreateCircuit(16, inverse=True)
        psi = random_state(16, 2)
    elif which == "grover":
        c = GroverSearch.CreateCircuit(8, 77, iterations=3)
        psi = orc.zero_state(c.QubitCount)
    else:
        c = DeutschJozsa.CreateCircuit([bool(bin(x).count("1") & 1) for x in range(1 << 7)])
        psi = orc.zero_state(c.QubitCount)
    want = orc.execute(c, psi)
    p = Plan(gpu_context, c, FP64, 0)
    with DeviceState(gpu_context, c.QubitCount, FP64) as st:
        st.Upload(psi)
        p.execute(st)
        got = st.Download()
    p.Dispose()
    assert np.max(np.abs(got - want)) <= 1e-12
