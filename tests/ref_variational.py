"""Reference-semantics variational evaluator on the CPU oracle (test infrastructure).

Mirrors VariationalEnergyEvaluator.EvaluateWithGradient (src/QuantumMatter.Application/
Variational/VariationalEnergyEvaluator.cs:34-86): bind the base circuit and, per rotation
occurrence, the +pi/2 and -pi/2 shifted circuits (the shift is an extra same-axis gate),
evolve each from |0...0> with the scalar oracle, take per-term expectations with the oracle's
ExpectationValue restatement and assemble energy and gradient with Neumaier compensation.
"""
from __future__ import annotations

import math

import numpy as np

import oracle as orc


def _neumaier(total: float, corr: float, value: float) -> tuple[float, float]:
    nxt = total + value
    corr += (total - nxt) + value if abs(total) >= abs(value) else (value - nxt) + total
    return nxt, corr


def energy(circuit, hamiltonian, params) -> float:
    state = orc.execute(circuit.Bind(list(params)))
    return orc.energy(state, hamiltonian)


def energy_and_gradient(circuit, hamiltonian, params) -> tuple[float, np.ndarray]:
    params = list(params)
    e = energy(circuit, hamiltonian, params)
    grad = np.zeros(circuit.ParameterCount)
    corr = np.zeros(circuit.ParameterCount)
    terms = hamiltonian.Terms
    for r, p in enumerate(circuit.RotationParameterIndices):
        plus = orc.execute(circuit.BindWithRotationShift(params, r, math.pi / 2))
        minus = orc.execute(circuit.BindWithRotationShift(params, r, -math.pi / 2))
        ep = [orc.expectation(plus, t.Observable) for t in terms]
        em = [orc.expectation(minus, t.Observable) for t in terms]
        for t, a, b in zip(terms, ep, em):
            contribution = t.Coefficient * (0.5 * a - 0.5 * b)
            grad[p], corr[p] = _neumaier(grad[p], corr[p], contribution)
    return e, grad + corr
