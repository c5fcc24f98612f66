"""Variational layer: binding semantics and the VQE solver's host logic (CPU), and the batched
B200 energy/gradient evaluator against the oracle-composed reference evaluator (GPU)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import ref_variational as ref
from quantummatter_b200.circuit import GateKind, QuantumCircuit
from quantummatter_b200.errors import ArgumentError, ArgumentOutOfRangeError
from quantummatter_b200.observables import PauliHamiltonian, PauliString, PauliTerm
from quantummatter_b200.variational import (ParameterizedCircuit, VariationalEnergyResult, VqeOptions, VqeSolver,
                                            VqeTerminationReason)
from quantummatter_b200.workloads import hardware_efficient_ansatz, uniform_parameters, xxz_chain


def Z(coefficient: float = 1.0, qubits: int = 1) -> PauliHamiltonian:
    return PauliHamiltonian(qubits, [PauliTerm(coefficient, PauliString("I" * (qubits - 1) + "Z"))])


# ---------------------------------------------------------------- CPU: template semantics

def test_bind_appends_the_shift_after_one_occurrence():
    """ParameterizedCircuit.cs:68-96: the shift is a separate same-axis gate, never added to the angle."""
    c = ParameterizedCircuit(2, 2).Ry(0, 0).Append(QuantumCircuit(2).CNot(0, 1)).Rz(1, 1).Ry(1, 0)
    b = c.BindWithRotationShift([1e100, 0.2], 2, math.pi / 2)
    kinds = [(op.Kind, op.Target, op.Angle) for op in b.Operations]
    assert kinds == [(GateKind.Ry, 0, 1e100), (GateKind.CNot, 1, 0.0), (GateKind.Rz, 1, 0.2),
                     (GateKind.Ry, 1, 1e100), (GateKind.Ry, 1, math.pi / 2)]
    assert c.RotationParameterIndices == (0, 1, 0) and c.OperationCount == 4
    with pytest.raises(ArgumentError):
        c.Bind([0.1])
    with pytest.raises(ArgumentOutOfRangeError):
        c.Bind([0.1, float("nan")])
    with pytest.raises(ArgumentOutOfRangeError):
        c.BindWithRotationShift([0.1, 0.2], 3, 1.0)


class FakeEvaluator:
    """Energy E(theta) = sum (theta_i - 1)^2 with exact gradients; counts calls."""

    def __init__(self):
        self.energies = 0
        self.gradients = 0

    def Evaluate(self, circuit, hamiltonian, params):
        self.energies += 1
        return float(sum((p - 1) ** 2 for p in params))

    def EvaluateWithGradient(self, circuit, hamiltonian, params):
        self.gradients += 1
        return VariationalEnergyResult(float(sum((p - 1) ** 2 for p in params)), tuple(2 * (p - 1) for p in params))


def test_vqe_solver_counts_and_termination_reasons():
    """VqeSolverTests.cs:33-181: accounting of energies, gradients and circuits; stopping reasons."""
    c = ParameterizedCircuit(1, 2).Ry(0, 0).Rz(0, 1)
    h = Z()
    fake = FakeEvaluator()
    r = VqeSolver(fake, VqeOptions(GradientTolerance=1e-9, InitialStepSize=0.5)).Solve(c, h, [0.0, 3.0])
    assert r.TerminationReason == VqeTerminationReason.GradientToleranceReached
    assert np.allclose(r.Parameters, [1.0, 1.0]) and r.Energy == 0
    assert r.GradientEvaluationCount == fake.gradients and r.EnergyEvaluationCount == fake.energies
    assert r.CircuitEvaluationCount == r.EnergyEvaluationCount + 5 * r.GradientEvaluationCount
    r = VqeSolver(FakeEvaluator(), VqeOptions(MaximumIterations=0)).Solve(c, h, [0.0, 0.0])
    assert r.TerminationReason == VqeTerminationReason.IterationLimitReached and r.CircuitEvaluationCount == 1
    r = VqeSolver(FakeEvaluator(), VqeOptions(MaximumCircuitEvaluations=5)).Solve(c, h, [0.0, 0.0])
    assert r.TerminationReason == VqeTerminationReason.EvaluationLimitReached
    with pytest.raises(ArgumentOutOfRangeError):
        VqeOptions(BacktrackingFactor=1.0).Validate()


# ---------------------------------------------------------------- GPU: batched evaluator

@pytest.fixture(scope="module")
def evaluator(gpu_context):
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    return B200VariationalEnergyEvaluator(gpu_context)


def near(a, b, tol=5e-12):
    assert abs(a - b) <= tol, (a, b)


@pytest.mark.gpu
def test_reference_gradient_cases(evaluator):
    """VariationalEnergyTests.cs:17-45: product rule for a shared parameter, a 1e100 angle, a 1e16
    identity offset and a 1e308 coefficient."""
    shared = ParameterizedCircuit(1, 2).Ry(0, 0).Ry(0, 0)
    angle = 0.37
    r = evaluator.EvaluateWithGradient(shared, Z(), [angle, 17])
    near(math.cos(2 * angle), r.Energy)
    near(-2 * math.sin(2 * angle), r.Gradient[0])
    assert r.Gradient[1] == 0
    single = ParameterizedCircuit(1, 1).Ry(0, 0)
    huge = 1e100
    r = evaluator.EvaluateWithGradient(single, Z(), [huge])
    near(math.cos(huge), r.Energy)
    near(-math.sin(huge), r.Gradient[0])
    offset = PauliHamiltonian(1, [PauliTerm(1e16, PauliString("I")), PauliTerm(1, PauliString("Z"))])
    near(-math.sin(angle), evaluator.EvaluateWithGradient(single, offset, [angle]).Gradient[0])
    large = evaluator.EvaluateWithGradient(single, Z(1e308), [math.pi / 2])
    assert abs(large.Gradient[0] / 1e308 + 1) <= 4e-12


def random_template(qubits: int, params: int, seed: int) -> ParameterizedCircuit:
    rng = np.random.default_rng(seed)
    c = ParameterizedCircuit(qubits, params)
    for _ in range(6 * qubits):
        r = rng.random()
        q = int(rng.integers(qubits))
        if r < 0.5:
            getattr(c, ("Rx", "Ry", "Rz")[int(rng.integers(3))])(q, int(rng.integers(params)))
        else:
            seg = QuantumCircuit(qubits)
            other = (q + 1 + int(rng.integers(qubits - 1))) % qubits if qubits > 1 else q
            if qubits > 1 and r < 0.75:
                seg.CNot(q, other)
            elif qubits > 1 and r < 0.85:
                seg.CZ(q, other)
            else:
                seg.H(q).S(q)
            c.Append(seg)
    return c


def random_hamiltonian(qubits: int, seed: int) -> PauliHamiltonian:
    rng = np.random.default_rng(seed)
    terms = [PauliTerm(float(rng.normal()), PauliString("".join(rng.choice(list("IXYZ"), size=qubits))))
             for _ in range(2 * qubits + 3)]
    return PauliHamiltonian(qubits, terms)


@pytest.mark.gpu
@pytest.mark.parametrize("qubits", [2, 5, 10, 12])
def test_energy_and_gradient_match_the_oracle_evaluator(evaluator, qubits):
    c = random_template(qubits, 4, seed=qubits)
    h = random_hamiltonian(qubits, seed=100 + qubits)
    params = uniform_parameters(4, 2, -math.pi, math.pi, seed=qubits)
    batch = evaluator.EvaluateBatch(c, h, params, withGradient=True)
    for v in range(2):
        e, g = ref.energy_and_gradient(c, h, params[v])
        scale = max(1.0, sum(abs(t.Coefficient) for t in h.Terms))
        near(batch.Energies[v], e, 5e-12 * scale)
        assert np.max(np.abs(batch.Gradients[v] - g)) <= 5e-12 * scale
    assert batch.Circuits == 2 * (1 + 2 * len(c.RotationParameterIndices))


@pytest.mark.gpu
def test_batched_vectors_equal_single_evaluations_bit_for_bit(evaluator):
    c = hardware_efficient_ansatz(10, 2)
    h = xxz_chain(10)
    params = uniform_parameters(c.ParameterCount, 5, -math.pi, math.pi, seed=3)
    batch = evaluator.EvaluateBatch(c, h, params, withGradient=True)
    for v in (0, 3):
        one = evaluator.EvaluateBatch(c, h, params[v], withGradient=True)
        assert one.Energies[0] == batch.Energies[v]
        assert np.array_equal(one.Gradients[0], batch.Gradients[v])


@pytest.mark.gpu
def test_fp32_energies_within_1e6_of_the_fp64_oracle(gpu_context):
    from quantummatter_b200.backend import FP32
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    n = 16
    c = hardware_efficient_ansatz(n, 4)
    h = xxz_chain(n)
    params = uniform_parameters(c.ParameterCount, 4, -math.pi, math.pi, seed=16)
    fp32 = B200VariationalEnergyEvaluator(gpu_context, FP32).EvaluateBatch(c, h, params, withGradient=False)
    for v in range(4):
        want = ref.energy(c, h, params[v])
        assert abs(fp32.Energies[v] - want) <= 1e-6, (fp32.Energies[v], want)


def structured_hamiltonian(qubits: int, diagonal: int, seed: int) -> PauliHamiltonian:
    """Terms that reach every branch of the tiled expectation compiled for a term list: flips
    whose highest bit is a thread bit of the tile (a zero is inserted below the register bits)
    with Z/Y on the bits just above; more than eight terms sharing one flip mask; flips on
    register bits; and `diagonal` Z-only terms (fewer than three, or a Walsh-Hadamard set)."""
    rng = np.random.default_rng(seed)
    terms = []

    def add(ops):
        lab = ["I"] * qubits
        for q, p in ops.items():
            lab[qubits - 1 - q] = p
        terms.append(PauliTerm(float(rng.normal()), PauliString("".join(lab))))

    for z in range(10):  # one flip mask {0, 1}, ten Z patterns above it
        ops = {0: "X", 1: "Y" if z % 2 else "X"}
        for q in range(2, qubits):
            if (z >> (q % 4)) & 1:
                ops[q] = "Z"
        add(ops)
    for q in range(qubits - 1):  # X/Y pairs on every bond, Z on the qubit after
        add({q: "X", q + 1: "X"})
        add({q: "Y", q + 1: "Y", (q + 2) % qubits: "Z"} if q + 2 < qubits else {q: "Y", q + 1: "Y"})
    for d in range(diagonal):
        add({d % qubits: "Z", (3 * d + 1) % qubits: "Z"} if d % 2 else {(5 * d) % qubits: "Z"})
    return PauliHamiltonian(qubits, terms)


@pytest.mark.gpu
@pytest.mark.parametrize("diagonal", [2, 6])
@pytest.mark.parametrize("fp32", [False, True])
def test_compiled_tile_expectation_matches_the_oracle(gpu_context, diagonal, fp32):
    from quantummatter_b200.backend import FP32, FP64
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    n = 14
    c = hardware_efficient_ansatz(n, 2)
    h = structured_hamiltonian(n, diagonal, seed=diagonal)
    params = uniform_parameters(c.ParameterCount, 3, -math.pi, math.pi, seed=14)
    from quantummatter_b200.backend import jit_info
    ev = B200VariationalEnergyEvaluator(gpu_context, FP32 if fp32 else FP64)
    before = jit_info()
    got = ev.EvaluateBatch(c, h, params, withGradient=False)
    after = jit_info()
    # passes and tile expectations ran compiled, none failed
    assert after["failed"] == before["failed"] and after["launches"] > before["launches"]
    scale = max(1.0, sum(abs(t.Coefficient) for t in h.Terms))
    for v in range(3):
        want = ref.energy(c, h, params[v])
        assert abs(got.Energies[v] - want) <= (1e-6 if fp32 else 5e-12) * scale, (v, got.Energies[v], want)


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [False, True])
def test_mixed_sizes_equal_separate_evaluations(gpu_context, fp32):
    """qm_vqe_evaluate_mixed: 10-, 12- and 14-qubit problems together (their own streams, rounds
    replayed as one graph) give the separate calls' energies and gradients bit for bit."""
    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    # a small device budget: several waves per size, so full rounds replay the captured graph
    ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=(24 if fp32 else 48) << 20,
                                         StagingMemoryBudgetBytes=1 << 30))
    ev = B200VariationalEnergyEvaluator(ctx, FP32 if fp32 else FP64)
    problems = []
    for n in (10, 12, 14):
        c = hardware_efficient_ansatz(n, 2)
        problems.append((c, xxz_chain(n, seed=n), uniform_parameters(c.ParameterCount, 3, -math.pi, math.pi, seed=n)))
    try:
        outs, total = ev.EvaluateMixed(problems)
        assert total.Circuits == sum(3 * (1 + 2 * len(c.RotationParameterIndices)) for c, _, _ in problems)
        assert total.Waves >= 3
        for (c, h, p), (e, g) in zip(problems, outs):
            alone = B200VariationalEnergyEvaluator(gpu_context, ev.precision).EvaluateBatch(c, h, p, withGradient=True)
            assert np.array_equal(e, alone.Energies)
            assert np.array_equal(g, alone.Gradients)
    finally:
        ctx.Dispose()
