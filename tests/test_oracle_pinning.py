"""Pins the CPU oracle (oracle/) against the reference test suite's known answers and the
independent dense-matrix fixtures.  CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

import dense_model as dm
import oracle as orc
from circuits import random_circuit, random_state
from conftest import golden_circuits, golden_hamiltonians, known_answers
from quantummatter_b200.circuit import GateKind, GateOperation, QuantumCircuit
from quantummatter_b200.observables import PauliHamiltonian, PauliString, PauliTerm


def _append(c: QuantumCircuit, kind: GateKind, target: int, angle: float) -> None:
    c.AppendValidated(GateOperation(kind, target, -1, angle))


def test_known_matrix_columns_on_every_target_with_spectators_set():
    """StateVectorBackendConformanceTests.cs:14-70: every column on every target of 4 qubits."""
    ka = known_answers()
    for name, inp, zero, one in ka["columns"]:
        kind = GateKind[name]
        for target in range(4):
            c = QuantumCircuit(4)
            spectators = 15 ^ (1 << target)
            for q in range(4):
                if q != target or inp == 1:
                    c.X(q)
            _append(c, kind, target, ka["angle"])
            s = orc.execute(c)
            for index in range(16):
                expected = complex(*zero) if index == spectators else complex(*one) if index == 15 else 0
                assert abs(s[index] - expected) <= 1e-12, (name, inp, target, index)


def test_cnot_and_swap_truth_tables_all_orders():
    """StateVectorBackendConformanceTests.cs:72-97."""
    for first in range(4):
        for second in range(4):
            if first == second:
                continue
            for basis in range(16):
                c = QuantumCircuit(4)
                for q in range(4):
                    if basis >> q & 1:
                        c.X(q)
                cn = c.Copy().CNot(first, second)
                exp = basis if not basis >> first & 1 else basis ^ (1 << second)
                s = orc.execute(cn)
                assert abs(s[exp] - 1) < 1e-15 and np.sum(np.abs(s)) == pytest.approx(1.0)
                sw = c.Copy().Swap(first, second)
                same = (basis >> first & 1) == (basis >> second & 1)
                exp = basis if same else basis ^ (1 << first) ^ (1 << second)
                s = orc.execute(sw)
                assert abs(s[exp] - 1) < 1e-15


def test_interference_and_ghz():
    """StateVectorBackendConformanceTests.cs:99-109."""
    s = orc.execute(QuantumCircuit(1).H(0).Z(0).H(0))
    assert abs(s[1] - 1) < 1e-12
    assert abs(orc.execute(QuantumCircuit(1).X(0).S(0))[1] - 1j) < 1e-12
    assert abs(orc.execute(QuantumCircuit(1).S(0).X(0))[1] - 1) < 1e-12
    g = orc.execute(QuantumCircuit(4).H(0).CNot(0, 2).CNot(2, 3).CNot(3, 1))
    assert abs(g[0] - math.sqrt(0.5)) < 1e-12 and abs(g[15] - math.sqrt(0.5)) < 1e-12
    assert np.all(np.abs(g[1:15]) < 1e-12)


def _inverse(c: QuantumCircuit) -> QuantumCircuit:
    inv = QuantumCircuit(c.QubitCount)
    for op in reversed(c.Operations):
        k = op.Kind
        if k in (GateKind.Rx, GateKind.Ry, GateKind.Rz, GateKind.Phase):
            inv.AppendValidated(GateOperation(k, op.Target, op.Control, -op.Angle, op.SecondControl))
        elif k == GateKind.S:
            inv.AppendValidated(GateOperation(GateKind.Sdg, op.Target, op.Control))
        elif k == GateKind.Sdg:
            inv.AppendValidated(GateOperation(GateKind.S, op.Target, op.Control))
        elif k == GateKind.T:
            inv.AppendValidated(GateOperation(GateKind.Tdg, op.Target, op.Control))
        elif k == GateKind.Tdg:
            inv.AppendValidated(GateOperation(GateKind.T, op.Target, op.Control))
        elif k == GateKind.Unitary:
            inv.AppendValidated(GateOperation(k, op.Target, op.Control, 0.0, -1, op.Unitary.Adjoint()))
        else:
            inv.AppendValidated(op)
    return inv


def test_long_circuit_preserves_norm_and_inverse_recovers_input():
    """StateVectorBackendConformanceTests.cs:111-143 (200 rounds on 5 qubits, tolerance 1e-11)."""
    c = QuantumCircuit(5)
    for r in range(200):
        c.H(r % 5).Rx((r + 1) % 5, 0.371).Ry((r + 2) % 5, -1.28).Rz((r + 3) % 5, 2.4)
        c.CNot(r % 5, (r + 1) % 5).Swap((r + 2) % 5, (r + 4) % 5)
    s = orc.execute(c)
    assert abs(np.vdot(s, s).real - 1) < 1e-11
    back = orc.execute(_inverse(c), s)
    assert abs(back[0] - 1) < 1e-11 and np.all(np.abs(back[1:]) < 1e-11)


def test_oracle_matches_dense_fixtures_on_random_circuits():
    """The dense-oracle method of StateVectorBackendConformanceTests.cs:146-245 (tolerance 2e-12)."""
    n = 0
    for circuit, initial, final in golden_circuits():
        got = orc.execute(circuit, initial)
        assert np.max(np.abs(got - final)) <= 2e-12
        n += 1
    assert n == 15


def test_prepared_gates_reproduce_the_scalar_backend_bit_for_bit():
    """PreparedStateVectorGate + the pair kernel equal CpuStateVectorBackend exactly."""
    for seed in range(6):
        c = random_circuit(5, 120, seed=seed)
        psi = random_state(5, seed)
        gates = orc.prepare(c)
        a = orc.apply_prepared(gates, len(c.Operations), 5, psi)
        b = orc.execute(c, psi)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("workers", [1, 2, 3, 7])
def test_parallel_avx512_baseline_matches_scalar(workers):
    """ParallelCpuBackendTests.cs:14-160: uneven partitions, 73-gate runs across the 32-gate block bound."""
    c = QuantumCircuit(9)
    for i in range(73):
        c.Ry(i % 9 if i % 2 else 6, 0.1 * i)
    for seed in range(3):
        c2 = random_circuit(9, 150, seed=50 + seed)
        for circ in (c, c2):
            psi = random_state(9, seed)
            want = orc.execute(circ, psi)
            got = orc.execute_parallel(circ, psi.copy(), workers=workers, min_parallel_qubits=1)
            assert np.max(np.abs(got - want)) <= 1e-12


def test_pauli_eigenstates_and_bell_correlations():
    """StateObservationTests.cs:158-190."""
    ka = known_answers()
    for labels, value, prep in ka["eigen"]:
        c = QuantumCircuit(1)
        for g in filter(None, prep.split(",")):
            getattr(c, g)(0)
        assert abs(orc.expectation(orc.execute(c), PauliString(labels)) - value) < 1e-12
    bell = orc.execute(QuantumCircuit(2).H(0).CNot(0, 1))
    for labels, value in ka["bell"]:
        assert abs(orc.expectation(bell, PauliString(labels)) - value) < 1e-12


def test_all_pauli_strings_match_dense_on_random_states():
    """StateObservationTests.cs:131: every Pauli product on up to 3 qubits against dense operators."""
    import itertools
    for n in (1, 2, 3):
        psi = random_state(n, seed=n) * 1.7  # unnormalised: the value is divided by the Born mass
        for labels in itertools.product("IXYZ", repeat=n):
            lab = "".join(labels)
            assert abs(orc.expectation(psi, PauliString(lab)) - dm.expectation(psi, lab)) < 1e-12


def test_energy_matches_dense_fixtures():
    for h, psi, energy, _ in golden_hamiltonians():
        assert abs(orc.energy(psi, h) - energy) < 5e-12


def test_energy_cancellation_and_empty_hamiltonian():
    """PauliHamiltonianTests.cs:40-53: Neumaier keeps the 1 between +-1e16."""
    s = orc.zero_state(1)
    assert orc.energy(s, PauliHamiltonian(1, [])) == 0
    assert orc.energy(s, PauliHamiltonian(1, [PauliTerm(-3, PauliString("I"))])) == -3
    canceling = PauliHamiltonian(1, [PauliTerm(1e16, PauliString("I")), PauliTerm(1, PauliString("I")),
                                     PauliTerm(-1e16, PauliString("I"))])
    assert orc.energy(s, canceling) == 1
    eig = np.array([math.sqrt(0.5), 1j * math.sqrt(0.5)])
    h = PauliHamiltonian(1, [PauliTerm(-2, PauliString("Y")), PauliTerm(0, PauliString("Z"))])
    assert abs(orc.energy(eig, h) + 2) < 1e-12


def test_depolarizing_boundaries_and_zero_noise_draw_nothing():
    """NoiseChannelTests.cs:37-64."""
    psi = random_state(2, seed=3)
    for kind in range(4):
        out, used = orc.noise_apply(kind, 0.0, 1, psi, [0.3])
        assert used == 0 and np.array_equal(out, psi)
    paulis = {0: np.eye(2), 1: dm.single_matrix(dm.X), 2: dm.single_matrix(dm.Y), 3: dm.single_matrix(dm.Z)}
    for draw, pauli in known_answers()["depolarizing_p1"]:
        out, used = orc.noise_apply(2, 1.0, 0, psi, [draw])
        assert used == 1
        assert np.max(np.abs(out - dm.embed(paulis[pauli], 0, 2) @ psi)) < 1e-15


def test_flip_boundary_and_unit_probability():
    """NoiseChannelTests.cs:131-141: draw == p selects identity; p == 1 needs no draw."""
    psi = random_state(2, seed=4)
    for kind, pauli in ((0, dm.X), (1, dm.Z)):
        out, used = orc.noise_apply(kind, 0.5, 0, psi, [0.5])
        assert used == 1 and np.array_equal(out, psi)
        out, used = orc.noise_apply(kind, 1.0, 0, psi, [])
        assert used == 0
        assert np.max(np.abs(out - dm.embed(dm.single_matrix(pauli), 0, 2) @ psi)) < 1e-15


def test_damping_boundaries():
    """NoiseChannelTests.cs:113-129."""
    r = math.sqrt(0.5)
    out, used = orc.noise_apply(3, 0.5, 0, np.array([r, 1j * r]), [0.25])
    assert used == 1
    assert np.max(np.abs(out - np.array([math.sqrt(2 / 3), 1j / math.sqrt(3)]))) < 1e-12
    out, used = orc.noise_apply(3, 1.0, 0, np.array([1j, 0]), [])
    assert used == 0 and np.array_equal(out, np.array([1j, 0]))
    out, used = orc.noise_apply(3, 1.0, 0, np.array([0, 1j]), [])
    assert used == 0 and np.array_equal(out, np.array([1j, 0]))
    out, used = orc.noise_apply(3, 5e-324, 0, np.array([0, 1j]), [0.0])
    assert np.max(np.abs(out - np.array([1j, 0]))) < 1e-12


def test_kraus_branches_reproduce_the_channel_density():
    """NoiseChannelTests.cs:66-111: the branch-weighted conditional states rebuild the Kraus density."""
    p = 0.37
    for kind in range(4):
        for n in (1, 2, 3):
            for t in range(n):
                psi = random_state(n, seed=10 * n + t)
                rho = np.zeros((1 << n, 1 << n), dtype=complex)
                if kind == 3:
                    m0, m1 = orc.qubit_masses(psi, t)
                    jump_w = p * m1
                    for draw, w in ((0.0, jump_w), (0.999999, 1 - jump_w)):
                        out, _ = orc.noise_apply(kind, p, t, psi, [draw])
                        rho += w * np.outer(out, out.conj())
                    k0 = np.array([[1, 0], [0, math.sqrt(1 - p)]])
                    k1 = np.array([[0, math.sqrt(p)], [0, 0]])
                    want = sum(dm.embed(k, t, n) @ np.outer(psi, psi.conj()) @ dm.embed(k, t, n).conj().T for k in (k0, k1))
                else:
                    branches = {0: [(0.99, 1 - p), (0.0, p)], 1: [(0.99, 1 - p), (0.0, p)],
                                2: [(0.99, 1 - 3 * p / 4), (0.0, p / 4), (p / 4 + 1e-9, p / 4), (p / 2 + 1e-9, p / 4)]}[kind]
                    for draw, w in branches:
                        out, _ = orc.noise_apply(kind, p, t, psi, [draw])
                        rho += w * np.outer(out, out.conj())
                    ops = {0: [(1 - p, np.eye(2)), (p, dm.single_matrix(dm.X))],
                           1: [(1 - p, np.eye(2)), (p, dm.single_matrix(dm.Z))],
                           2: [(1 - 3 * p / 4, np.eye(2)), (p / 4, dm.single_matrix(dm.X)),
                               (p / 4, dm.single_matrix(dm.Y)), (p / 4, dm.single_matrix(dm.Z))]}[kind]
                    want = sum(w * dm.embed(k, t, n) @ np.outer(psi, psi.conj()) @ dm.embed(k, t, n).conj().T for w, k in ops)
                assert np.max(np.abs(rho - want)) < 2e-12


def test_sampling_uses_the_strict_upper_bound_and_skips_zero_plateaus():
    """StateVectorSimulator.cs:68-90: a draw on an exact CDF boundary goes to the next supported index."""
    psi = np.array([math.sqrt(0.5), 0, 0, math.sqrt(0.5)], dtype=np.complex128)
    out = orc.sample(psi, [0.0, 0.25, 0.4999999, 0.5, 0.9999999])
    total = 0.5 + 0.5
    assert list(out) == [0, 0, 0, 3, 3]
    assert total == 1.0
    s, k = orc.measure_all(psi, 0.75)
    assert k == 3 and s[3] == 1 and np.sum(np.abs(s)) == 1


def test_seeded_random_stand_in_is_deterministic_and_in_range():
    a, b = orc.DotNetRandom(42), orc.DotNetRandom(42)
    xs = [a.NextDouble() for _ in range(2000)]
    assert xs == [b.NextDouble() for _ in range(2000)]
    assert min(xs) >= 0 and max(xs) < 1 and 0.45 < sum(xs) / len(xs) < 0.55
    assert xs != [orc.DotNetRandom(43).NextDouble() for _ in range(2000)]
