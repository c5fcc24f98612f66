"""Compiled passes run on the CPU (tests/jit_emulator.*) against the oracle.

The generated source of every pass of a plan is built with g++ and run as C++, chained as the
library chains it, so the deferred-phase algebra (rotations between pending phases, phases
rewritten by X, CNOT and SWAP, resolved before controlled ops and Toffolis, carried across
passes and flushed by the last one) is checked here without a GPU, on circuits that reach each
of those paths.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import jit_emulator as je
import oracle as orc
from circuits import random_circuit, random_state
from quantummatter_b200.algorithms import QuantumFourierTransform
from quantummatter_b200.backend import FP32, FP64
from quantummatter_b200.circuit import QuantumCircuit, u3
from quantummatter_b200.workloads import SplitMix64, brick_circuit
from test_abi import diagonal_heavy_circuit

pytestmark = pytest.mark.skipif(not je.available(), reason="g++ not found")


def frame_mix(n: int, layers: int, seed: int) -> QuantumCircuit:
    """U3 layers with X, CNOT (register and thread controls), SWAP, CZ, Ry and H in between:
    pending phases get conjugated, moved between sets and resolved."""
    rng = SplitMix64(seed)
    c = QuantumCircuit(n)
    for layer in range(layers):
        for q in range(n):
            c.U(q, u3(rng.uniform(0, 6.3), rng.uniform(0, 6.3), rng.uniform(0, 6.3)))
        c.X(layer % n).CNot((layer + 3) % n, (layer + 1) % n).Swap(layer % n, (layer + 5) % n)
        c.CZ(1, n - 2).Ry((layer + 2) % n, rng.uniform(0, 6.3)).H((layer + 4) % n)
        if n > 3:
            c.Toffoli(0, 1, n - 1)
        for q in range(layer % 2, n - 1, 2):
            c.CNot(q, q + 1)
    return c


CASES = [
    ("brick_fp64", lambda: brick_circuit(14, 10, seed=8), FP64, 1e-12),
    ("brick_fp32", lambda: brick_circuit(14, 10, seed=9), FP32, 2e-5),
    ("frame_mix", lambda: frame_mix(13, 5, 11), FP64, 1e-12),
    ("random_relabeled_fp64", lambda: random_circuit(14, 400, seed=14), FP64, 1e-12),
    ("random_relabeled_fp32", lambda: random_circuit(14, 400, seed=14), FP32, 2e-5),
    ("random", lambda: random_circuit(12, 250, seed=21), FP64, 1e-12),
    ("diagonal", lambda: diagonal_heavy_circuit(12, 250, seed=22), FP64, 1e-12),
    ("qft", lambda: QuantumFourierTransform.CreateCircuit(13), FP64, 1e-12),
]


@pytest.mark.parametrize("precision,width,tol", [(FP64, 9, 1e-12), (FP32, 13, 2e-5)], ids=["fp64-k9", "fp32-k13"])
def test_relabeling_passes_at_other_block_widths(precision, width, tol):
    """Generated kernels of relabeling plans with 9-qubit blocks (32 threads) and 13-qubit blocks
    (512 threads, complex64 only): lane codes and permuted stores at both ends of the range."""
    from quantummatter_b200.circuit import prepare
    from plan_emulator import program
    c = random_circuit(16, 400, seed=16)
    g, n = prepare(c)
    passes, ops, _ = program(16, precision, g, n, width)
    assert any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
    assert any(o.code == 0 and o.reserved for o in ops)
    psi = random_state(16, 2)
    want = orc.execute(c, psi)
    got = je.run_plan(c, precision, psi, width)
    assert np.max(np.abs(got - want)) <= tol


def test_cases_reach_relabeling_passes():
    """The relabeled cases plan passes that write qubits to other index bits (pending phases are
    carried through the relabeling) and stages that set the store lanes: the planner keeps
    relabeling there because it saves passes."""
    from quantummatter_b200.circuit import prepare
    from plan_emulator import program
    for make, precision in ((lambda: random_circuit(14, 400, seed=14), FP64),
                            (lambda: random_circuit(14, 400, seed=14), FP32)):
        c = make()
        g, n = prepare(c)
        passes, ops, _ = program(c.QubitCount, precision, g, n, 0)
        assert any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
        assert any(o.code == 0 and o.reserved for o in ops)


@pytest.mark.parametrize("name,make,precision,tol", CASES, ids=[c[0] for c in CASES])
def test_compiled_passes_on_the_cpu_match_the_oracle(name, make, precision, tol):
    c = make()
    psi = random_state(c.QubitCount, 3)
    want = orc.execute(c, psi)
    got = je.run_plan(c, precision, psi)
    assert np.max(np.abs(got - want)) <= tol
    assert abs(np.linalg.norm(got) - math.sqrt(np.vdot(psi, psi).real)) <= 100 * tol


PIPELINED = [
    ("fp64_two_teams", FP64, "1", 1, 1e-12),
    ("fp64_two_teams_idle_team", FP64, "1", 3, 1e-12),
    ("fp64_one_team", FP64, "0", 2, 1e-12),
    ("fp32_second_tile", FP32, "1", 3, 2e-5),
]


@pytest.mark.timeout(600)
@pytest.mark.parametrize("name,precision,teams,grid,tol", PIPELINED, ids=[c[0] for c in PIPELINED])
def test_pipelined_passes_on_the_cpu_match_the_oracle(monkeypatch, name, precision, teams, grid, tol):
    """The forms of states of 26 qubits and more, generated here for 14 qubits (QM_PIPE_QUBITS):
    the next tile copied during the current item, and for complex128 the block as two teams that
    hand a compute token back and forth by named barriers.  With 3 blocks over 4 work items, two
    blocks' team 1 has no item and must still pass the token on; a protocol whose arrivals do not
    match hangs here (the timeout) rather than on a GPU."""
    monkeypatch.setenv("QM_PIPE_QUBITS", "12")
    monkeypatch.setenv("QM_TEAMS", teams)
    c = brick_circuit(14, 12, seed=31)
    from quantummatter_b200.circuit import prepare
    g, n = prepare(c)
    src = je._text(je.load().qm_jit_source, 14, precision, g, n, 0, 0).decode()
    assert "qm_cp" in src
    assert ("const u32 team = threadIdx.x >>" in src) == (precision == FP64 and teams == "1")
    psi = random_state(14, 4)
    want = orc.execute(c, psi)
    got = je.run_plan(c, precision, psi, grid=grid)
    assert np.max(np.abs(got - want)) <= tol


@pytest.mark.timeout(900)
def test_twenty_qubit_brick_plan_on_the_cpu_matches_the_oracle():
    """The benchmark circuit's structure at 20 qubits: eight qubits outside every block, relabeling
    passes, the CNOTs planned as CZs with their signs deferred, rotations whose phase is chosen at
    run time by thread and work-item parities (in the shear form), phases carried across passes."""
    from quantummatter_b200.circuit import prepare
    from plan_emulator import program
    c = brick_circuit(20, 20, seed=12)
    g, n = prepare(c)
    passes, ops, _ = program(20, FP64, g, n, 0)
    assert any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
    assert sum(o.code == 5 for o in ops) > sum(o.code == 3 for o in ops)  # CZs, few CNOTs left
    src = je._text(je.load().qm_jit_source, 20, FP64, g, n, 0, 1).decode()
    assert "2 * (k" in src and "const double pu" in src
    psi = random_state(20, 6)
    want = orc.execute(c, psi)
    got = je.run_plan(c, FP64, psi)
    assert np.max(np.abs(got - want)) <= 1e-12
