"""The C-ABI library on the CPU: it loads, exports every declared entry point, keeps the
struct layouts of include/qm_b200.h, prepares gates exactly as the oracle does, and its
fusion planner produces programs that the CPU emulator runs to the oracle's result."""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

import oracle as orc
import plan_emulator as pe
from circuits import random_circuit, random_state
from conftest import ROOT
from quantummatter_b200 import _lib
from quantummatter_b200.circuit import QuantumCircuit, prepare
from quantummatter_b200.errors import ArgumentError, ArgumentOutOfRangeError, NotSupportedError
from quantummatter_b200.workloads import brick_circuit

HEADER = ROOT / "include" / "qm_b200.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(qm_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_entry_point():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert names == set(_lib.SIGNATURES), "the ctypes binding covers exactly the header"
    assert lib.qm_abi_version() == 2
    limit = re.search(r"#define QM_NOALLOC_MAX_TERMS (\d+)", HEADER.read_text())
    assert limit and int(limit.group(1)) == _lib.NOALLOC_MAX_TERMS


def test_shipped_abi_inventory_matches_the_header():
    """include/qm_b200.shipped.txt is the shipped surface (prototypes, struct fields, defines),
    as PublicAPI.Shipped.txt is for the reference's assemblies: changing the header without it
    fails here.  Regenerate with `python include/shipped_abi.py --write` and, for a change that
    breaks callers, raise QM_ABI_VERSION."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("shipped_abi", ROOT / "include" / "shipped_abi.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    want = (ROOT / "include" / "qm_b200.shipped.txt").read_text().splitlines()
    got = mod.inventory(HEADER.read_text())
    added, removed = sorted(set(got) - set(want)), sorted(set(want) - set(got))
    assert not added and not removed, {"not in the inventory": added, "gone from the header": removed}
    functions = {re.search(r"\b(qm_\w+)\(", line).group(1) for line in got if line.startswith("function ")}
    assert functions == declared_symbols()


def test_struct_layouts_match_the_header():
    assert C.sizeof(_lib.Operation) == 88
    assert C.sizeof(_lib.Gate) == 80
    assert C.sizeof(_lib.PauliTermC) == 24
    assert C.sizeof(_lib.FusedOpInfo) == 88
    assert C.sizeof(_lib.FusedPassInfo) == 116
    assert C.sizeof(_lib.Options) == 56


def test_prepared_gates_equal_the_oracle_bit_for_bit():
    """qm_prepare_gates restates PreparedStateVectorGate.Prepare with the host libm."""
    for seed in range(8):
        c = random_circuit(6, 200, seed=seed)
        got, n = prepare(c)
        want = orc.prepare(c)
        assert C.string_at(C.addressof(got), n * 80) == C.string_at(C.addressof(want), n * 80)


def test_prepare_validates_like_the_circuit_builders():
    lib = _lib.load()
    ops = (_lib.Operation * 1)()
    gates = (_lib.Gate * 1)()
    ops[0].kind, ops[0].target, ops[0].control, ops[0].second_control = 9, 1, 1, -1
    with pytest.raises(ArgumentError):
        _lib.check(lib.qm_prepare_gates(ops, 1, 2, gates))
    ops[0].control = 5
    with pytest.raises(ArgumentOutOfRangeError):
        _lib.check(lib.qm_prepare_gates(ops, 1, 2, gates))
    ops[0].kind, ops[0].control = 42, -1
    with pytest.raises(NotSupportedError):
        _lib.check(lib.qm_prepare_gates(ops, 1, 2, gates))
    ops[0].kind, ops[0].angle = 6, float("nan")
    with pytest.raises(ArgumentOutOfRangeError):
        _lib.check(lib.qm_prepare_gates(ops, 1, 2, gates))


def _emulate_against_oracle(circuit: QuantumCircuit, width: int, precision: int = 0, seed: int = 0) -> int:
    n = circuit.QubitCount
    gates, count = prepare(circuit)
    passes, ops, planned = pe.program(n, precision, gates, count, width)
    psi = random_state(n, seed)
    got = pe.emulate(psi, n, passes, ops)
    want = orc.execute(circuit, psi)
    assert np.max(np.abs(got - want)) <= 1e-12
    return len(passes)


@pytest.mark.parametrize("width", [9, 10])
def test_planner_programs_reproduce_the_oracle_on_random_circuits(width):
    for seed in range(4):
        c = random_circuit(12, 160, seed=200 + seed)
        _emulate_against_oracle(c, width, seed=seed)


def test_planner_handles_controls_and_diagonals_outside_the_block():
    c = QuantumCircuit(12)
    for q in range(12):
        c.H(q)
    c.CZ(11, 0).CPhase(10, 11, 0.3).Toffoli(11, 10, 2).CRy(11, 1, 0.7).Rz(11, 1.1).Swap(0, 5)
    c.Controlled(c.Operations[0].Kind, 9, 3).Phase(10, -0.4).CNot(0, 11).Z(11).S(10).T(9)
    for q in range(12):
        c.Rx(q, 0.1 * q)
    _emulate_against_oracle(c, 9, seed=3)


def _layout_after(qubits: int, passes) -> list[int]:
    """The qubit held at each index bit after the passes (each writes local bit b to qubits_out[b])."""
    at = list(range(qubits))
    for p in passes:
        k = p.block_qubits
        held = {p.qubits[b]: at[p.qubits[b]] for b in range(k)}
        for b in range(k):
            at[p.qubits_out[b]] = held[p.qubits[b]]
    return at


@pytest.mark.parametrize("precision,low", [(0, 3), (1, 4)], ids=["fp64", "fp32"])
def test_relabeling_plans_restore_the_qubit_order(precision, low):
    """The 30-qubit brick of depth 40: passes follow the light cone by writing the qubits the
    next pass needs to the lowest index bits, and the last passes put every qubit back.  Every
    pass writes its tile to the bits it read; its store keeps the coalesced run (the lowest
    index bits) on the lowest thread ranks."""
    c = brick_circuit(30, 40)
    gates, count = prepare(c)
    passes, ops, planned = pe.program(30, precision, gates, count, 0)
    assert len(passes) <= (32 if precision == 0 else 36)  # 55 and 62 without relabeling
    assert planned == len(passes) * 2 * ((8 if precision == 1 else 16) << 30)
    assert _layout_after(30, passes) == list(range(30))
    relabeled = 0
    for p in passes:
        k = p.block_qubits
        q = [p.qubits[b] for b in range(k)]
        q_out = [p.qubits_out[b] for b in range(k)]
        assert sorted(q_out) == q and q[:low] == list(range(low))
        assert [p.out_bit[r] for r in range(low)] == list(range(low))
        # a stage's barriers order the stores of one thread after the loads of every other
        assert q_out == q or any(o.code == 0 for o in ops[p.op_begin:p.op_begin + p.op_count])
        relabeled += q_out != q
    assert relabeled >= len(passes) // 2


def test_relabeling_is_kept_only_where_it_saves_passes():
    """A 14-qubit brick of depth 10 needs 3 passes either way: it keeps the plain plan (no lane
    stages, no restoring pass).  The 30-qubit brick of depth 40 keeps its relabeling plan, and a
    subprocess with QM_RELABEL=0 shows the plain plan it replaced."""
    import json
    import os
    import subprocess
    import sys

    def counts(c, precision=0):
        gates, count = prepare(c)
        passes, ops, _ = pe.program(c.QubitCount, precision, gates, count, 0)
        relabels = any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
        return len(passes), relabels

    assert counts(brick_circuit(14, 10, seed=8)) == (3, False)
    relabeled, relabels = counts(brick_circuit(30, 40))
    assert relabels
    script = ("import json, sys; sys.path[:0] = ['tests', 'oracle']; import plan_emulator as pe; "
              "from quantummatter_b200.circuit import prepare; from quantummatter_b200.workloads import brick_circuit; "
              "g, n = prepare(brick_circuit(30, 40)); print(json.dumps(len(pe.program(30, 0, g, n, 0)[0])))")
    out = subprocess.run([sys.executable, "-c", script], cwd=ROOT, capture_output=True, text=True, timeout=300,
                         env={**os.environ, "QM_RELABEL": "0"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert relabeled < json.loads(out.stdout.strip().splitlines()[-1])


def _lowest_ranks(registers, lanes, k, n):
    free = [b for b in range(k) if b not in registers and b not in lanes]
    return (list(lanes) + free)[:n]


@pytest.mark.parametrize("precision,low,allowed", [(0, 3, 0.02), (1, 4, 0.1)], ids=["fp64", "fp32"])
def test_exchanges_keep_shared_memory_free_of_bank_conflicts(precision, low, allowed):
    """An exchange goes through shared memory in phases of 2^low threads (ranks 0..low-1) and the
    swizzle sends local bit p to bank-group bit p mod low: nearly every exchange side but a
    relabeling pass's final lanes (fixed by the store) holds bits of distinct classes on those
    ranks (stages may lack a class among their free bits: 2 of 209 complex128 sides of the brick
    once its CNOTs plan as CZs)."""
    c = brick_circuit(30, 40)
    gates, count = prepare(c)
    passes, ops, _ = pe.program(30, precision, gates, count, 0)
    sides = colliding = 0
    for p in passes:
        k = p.block_qubits
        registers, lanes = list(p.reg_in), []
        stages = [o for o in ops[p.op_begin:p.op_begin + p.op_count] if o.code == 0]
        for i, o in enumerate(stages):
            new_lanes = [(o.reserved >> (4 + 4 * r)) & 15 for r in range(o.reserved & 15)]
            checked = [(registers, lanes)]
            if i < len(stages) - 1:  # the last stage's read side holds the store's ranks
                checked.append((list(o.reg_pos), new_lanes))
            for regs, ln in checked:
                ranks = _lowest_ranks(regs, ln, k, low)
                sides += 1
                colliding += len({b % low for b in ranks}) < low
            registers, lanes = list(o.reg_pos), new_lanes
    assert sides > 100 and colliding <= allowed * sides, (colliding, sides)


@pytest.mark.parametrize("precision,width", [(0, 9), (0, 10), (0, 11), (1, 9), (1, 11), (1, 13)])
def test_relabeling_plans_match_the_oracle_at_every_block_width(precision, width):
    """Explicit fusion widths plan relabeling passes too (lanes of 3 bits in FP64, 4 in FP32); this
    circuit needs fewer passes with them at every width, so the planner keeps them."""
    c = random_circuit(16, 400, seed=16)
    gates, count = prepare(c)
    passes, ops, _ = pe.program(16, precision, gates, count, width)
    assert all(p.block_qubits == width for p in passes)
    assert any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
    psi = random_state(16, 1)
    got = pe.emulate(psi, 16, passes, ops)
    assert np.max(np.abs(got - orc.execute(c, psi))) <= 1e-12


def test_relabeling_plan_matches_the_oracle_when_emulated():
    c = random_circuit(18, 400, seed=18)  # X, CNOT, SWAP, controlled gates, Toffolis
    gates, count = prepare(c)
    passes, ops, _ = pe.program(18, 0, gates, count, 0)
    assert any(p.qubits_out[b] != p.qubits[b] for p in passes for b in range(p.block_qubits))
    psi = random_state(18, 4)
    got = pe.emulate(psi, 18, passes, ops)
    assert np.max(np.abs(got - orc.execute(c, psi))) <= 1e-12


def test_planner_brick_circuit_pass_counts_and_bytes():
    c = brick_circuit(16, 8, seed=11)
    gates, count = prepare(c)
    passes, ops, planned = pe.program(16, 0, gates, count, 12)
    assert planned == len(passes) * 2 * (16 << 16)
    assert len(passes) < count / 8, "fusion must cut launches by an order of magnitude"
    psi = random_state(16, 5)
    got = pe.emulate(psi, 16, passes, ops)
    assert np.max(np.abs(got - orc.execute(c, psi))) <= 1e-12


def diagonal_heavy_circuit(qubits: int, gates: int, seed: int) -> QuantumCircuit:
    """Mostly commuting diagonals (phases, CZ, Z) between a few rotations and CNOTs: exercises the
    planner's diagonal groups, including controlled phases that stay outside the groups."""
    rng = np.random.default_rng(seed)
    c = QuantumCircuit(qubits)
    for _ in range(gates):
        q = int(rng.integers(qubits))
        o = (q + 1 + int(rng.integers(qubits - 1))) % qubits
        r = rng.random()
        if r < 0.2:
            c.Rz(q, float(rng.uniform(-3, 3)))
        elif r < 0.3:
            c.Phase(q, float(rng.uniform(-3, 3)))
        elif r < 0.4:
            (c.S, c.T, c.Z, c.Sdg)[int(rng.integers(4))](q)
        elif r < 0.6:
            c.CZ(q, o)
        elif r < 0.67:
            c.CPhase(q, o, float(rng.uniform(-3, 3)))
        elif r < 0.85:
            c.Ry(q, float(rng.uniform(-3, 3)))
        elif r < 0.93:
            c.H(q)
        else:
            c.CNot(q, o)
    return c


@pytest.mark.parametrize("width", [9, 11])
def test_planner_groups_commuting_diagonals(width):
    for seed in range(3):
        c = diagonal_heavy_circuit(12, 250, seed)
        gates, count = prepare(c)
        passes, ops, _ = pe.program(12, 0, gates, count, width)
        assert any(op.code == pe.OP_DIAG_GROUP for op in ops)
        psi = random_state(12, seed)
        assert np.max(np.abs(pe.emulate(psi, 12, passes, ops) - orc.execute(c, psi))) <= 1e-12


def test_per_gate_width_counts_one_launch_per_gate():
    c = brick_circuit(10, 3, seed=1)
    gates, count = prepare(c)
    np_, no, nbytes = C.c_int32(), C.c_int32(), C.c_int64()
    _lib.check(_lib.load().qm_plan_program(10, 0, gates, count, 1, C.byref(np_), None, 0, C.byref(no), None, 0,
                                           C.byref(nbytes)))
    assert np_.value == 0 and no.value == 0
    # 30 dense U3 (2S each) + 5 + 4 + 5 CNOT (S each), S = 16 * 2^10
    assert nbytes.value == 30 * 2 * (16 << 10) + 14 * (16 << 10)


def test_no_device_behaviour_on_a_cpu_host():
    """Without a GPU, device discovery returns an empty list and context creation reports
    PlatformNotSupported (CudaStateVectorBackend.cs:31-35)."""
    lib = _lib.load()
    n = C.c_int32(-1)
    assert lib.qm_device_count(C.byref(n)) == 0
    if n.value > 0:
        pytest.skip("a CUDA device is visible")
    o = _lib.Options()
    lib.qm_options_default(C.byref(o))
    h = C.c_void_p()
    assert lib.qm_context_create(C.byref(o), C.byref(h)) == 4
    assert "No compatible NVIDIA CUDA device" in _lib.last_error()


def test_cnots_between_single_qubit_matrices_plan_as_cz(monkeypatch):
    """CNOT(c, t) = H_t CZ(c, t) H_t: where the gates before and after a CNOT on its target are
    single-qubit matrices, the planner merges the Hadamards into them and plans a CZ, a diagonal
    that needs no register for t.  The 30-qubit brick then plans in 25 passes instead of 29 (566
    of its 580 CNOTs; the last layer's have no gate after them); QM_CZ_REWRITE=0 keeps the
    CNOTs.  The rewritten plans reproduce the oracle."""
    c = brick_circuit(30, 40)
    gates, count = prepare(c)

    def counts():
        passes, ops, _ = pe.program(30, 0, gates, count, 0)
        return len(passes), sum(o.code == 3 for o in ops), sum(o.code == 5 for o in ops)

    assert counts() == (25, 14, 566)
    monkeypatch.setenv("QM_CZ_REWRITE", "0")
    assert counts()[:2] == (29, 580)
    monkeypatch.delenv("QM_CZ_REWRITE")
    for seed in range(3):
        _emulate_against_oracle(brick_circuit(16, 12, seed=seed), 0, seed=seed)
        _emulate_against_oracle(random_circuit(14, 300, seed=40 + seed), 0, seed=seed)
