"""Parity at the benchmark sizes: the 30-qubit brick, the 18-22-qubit variational batch and the
24-qubit noise trajectories, on the GPU against the oracle or an oracle-checked device path.

- 30 qubits, FP64: the compiled relabeling plan (the timed headline path) against the per-gate
  path over the whole 2^30 vector (16 GiB each), and a two-layer prefix against the oracle's
  parallel restatement on the host.
- 30 qubits, FP32: the compiled plan against the FP64 result; the error is bounded and printed.
- Variational evaluator at 18, 20 and 22 qubits (hardware-efficient ansatz, XXZ chain): energies
  and a sample of gradient components of two parameter vectors against the oracle evaluator
  (VariationalEnergyEvaluator.cs:34-86 restated), FP64 to 5e-12 and FP32 to 1e-6.
- Noise trajectories at 24 qubits: four trajectories of RY layers and CZ ladders with every channel
  kind against the oracle's NoisyCircuit.Execute restatement on the same draws.

The 2^30 comparisons run on the device through zero-copy torch views of the library's buffers.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle as orc
import ref_variational as ref
from quantummatter_b200.backend import FP32, FP64, DeviceState, Plan, jit_info
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.workloads import brick_circuit, hardware_efficient_ansatz, uniform_parameters, xxz_chain

pytestmark = pytest.mark.gpu


class _DeviceBuffer:
    """A raw device allocation of the library exposed through __cuda_array_interface__."""

    def __init__(self, pointer: int, length: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (length,), "typestr": typestr, "data": (pointer, False),
                                         "version": 3, "strides": None}


def device_view(state: DeviceState):
    """The state's amplitudes as a flat real torch tensor on the GPU (re, im interleaved), no copy."""
    import torch
    length = 2 << state.QubitCount
    typestr = "<f8" if state.precision == FP64 else "<f4"
    return torch.as_tensor(_DeviceBuffer(state.device_pointer(), length, typestr), device="cuda")


def max_abs_diff(a: DeviceState, b: DeviceState, chunk: int = 1 << 27) -> float:
    """Largest |a_i - b_i| over the amplitudes (complex modulus), in FP64, chunk by chunk."""
    import torch
    va, vb = device_view(a), device_view(b)
    worst = 0.0
    for start in range(0, va.numel(), 2 * chunk):
        x = va[start:start + 2 * chunk].double().view(-1, 2)
        y = vb[start:start + 2 * chunk].double().view(-1, 2)
        d = torch.linalg.vector_norm(x - y, dim=1).max().item()
        worst = max(worst, d)
    torch.cuda.synchronize()
    return worst


def _compiled_plan(ctx, circuit, precision):
    before = jit_info()
    plan = Plan(ctx, circuit, precision)
    return plan, before


def test_30_qubit_compiled_plan_equals_the_per_gate_path(gpu_context):
    """The headline plan (relabeling passes, deferred phases carried across all of them, qubit
    order restored) against one launch per gate, over all 2^30 amplitudes."""
    c = brick_circuit(30, 40)
    plan, before = _compiled_plan(gpu_context, c, FP64)
    try:
        passes, _, _ = plan.stats()
        assert passes < 40
        with DeviceState(gpu_context, 30, FP64) as fused, DeviceState(gpu_context, 30, FP64) as per_gate:
            plan.execute(fused)
            per_gate.Evolve(c, fusion_width=1)
            diff = max_abs_diff(fused, per_gate)
    finally:
        plan.Dispose()
    after = jit_info()
    if before["available"]:
        assert after["failed"] == before["failed"] and after["launches"] > before["launches"]
    print(f"30q compiled plan vs per-gate path: max |d amp| = {diff:.3e}")
    assert diff <= 1e-12


def test_30_qubit_prefix_matches_the_oracle(gpu_context):
    """The first two layers of the 30-qubit brick (60 U3 + 29 CNOT) through a compiled plan and
    through the one-shot port, against the oracle's parallel/AVX-512 restatement on the host."""
    c = brick_circuit(30, 40)
    prefix = QuantumCircuit(30)
    for op in c.Operations[:89]:
        prefix.AppendValidated(op)
    want = orc.execute_parallel(prefix)
    plan = Plan(gpu_context, prefix, FP64)
    try:
        with DeviceState(gpu_context, 30, FP64) as st:
            plan.execute(st)
            got = st.Download()
            err_plan = float(np.max(np.abs(got - want)))
            del got
            st.Reset()
            st.Evolve(prefix)
            got = st.Download()
            err_port = float(np.max(np.abs(got - want)))
    finally:
        plan.Dispose()
    print(f"30q prefix: plan {err_plan:.3e}, one-shot {err_port:.3e}")
    assert err_plan <= 1e-12 and err_port <= 1e-12


def test_30_qubit_fp32_error_against_fp64(gpu_context):
    """The complex64 form of the headline circuit (its own relabeling plan) against the complex128
    result: every amplitude within 2e-6 (the typical amplitude is 2^-15 = 3e-5)."""
    c = brick_circuit(30, 40)
    p64, p32 = Plan(gpu_context, c, FP64), Plan(gpu_context, c, FP32)
    try:
        with DeviceState(gpu_context, 30, FP64) as a, DeviceState(gpu_context, 30, FP32) as b:
            p64.execute(a)
            p32.execute(b)
            diff = max_abs_diff(a, b)
            _, mass = b.ExpectationValues([])
    finally:
        p64.Dispose()
        p32.Dispose()
    print(f"30q FP32 vs FP64: max |d amp| = {diff:.3e}, FP32 mass - 1 = {mass - 1:.3e}")
    assert diff <= 2e-6
    assert abs(mass - 1) <= 1e-4


def _gradient_sample(circuit, hamiltonian, params, indices):
    """Oracle energy and the gradient components `indices` (parameter-shift, termwise differences,
    Neumaier per parameter), with the parallel restatement evolving each circuit."""
    params = list(params)
    terms = hamiltonian.Terms
    energy = orc.energy(orc.execute_parallel(circuit.Bind(params)), hamiltonian)
    occurrences = circuit.RotationParameterIndices
    grad = {}
    for p in indices:
        total, corr = 0.0, 0.0
        for r, q in enumerate(occurrences):
            if q != p:
                continue
            plus = orc.execute_parallel(circuit.BindWithRotationShift(params, r, math.pi / 2))
            minus = orc.execute_parallel(circuit.BindWithRotationShift(params, r, -math.pi / 2))
            for t in terms:
                a, b = orc.expectation(plus, t.Observable), orc.expectation(minus, t.Observable)
                total, corr = ref._neumaier(total, corr, t.Coefficient * (0.5 * a - 0.5 * b))
        grad[p] = total + corr
    return energy, grad


@pytest.mark.parametrize("qubits", [18, 20, 22])
def test_variational_batch_at_benchmark_sizes(gpu_context, qubits):
    """Hardware-efficient ansatz of 4 layers on an XXZ chain: two parameter vectors, energies and
    six gradient components each (first, last and four spread between), FP64 and FP32."""
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    c = hardware_efficient_ansatz(qubits, 4)
    h = xxz_chain(qubits, seed=qubits)
    params = uniform_parameters(c.ParameterCount, 2, -math.pi, math.pi, seed=100 + qubits)
    P = c.ParameterCount
    indices = sorted({0, P // 5, 2 * P // 5, 3 * P // 5, 4 * P // 5, P - 1})
    scale = max(1.0, sum(abs(t.Coefficient) for t in h.Terms))
    r64 = B200VariationalEnergyEvaluator(gpu_context, FP64).EvaluateBatch(c, h, params, withGradient=True)
    r32 = B200VariationalEnergyEvaluator(gpu_context, FP32).EvaluateBatch(c, h, params, withGradient=True)
    worst64, worst32 = 0.0, 0.0
    for v in range(2):
        e, g = _gradient_sample(c, h, params[v], indices)
        worst64 = max(worst64, abs(r64.Energies[v] - e), *(abs(r64.Gradients[v][p] - g[p]) for p in indices))
        worst32 = max(worst32, abs(r32.Energies[v] - e), *(abs(r32.Gradients[v][p] - g[p]) for p in indices))
    print(f"{qubits}q variational: FP64 worst {worst64:.3e}, FP32 worst {worst32:.3e} (scale {scale:.1f})")
    assert worst64 <= 5e-12 * scale
    assert worst32 <= 1e-6 * scale


def test_24_qubit_trajectories_match_the_oracle(gpu_context):
    """Four 24-qubit trajectories of the benchmark's structure (RY layers, CZ ladders, depolarizing
    after every gate, damping on every qubit per layer) with probabilities raised so that branches
    occur, FP64 and FP32, against the oracle on the same draws."""
    from quantummatter_b200.noise import NoiseChannel, NoisyCircuit
    from quantummatter_b200.trajectories import B200NoisySimulator
    from test_trajectories import oracle_rows, z_observables
    n, layers = 24, 4
    rng = np.random.default_rng(24)
    nc = NoisyCircuit(n)
    for _ in range(layers):
        ry = QuantumCircuit(n)
        for q in range(n):
            ry.Ry(q, float(rng.uniform(0, 2 * np.pi)))
        nc.Append(ry)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.Depolarizing(0.05), q)
        for q in range(n - 1):
            cz = QuantumCircuit(n)
            cz.CZ(q, q + 1)
            nc.Append(cz)
            nc.ApplyNoise(NoiseChannel.Depolarizing(0.1), q)
            nc.ApplyNoise(NoiseChannel.Depolarizing(0.1), q + 1)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.AmplitudeDamping(0.2), q)
    draws = np.random.default_rng(7).random((4, nc.MaxDraws()))
    obs = z_observables(n)
    values, masses, used, branches = oracle_rows(nc, draws, obs)
    for precision, tol in ((FP64, 1e-12), (FP32, 2e-5)):
        res = B200NoisySimulator(gpu_context, precision=precision).RunBatch(nc, draws, obs, branches=True)
        ok = res.ambiguous == 0
        if precision == FP64:
            assert ok.all()
        assert ok.sum() >= 3
        assert np.array_equal(res.consumed[ok], used[ok])
        assert np.array_equal(res.branches[ok], branches[ok])
        assert np.max(np.abs(res.values[ok] - values[ok])) <= tol
        assert np.max(np.abs(res.masses[ok] - masses[ok]) / masses[ok]) <= tol
    assert {0, 1, 2, 3} <= set(np.unique(branches).tolist())  # no p = 0 placement here, so no skips
