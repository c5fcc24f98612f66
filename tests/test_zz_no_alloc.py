"""qm_expectation_pauli_noalloc against qm_expectation_pauli, through the C ABI.

The allocation-free entry point reads a caller-owned device state and keeps its reduction
scratch in a fixed device array; it must give the same per-term values and mass as the
allocating entry point on the same state, call after call.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from quantummatter_b200 import _lib
from quantummatter_b200._lib import check, load
from quantummatter_b200.backend import FP32, FP64, DeviceState
from quantummatter_b200.observables import PauliString, observable_array
from quantummatter_b200.workloads import brick_circuit

TOL = 1e-12  # both paths accumulate in FP64; only the summation order differs
QM_E_RANGE = 10


def labels_for(n: int, seed: int, count: int) -> list[str]:
    """Random Pauli labels plus long runs sharing one flip mask (more than one group's worth)."""
    rng = np.random.default_rng(seed)
    out = ["I" * n, "Z" * n]
    while len(out) < count - 12:
        out.append("".join(rng.choice(list("IXYZ"), size=n)))
    for i in range(12):  # same X/Y positions, different Z/Y split: one flip mask
        lab = ["X" if (q + i) % 3 == 0 else ("Z" if (q * 7 + i) % 2 else "I") for q in range(n)]
        out.append("".join(lab))
    return out[:count]


def noalloc(state: DeviceState, observables: list[PauliString]) -> tuple[np.ndarray, float]:
    arr, n = observable_array(observables)
    out = np.full(max(1, n), np.nan)
    mass = C.c_double(np.nan)
    check(load().qm_expectation_pauli_noalloc(C.c_void_p(state.device_pointer()), state.QubitCount, state.precision,
                                               arr, n, out.ctypes.data_as(_lib.DP), C.byref(mass), None))
    return out[:n], mass.value


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [FP64, FP32])
@pytest.mark.parametrize("qubits", [3, 12, 20])
def test_noalloc_matches_the_allocating_entry_point(gpu_context, precision, qubits):
    obs = [PauliString(lab) for lab in labels_for(qubits, 100 + qubits, 64)]
    circuit = brick_circuit(qubits, 6, seed=qubits)
    with DeviceState(gpu_context, qubits, precision) as st:
        st.Evolve(circuit)
        want, want_mass = st.ExpectationValues(obs)
        first, first_mass = noalloc(st, obs)
        second, second_mass = noalloc(st, obs)
    assert abs(first_mass - want_mass) <= TOL * want_mass
    assert np.max(np.abs(first - want)) <= TOL
    # two calls in a row on the same scratch give the same sums
    assert second_mass == first_mass
    assert np.array_equal(second, first)


@pytest.mark.gpu
def test_noalloc_reserves_no_device_memory(gpu_context):
    """After a warm-up call has loaded the modules, calls leave the device's free memory unchanged."""
    import torch
    n = 22
    obs = [PauliString(lab) for lab in labels_for(n, 7, 40)]
    with DeviceState(gpu_context, n, FP64) as st:
        st.Evolve(brick_circuit(n, 4, seed=3))
        noalloc(st, obs)
        free_before, _ = torch.cuda.mem_get_info(0)
        for _ in range(3):
            noalloc(st, obs)
        free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before


@pytest.mark.gpu
def test_noalloc_limits_and_mass_only(gpu_context):
    n = 10
    with DeviceState(gpu_context, n, FP64) as st:
        re, im = np.random.default_rng(5).standard_normal((2, 1 << n))
        psi = re + 1j * im
        st.Upload(psi)
        vals, mass = noalloc(st, [])
        assert vals.size == 0 and abs(mass - np.vdot(psi, psi).real) <= TOL * mass
        too_many = [PauliString("Z" + "I" * (n - 1))] * (_lib.NOALLOC_MAX_TERMS + 1)
        arr, count = observable_array(too_many)
        out = np.zeros(count)
        m = C.c_double()
        rc = load().qm_expectation_pauli_noalloc(C.c_void_p(st.device_pointer()), n, FP64, arr, count,
                                                 out.ctypes.data_as(_lib.DP), C.byref(m), None)
        assert rc == QM_E_RANGE
        buf = C.create_string_buffer(512)
        load().qm_last_error(buf, 512)
        assert b"at most" in buf.value
        # the largest accepted call still works after the rejection
        vals, mass2 = noalloc(st, too_many[:-1])
        want, _ = st.ExpectationValues(too_many[:-1])
        assert np.max(np.abs(vals - want)) <= TOL and abs(mass2 - mass) <= TOL * mass
