"""ctypes binding of libqmb200.so (the C ABI of include/qm_b200.h).

The binding loads the in-tree shared object and fails loudly when it is missing: there
is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

from .errors import raise_for_status

# QM_B200_LIBRARY selects another build of the same ABI (e.g. one compiled with other
# register-blocking parameters); by default the in-tree library is used.
LIB_PATH = Path(os.environ.get("QM_B200_LIBRARY") or Path(__file__).resolve().parent / "libqmb200.so")

# ---------------------------------------------------------------- structs (layouts of qm_b200.h)


class Operation(C.Structure):
    _fields_ = [("kind", C.c_int32), ("target", C.c_int32), ("control", C.c_int32),
                ("second_control", C.c_int32), ("angle", C.c_double), ("unitary", C.c_double * 8)]


class Gate(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("target", C.c_int32), ("control_mask", C.c_uint32),
                ("swap_control", C.c_int32), ("a", C.c_double * 2), ("b", C.c_double * 2),
                ("c", C.c_double * 2), ("d", C.c_double * 2)]


class Options(C.Structure):
    _fields_ = [("device_index", C.c_int32), ("enable_profiling", C.c_int32),
                ("device_budget_bytes", C.c_int64), ("staging_budget_bytes", C.c_int64),
                ("fusion_width", C.c_int32), ("reserved", C.c_int32 * 7)]


class Profile(C.Structure):
    _fields_ = [("device_seconds", C.c_double), ("transfer_seconds", C.c_double),
                ("state_bytes", C.c_int64), ("kernel_launches", C.c_int32), ("passes", C.c_int32),
                ("planned_bytes", C.c_int64)]


class DeviceInfo(C.Structure):
    _fields_ = [("index", C.c_int32), ("sm_count", C.c_int32), ("major", C.c_int32), ("minor", C.c_int32),
                ("driver_version", C.c_int32), ("reserved", C.c_int32), ("memory_bytes", C.c_int64),
                ("name", C.c_char * 256)]


class PauliTermC(C.Structure):
    _fields_ = [("flip_mask", C.c_uint32), ("sign_mask", C.c_uint32), ("y_count", C.c_int32),
                ("reserved", C.c_int32), ("coefficient", C.c_double)]


class FusedPassInfo(C.Structure):
    _fields_ = [("block_qubits", C.c_int32), ("op_begin", C.c_int32), ("op_count", C.c_int32),
                ("qubits", C.c_int32 * 14), ("block_mask", C.c_uint32), ("stages", C.c_int32),
                ("reg_in", C.c_int8 * 4), ("reg_out", C.c_int8 * 4), ("qubits_out", C.c_int8 * 16),
                ("out_bit", C.c_int8 * 16)]


class FusedOpInfo(C.Structure):
    _fields_ = [("code", C.c_uint8), ("reg", C.c_int8), ("reg2", C.c_int8), ("local", C.c_int8),
                ("reg_pos", C.c_int8 * 4), ("cmask_local", C.c_uint16), ("flags", C.c_uint16),
                ("cmask_outer", C.c_uint32), ("target_outer", C.c_uint32), ("reserved", C.c_uint32),
                ("coef", C.c_double * 8)]


class TemplateOp(C.Structure):
    _fields_ = [("operation", Operation), ("parameter", C.c_int32), ("reserved", C.c_int32)]


class VqeStats(C.Structure):
    _fields_ = [("circuits", C.c_int64), ("waves", C.c_int32), ("batch_states", C.c_int32),
                ("passes_per_circuit", C.c_int32), ("tile_passes", C.c_int32), ("device_seconds", C.c_double),
                ("wall_seconds", C.c_double)]


class ChannelC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("target", C.c_int32), ("probability", C.c_double),
                ("position", C.c_int32), ("reserved", C.c_int32)]


class TrajectoryOutputs(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_double)), ("masses", C.POINTER(C.c_double)),
                ("consumed", C.POINTER(C.c_int32)), ("branches", C.POINTER(C.c_int8)),
                ("ambiguous", C.POINTER(C.c_int32)), ("outcomes", C.POINTER(C.c_int64)),
                ("probability_means", C.POINTER(C.c_double)), ("probability_stderr", C.POINTER(C.c_double))]


class VqeProblem(C.Structure):
    _fields_ = [("qubits", C.c_int32), ("precision", C.c_int32), ("operations", C.c_void_p),
                ("operation_count", C.c_int32), ("parameter_count", C.c_int32), ("terms", C.c_void_p),
                ("term_count", C.c_int32), ("vectors", C.c_int32), ("coefficients", C.POINTER(C.c_double)),
                ("parameters", C.POINTER(C.c_double)), ("with_gradient", C.c_int32), ("reserved", C.c_int32),
                ("energies", C.POINTER(C.c_double)), ("gradients", C.POINTER(C.c_double))]


class ServeOptions(C.Structure):
    _fields_ = [("device_index", C.c_int32), ("workers", C.c_int32), ("budget_bytes", C.c_int64),
                ("context_budget_bytes", C.c_int64), ("cache_bytes", C.c_int64), ("max_batch", C.c_int32),
                ("reserved", C.c_int32 * 5)]


class ServeResult(C.Structure):
    _fields_ = [("kind", C.c_int32), ("status", C.c_int32), ("batch", C.c_int32), ("ambiguous", C.c_int32),
                ("values", C.c_int32), ("outcomes", C.c_int32), ("parameters", C.c_int32), ("reserved", C.c_int32),
                ("mass", C.c_double), ("energy", C.c_double), ("submitted", C.c_double), ("started", C.c_double),
                ("finished", C.c_double)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("jobs", C.c_int64), ("vqe_jobs", C.c_int64),
                ("vqe_steps", C.c_int64), ("budget_bytes", C.c_int64), ("reserved_bytes", C.c_int64),
                ("peak_reserved_bytes", C.c_int64), ("queued", C.c_int32), ("running", C.c_int32),
                ("max_batch", C.c_int32), ("reserved", C.c_int32)]


class TrajectoryStats(C.Structure):
    _fields_ = [("segments", C.c_int32), ("passes", C.c_int32), ("mass_passes", C.c_int32),
                ("waves", C.c_int32), ("batch_states", C.c_int32), ("reserved", C.c_int32),
                ("device_seconds", C.c_double), ("wall_seconds", C.c_double)]


NEXT_DOUBLE_FN = C.CFUNCTYPE(C.c_double, C.c_void_p)

NOALLOC_MAX_TERMS = 64  # QM_NOALLOC_MAX_TERMS

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
DP = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)
I32P = C.POINTER(C.c_int32)

# name: (restype, argtypes) for every entry point of include/qm_b200.h
SIGNATURES = {
    "qm_abi_version": (I32, []),
    "qm_last_error": (I32, [C.c_char_p, C.c_size_t]),
    "qm_options_default": (None, [C.POINTER(Options)]),
    "qm_device_count": (I32, [I32P]),
    "qm_device_info_get": (I32, [I32, C.POINTER(DeviceInfo)]),
    "qm_context_create": (I32, [C.POINTER(Options), C.POINTER(P)]),
    "qm_context_destroy": (I32, [P]),
    "qm_host_alloc": (I32, [P, I64, C.POINTER(P)]),
    "qm_host_free": (I32, [P, P]),
    "qm_prepare_gates": (I32, [C.POINTER(Operation), I32, I32, C.POINTER(Gate)]),
    "qm_execute_host": (I32, [P, I32, C.POINTER(Operation), I32, P, I64, I32P, C.POINTER(Profile)]),
    "qm_noise_apply_host": (I32, [P, I32, C.c_double, I32, P, I64, NEXT_DOUBLE_FN, P, I32P]),
    "qm_state_create": (I32, [P, I32, I32, C.POINTER(P)]),
    "qm_state_destroy": (I32, [P]),
    "qm_state_reset": (I32, [P]),
    "qm_state_upload": (I32, [P, P, I64]),
    "qm_state_download": (I32, [P, P, I64]),
    "qm_state_device_pointer": (I32, [P, C.POINTER(P)]),
    "qm_execute": (I32, [P, C.POINTER(Gate), I32, I32, C.POINTER(Profile)]),
    "qm_plan_create": (I32, [P, I32, I32, C.POINTER(Gate), I32, I32, C.POINTER(P)]),
    "qm_plan_execute": (I32, [P, P, C.POINTER(Profile)]),
    "qm_plan_stats": (I32, [P, I32P, I32P, I64P]),
    "qm_plan_destroy": (I32, [P]),
    "qm_plan_autotune": (I32, [P, I32, I32, P, I32, I32P, I32, C.POINTER(P), I32P]),
    "qm_vqe_evaluate_mixed": (I32, [P, C.POINTER(VqeProblem), I32, C.POINTER(VqeStats)]),
    "qm_serve_create": (I32, [C.POINTER(ServeOptions), C.POINTER(P)]),
    "qm_serve_destroy": (I32, [P]),
    "qm_serve_submit_expectation": (I32, [P, I32, I32, P, I32, P, I32, I64P]),
    "qm_serve_submit_shots": (I32, [P, I32, I32, P, I32, DP, I32, I64P]),
    "qm_serve_session_create": (I32, [P, I32, I32, P, I32, I32, P, I32, DP, C.c_double, I64P]),
    "qm_serve_session_parameters": (I32, [P, I64, DP, I32, I64P]),
    "qm_serve_session_destroy": (I32, [P, I64]),
    "qm_serve_submit_vqe_step": (I32, [P, I64, I64P]),
    "qm_serve_wait": (I32, [P, I64, C.c_double, I32P]),
    "qm_serve_take_result": (I32, [P, I64, C.POINTER(ServeResult), DP, I32, C.POINTER(C.c_int64), I32, DP, I32]),
    "qm_serve_get_stats": (I32, [P, C.POINTER(ServeStats)]),
    "qm_graph_create": (I32, [P, P, C.POINTER(P)]),
    "qm_graph_launch": (I32, [P, C.POINTER(Profile)]),
    "qm_graph_destroy": (I32, [P]),
    "qm_plan_program": (I32, [I32, I32, C.POINTER(Gate), I32, I32, I32P, C.POINTER(FusedPassInfo), I32, I32P,
                              C.POINTER(FusedOpInfo), I32, I64P]),
    "qm_qubit_masses": (I32, [P, I32, DP, DP]),
    "qm_apply_pauli": (I32, [P, I32, I32]),
    "qm_apply_damping": (I32, [P, I32, I32, C.c_double, C.c_double, C.c_double]),
    "qm_expectation_pauli": (I32, [P, C.POINTER(PauliTermC), I32, DP, DP]),
    "qm_expectation_energy": (I32, [P, C.POINTER(PauliTermC), I32, DP]),
    "qm_measure_all": (I32, [P, C.c_double, I64P, I32P]),
    "qm_sample": (I32, [P, DP, I32, I64P, I32P]),
    "qm_batch_create": (I32, [P, I32, I32, I32, C.POINTER(P)]),
    "qm_batch_destroy": (I32, [P]),
    "qm_batch_reset": (I32, [P, I32]),
    "qm_batch_state": (I32, [P, I32, P, I64, I32]),
    "qm_batch_execute": (I32, [P, I32, C.POINTER(Gate), I32P, I32, DP, I32, I32]),
    "qm_batch_expectation": (I32, [P, I32, C.POINTER(PauliTermC), I32, DP, DP]),
    "qm_vqe_evaluate": (I32, [P, I32, I32, C.POINTER(TemplateOp), I32, I32, C.POINTER(PauliTermC), I32, DP, I32, I32,
                              DP, DP, C.POINTER(VqeStats)]),
    "qm_marginal_probability": (I32, [P, I32P, I32, I32, DP]),
    "qm_measure": (I32, [P, I32P, I32, C.c_double, I32P, I32P]),
    "qm_jit_info": (I32, [I32P, I64P, I64P, I64P]),
    "qm_dense_info": (I32, [I64P, I64P]),
    "qm_jit_source": (I32, [I32, I32, C.POINTER(Gate), I32, I32, I32, C.c_char_p, C.c_size_t,
                            C.POINTER(C.c_size_t)]),
    "qm_jit_constants": (I32, [I32, I32, C.POINTER(Gate), I32, I32, I32, C.c_void_p, C.c_size_t,
                               C.POINTER(C.c_size_t)]),
    "qm_state_noise_apply": (I32, [P, I32, C.c_double, I32, NEXT_DOUBLE_FN, P]),
    "qm_jit_expect_source": (I32, [I32, I32, C.POINTER(PauliTermC), I32, I32, C.c_char_p, C.c_size_t,
                                   C.POINTER(C.c_size_t)]),
    "qm_vqe_evaluate_coefficients": (I32, [P, I32, I32, C.POINTER(TemplateOp), I32, I32, C.POINTER(PauliTermC), I32,
                                           DP, DP, I32, I32, DP, DP, C.POINTER(VqeStats)]),
    "qm_trajectories_run": (I32, [P, I32, I32, C.POINTER(Gate), I32, C.POINTER(ChannelC), I32, I32, DP, I32,
                                  C.POINTER(PauliTermC), I32, C.POINTER(TrajectoryOutputs),
                                  C.POINTER(TrajectoryStats)]),
    "qm_random_doubles": (I32, [I32, I64, I64, DP]),
    "qm_expectation_pauli_noalloc": (I32, [P, I32, I32, C.POINTER(PauliTermC), I32, DP, DP, P]),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None


def load() -> C.CDLL:
    """Loads libqmb200.so; raises OSError when it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m quantummatter_b200.build` "
                          "(the CUDA library has no fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().qm_last_error(buf, len(buf))
    return buf.value.decode("utf-8", "replace")


def check(status: int) -> None:
    """Raises the exception that mirrors a nonzero qm_status."""
    if status != 0:
        raise_for_status(status, last_error())
