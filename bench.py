#!/usr/bin/env python3
"""Benchmark of the B200 state-vector engine on the 30-qubit random brick circuit.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32] [--width k]
    python bench.py --impl reference ...      # the reference's CPU path (parallel/AVX-512 port)

Workload: 30 qubits, depth 40, every layer U3(theta, phi, lambda) on all qubits (angles
uniform in [0, 2pi) from a SplitMix64 seed) then brick CNOTs: 1200 U3 + 580 CNOT = 1780 gates
on a 16 GiB complex128 state.  A step is one full evolution of the resident state by the
circuit.  value = amplitude updates per second = steps * 1780 * 2^30 / time (summed over
ranks).  Inputs are larger than L2 (16 GiB state), so no flush is needed between steps.

e2e: the same metric through the drop-in port qm_execute_host with a pinned host buffer,
the host->device upload and device->host commit inside the timed region every step.

Multi-GPU: one process per GPU, each an independent replica (the single-state path does not
shard); timing is the max over ranks; value sums the ranks' work (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

QUBITS = 30
DEPTH = 40
FALLBACK_HBM_GBS = 6650.0
DEFAULT_DRAW_SEED = 20260101


def measured_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": FALLBACK_HBM_GBS, "bf16_tflops": 1590.0}, "fallback"


def fp64_roofline(flops_per_step: float, steps: int, seconds: float, launches: int, clocks: dict) -> dict:
    """FP64 side of the pass roofline: the flops the compiled passes issue per launch, their rate,
    and the CUDA-core FP64 peak (64 FMA = 128 flops per clock per SM, 148 SMs) at the median SM
    clock sampled during the timed region (1965 MHz when no sample was taken)."""
    mhz = clocks.get("sm_mhz") or 1965.0
    peak = 128 * 148 * mhz * 1e6 / 1e12
    achieved = flops_per_step * steps / seconds / 1e12
    return {"achieved_tflops": achieved, "peak_tflops": peak, "frac": achieved / peak,
            "flops_per_launch": flops_per_step / max(1, launches), "peak_source": "nominal at the sampled SM clock"}


def profile_value(name: str, kernel_key: str) -> float | None:
    """A figure of the dominant kernel from the committed ncu summaries (`name[kernel]: value`)."""
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"{re.escape(name)}\[{re.escape(kernel_key)}\]:\s*([0-9.eE+]+)", f.read_text())
        if m:
            return float(m.group(1))
    return None


def profile_traffic(kernel_key: str) -> float | None:
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    return profile_value("traffic", kernel_key)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                return
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        return dist, rank, world, local
    return None, 0, 1, 0


def barrier_max(dist, value: float, local: int) -> float:
    if dist is None:
        return value
    import torch
    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def first_layer_gates(qubits: int) -> int:
    """Gates of the brick circuit's first layer: a U3 on every qubit, then CNOTs on the even pairs."""
    return qubits + qubits // 2


def cpu_baseline(circuit, qubits: int, sample_gates: int) -> dict:
    """The reference's parallel/AVX-512 CPU path (oracle port) on the first layer of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as orc
    from quantummatter_b200.circuit import QuantumCircuit
    sub = QuantumCircuit(qubits)
    for op in circuit.Operations[:sample_gates]:
        sub.AppendValidated(op)
    threads = orc.hardware_threads()
    state = np.zeros(1 << qubits, dtype=np.complex128)
    state[0] = 1
    orc.execute_parallel(sub, state, workers=threads)  # warm-up (first touch, pool start)
    t0 = time.perf_counter()
    orc.execute_parallel(sub, state, workers=threads)
    dt = time.perf_counter() - t0
    return {"value": sample_gates * (1 << qubits) / dt, "unit": "amp-updates/s", "cores": threads, "kind": "port",
            "sample": f"first layer of the {qubits}-qubit circuit ({sample_gates} gates: {qubits} U3 + "
                      f"{sample_gates - qubits} CNOT) on the full state, AVX-512 + gate blocking, {threads} worker "
                      f"threads, {dt:.2f} s"}


class _DeviceBuffer:
    """A raw device allocation of the library exposed through __cuda_array_interface__."""

    def __init__(self, pointer: int, length: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (length,), "typestr": typestr, "data": (pointer, False),
                                         "version": 3, "strides": None}


def max_abs_diff(a, b, chunk: int = 1 << 27) -> float:
    """Largest complex |a_i - b_i| between two library states of one size, on the device (torch
    views of the library's buffers, no copy), accumulated in FP64."""
    import torch

    from quantummatter_b200.backend import FP64
    views = []
    for st in (a, b):
        typestr = "<f8" if st.precision == FP64 else "<f4"
        views.append(torch.as_tensor(_DeviceBuffer(st.device_pointer(), 2 << st.QubitCount, typestr), device="cuda"))
    worst = 0.0
    for start in range(0, views[0].numel(), 2 * chunk):
        x = views[0][start:start + 2 * chunk].double().view(-1, 2)
        y = views[1][start:start + 2 * chunk].double().view(-1, 2)
        worst = max(worst, torch.linalg.vector_norm(x - y, dim=1).max().item())
    torch.cuda.synchronize()
    return worst


def fp32_side_run(ctx, circuit, state64, plan64, steps: int) -> dict:
    """The complex64 form of the same circuit: its own plan timed on the device, and the largest
    amplitude error of one evolution from |0...0> against the complex128 plan's."""
    from quantummatter_b200.backend import FP32, DeviceState, Plan
    qubits, gates = circuit.QubitCount, len(circuit.Operations)
    plan32 = Plan(ctx, circuit, FP32)
    try:
        with DeviceState(ctx, qubits, FP32) as st:
            plan32.execute(st)
            seconds = [plan32.execute(st, profile=True).DeviceEvolutionSeconds for _ in range(steps)]
            st.Reset()
            plan32.execute(st)
            state64.Reset()
            plan64.execute(state64)
            err = max_abs_diff(state64, st)
        passes = plan32.stats()[0]
    finally:
        plan32.Dispose()
    per = sum(seconds) / len(seconds)
    return {"value": gates * (1 << qubits) / per, "unit": "amp-updates/s", "ms_per_step": 1e3 * per,
            "steps": steps, "passes": passes, "max_abs_err_vs_fp64": err,
            "err_reference": "complex128 compiled plan on the same GPU, one evolution from |0...0>"}


def vqe_side_run(ctx, qubits: int = 22, vectors: int = 16) -> dict:
    """A bounded batched-variational run beside the headline: the hardware-efficient ansatz (4
    layers) on a `qubits`-site XXZ chain, `vectors` parameter vectors with full parameter-shift
    gradients, FP32 and FP64 batched, against the plain form (one FP64 circuit at a time on a
    resident state); warm-up with the full batch so no compilation or graph capture is timed, then
    the faster of two timed calls."""
    import numpy as np

    from quantummatter_b200.backend import FP32, FP64, DeviceState
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    from quantummatter_b200.workloads import hardware_efficient_ansatz, uniform_parameters, xxz_chain
    c = hardware_efficient_ansatz(qubits, 4)
    h = xxz_chain(qubits)
    params = uniform_parameters(c.ParameterCount, vectors, -np.pi, np.pi, seed=qubits)
    out, res = {}, {}
    for name, prec in (("fp32", FP32), ("fp64", FP64)):
        ev = B200VariationalEnergyEvaluator(ctx, prec)
        ev.EvaluateBatch(c, h, params, withGradient=True)
        best = None
        for _ in range(2):  # one call is about a second of wall time: keep the faster of two
            t0 = time.perf_counter()
            r = ev.EvaluateBatch(c, h, params, withGradient=True)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        res[name] = r
        out[f"batched_{name}_evals_per_s"] = r.Circuits / best
    bound = [c.Bind(list(params[0]))] + [c.BindWithRotationShift(list(params[0]), r, s)
                                         for r in range(8) for s in (np.pi / 2, -np.pi / 2)]
    with DeviceState(ctx, qubits, FP64) as st:
        st.Evolve(bound[0])
        st.ExpectationEnergy(h)
        t0 = time.perf_counter()
        for b in bound:
            st.Reset()
            st.Evolve(b)
            st.ExpectationEnergy(h)
        plain = len(bound) / (time.perf_counter() - t0)
    out["plain_fp64_evals_per_s"] = plain
    out["batched_fp32_over_plain"] = out["batched_fp32_evals_per_s"] / plain
    out["fp32_max_abs_dE_vs_fp64"] = float(np.max(np.abs(res["fp32"].Energies - res["fp64"].Energies)))
    out["fp32_max_abs_dgrad_vs_fp64"] = float(np.max(np.abs(res["fp32"].Gradients - res["fp64"].Gradients)))
    out["config"] = (f"hardware-efficient ansatz, 4 layers, {qubits}-site XXZ chain, {vectors} vectors with full "
                     f"parameter-shift gradients ({res['fp64'].Circuits} circuits per batch)")
    return out


def run_widths(args) -> None:
    """Fusion-width sweep of the 30-qubit brick (depth 40): widths k = 1..6 (dense fused gates of at
    most k qubits, one sweep of the state each; k = 1 is one launch per gate) and the default fused
    blocks of 12 qubits, in complex128 and complex64.  Per width and precision: amp-updates/s, the
    plan's HBM GB/s (read + write of every sweep) against the copy peak, and the largest amplitude
    error of one evolution from |0...0> against the complex128 fused-block plan, which equals the
    per-gate path over all 2^30 amplitudes to 1e-12 (tests/test_headline_parity.py)."""
    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context, DeviceState, Plan
    from quantummatter_b200.workloads import brick_circuit
    qubits, depth = args.qubits, args.depth
    circuit = brick_circuit(qubits, depth)
    gates, amps = len(circuit.Operations), 1 << qubits
    peaks, peak_kind = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=150 << 30, StagingMemoryBudgetBytes=1 << 30,
                                         EnableProfiling=True))
    widths = [int(w) for w in args.widths.split(",")]
    rows = []
    ref_plan = Plan(ctx, circuit, FP64)
    ref = DeviceState(ctx, qubits, FP64)
    ref_plan.execute(ref)
    with ClockSampler(0) as clocks:
        for precision, name in ((FP64, "fp64"), (FP32, "fp32")):
            for width in widths:
                plan = Plan(ctx, circuit, precision, width)
                passes, launches, planned = plan.stats()
                try:
                    with DeviceState(ctx, qubits, precision) as st:
                        plan.execute(st)
                        err = max_abs_diff(ref, st)
                        secs = [plan.execute(st, profile=True).DeviceEvolutionSeconds for _ in range(args.steps)]
                finally:
                    plan.Dispose()
                per = sum(secs) / len(secs)
                gbs = planned / per / 1e9
                rows.append({"precision": name, "width": width,
                             "scheme": "one launch per gate" if width == 1 else
                             (f"dense fused gates of <= {width} qubits" if width <= 6 else f"fused blocks of {width} qubits"),
                             "launches": launches, "amp_updates_per_s": gates * amps / per, "ms_per_step": 1e3 * per,
                             "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak, "max_abs_err_vs_fp64": err})
                print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    ref.Dispose()
    ref_plan.Dispose()
    line = {"metric": f"amp-updates/s at {qubits}q by fusion width", "unit": "amp-updates/s",
            "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "data": "synthetic",
            "config": {"workload": f"brick circuit, {qubits} qubits, depth {depth}, U3 + CNOT, {gates} gates",
                       "peak_gbs": hbm_peak, "peak_source": peak_kind,
                       "error_reference": "complex128 fused-block plan, one evolution from |0...0>"},
            "sweep": rows, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    ctx.Dispose()


def run_reference(args) -> None:
    """`--impl reference`: the reference's own CPU implementation (parallel/AVX-512 port) on this
    arm's workload; each step is a bounded sample of the circuit."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from quantummatter_b200.workloads import brick_circuit
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as orc
    from quantummatter_b200.circuit import QuantumCircuit
    circuit = brick_circuit(QUBITS, DEPTH)
    sample = first_layer_gates(QUBITS)
    sub = QuantumCircuit(QUBITS)
    for op in circuit.Operations[:sample]:
        sub.AppendValidated(op)
    threads = orc.hardware_threads()
    state = np.zeros(1 << QUBITS, dtype=np.complex128)
    state[0] = 1
    for _ in range(args.warmup):
        orc.execute_parallel(sub, state, workers=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.execute_parallel(sub, state, workers=threads)
    dt = time.perf_counter() - t0
    value = args.steps * sample * (1 << QUBITS) / dt
    line = {
        "impl": "reference", "metric": "amp-updates/s at 30q", "value": value, "unit": "amp-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "brick circuit, 30 qubits, depth 40, U3 + CNOT, 1780 gates, complex128 state",
                   "qubits": QUBITS, "depth": DEPTH, "gates": len(circuit.Operations),
                   "sample_per_step": f"first layer of the circuit ({sample} gates: {QUBITS} U3 + "
                                      f"{sample - QUBITS} CNOT) on the full 2^30 state"},
        "cpu_baseline": {"value": value, "unit": "amp-updates/s", "cores": threads, "kind": "port",
                         "sample": f"first layer ({sample} gates) per step, {threads} threads, AVX-512 + gate "
                                   f"blocking"},
        "e2e": {"value": value, "unit": "amp-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_vqe(args) -> None:
    """Batched VQE energy/gradient workload: hardware-efficient ansatz (4 layers of RY, RZ, CZ
    ladder, P = 8n) on 16-, 18-, 20- and 22-qubit XXZ chains, `--vectors` parameter vectors per
    size drawn uniform in [-pi, pi], each with its full parameter-shift gradient (1 + 2P circuits).
    Reports energy evaluations per second for the batched FP32 and FP64 forms and for the plain
    form (one FP64 circuit at a time on a resident device state), and the FP32 energies' largest
    |delta E| against the FP64 batch."""
    import numpy as np

    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context, DeviceState
    from quantummatter_b200.variational import B200VariationalEnergyEvaluator
    from quantummatter_b200.workloads import hardware_efficient_ansatz, uniform_parameters, xxz_chain
    sizes = [int(s) for s in args.sizes.split(",")]
    ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=120 << 30, StagingMemoryBudgetBytes=1 << 30,
                                         FusionWidth=args.width))
    results = {}
    total_circuits = 0
    max_de = 0.0
    timings = {"fp32": 0.0, "fp64": 0.0}
    per_size_energies = {}
    for n in sizes:
        c = hardware_efficient_ansatz(n, 4)
        h = xxz_chain(n)
        params = uniform_parameters(c.ParameterCount, args.vectors, -np.pi, np.pi, seed=n)
        per = {}
        for name, prec in (("fp32", FP32), ("fp64", FP64)):
            ev = B200VariationalEnergyEvaluator(ctx, prec)
            ev.EvaluateBatch(c, h, params, withGradient=True)  # warm-up: plans, kernel attributes, graph capture
            t0 = time.perf_counter()
            r = ev.EvaluateBatch(c, h, params, withGradient=True)
            dt = time.perf_counter() - t0
            timings[name] += dt
            per[name] = r
            results[f"n{n}_{name}"] = {"seconds": dt, "circuits": r.Circuits, "evals_per_s": r.Circuits / dt,
                                       "waves": r.Waves, "batch_states": r.BatchStates,
                                       "passes_per_circuit": r.PassesPerCircuit, "tile_passes": r.TilePasses}
        per_size_energies[n] = per["fp32"].Energies
        de = float(np.max(np.abs(per["fp32"].Energies - per["fp64"].Energies)))
        dg = float(np.max(np.abs(per["fp32"].Gradients - per["fp64"].Gradients)))
        results[f"n{n}_fp32_max_abs_dE"] = de
        results[f"n{n}_fp32_max_abs_dgrad"] = dg
        max_de = max(max_de, de)
        total_circuits += per["fp64"].Circuits
    # every size in one call: each round's waves of all sizes on their own streams, one graph launch
    mixed_problems = []
    for n in sizes:
        c = hardware_efficient_ansatz(n, 4)
        mixed_problems.append((c, xxz_chain(n), uniform_parameters(c.ParameterCount, args.vectors, -np.pi, np.pi,
                                                                    seed=n)))
    ev32 = B200VariationalEnergyEvaluator(ctx, FP32)
    ev32.EvaluateMixed([(c, h, p[:2]) for c, h, p in mixed_problems])  # warm-up
    t0 = time.perf_counter()
    mixed_outs, mixed_total = ev32.EvaluateMixed(mixed_problems)
    mixed_dt = time.perf_counter() - t0
    mixed_equal = all(np.array_equal(o[0], results_e) for o, results_e in
                      zip(mixed_outs, [per_size_energies[n] for n in sizes]))
    # plain form: one FP64 circuit at a time, resident state, per-term energy on the device
    n = sizes[-1]
    c = hardware_efficient_ansatz(n, 4)
    h = xxz_chain(n)
    params = uniform_parameters(c.ParameterCount, 1, -np.pi, np.pi, seed=n)[0]
    bound = [c.Bind(list(params))] + [c.BindWithRotationShift(list(params), r, s)
                                      for r in range(8) for s in (np.pi / 2, -np.pi / 2)]
    with DeviceState(ctx, n, FP64) as st:
        st.Evolve(bound[0])
        st.ExpectationEnergy(h)
        t0 = time.perf_counter()
        for b in bound:
            st.Reset()
            st.Evolve(b)
            st.ExpectationEnergy(h)
        plain_dt = (time.perf_counter() - t0) / len(bound)
    batched_n = results[f"n{n}_fp32"]["evals_per_s"]
    line = {
        "metric": "energy evals/s (batched VQE energy + parameter-shift gradient)", "unit": "evals/s",
        "value": total_circuits / timings["fp32"], "higher_is_better": True, "n_gpus": 1, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "hardware-efficient ansatz, 4 layers RY/RZ/CZ ladder, XXZ chain, "
                               f"sizes {sizes}, {args.vectors} vectors each, full parameter-shift gradients",
                   "circuits": total_circuits},
        "fp64_value": total_circuits / timings["fp64"],
        "mixed_fp32_evals_per_s": mixed_total.Circuits / mixed_dt,
        "mixed_fp32": {"rounds": mixed_total.Waves, "batch_states": mixed_total.BatchStates,
                       "device_seconds": mixed_total.DeviceSeconds, "wall_seconds": mixed_dt,
                       "energies_equal_per_size_runs": bool(mixed_equal),
                       "form": "all sizes in one qm_vqe_evaluate_mixed call: each round one graph launch with a "
                               "branch per size"},
        "fp32_max_abs_dE_vs_fp64": max_de,
        f"plain_fp64_evals_per_s_n{n}": 1.0 / plain_dt,
        f"batched_fp32_over_plain_n{n}": batched_n * plain_dt,
        "per_size": results,
    }
    print(json.dumps(line), flush=True)
    ctx.Dispose()


def run_trajectories(args) -> None:
    """Batched noise trajectories: RY / CZ-ladder circuit (24 qubits, depth 30) with
    depolarizing noise after every gate and amplitude damping on every qubit per layer,
    `--trajectories` trajectories from one seeded System.Random stream (reference draw order),
    <Z_i> and <Z_i Z_i+1> per trajectory.  FP32 state, FP64 renormalisation and reductions."""
    import numpy as np

    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context
    from quantummatter_b200.observables import PauliString
    from quantummatter_b200.trajectories import B200NoisySimulator, random_doubles
    from quantummatter_b200.workloads import noisy_ry_cz_ladder
    n, depth, T = args.traj_qubits, args.traj_depth, args.trajectories
    prec = FP64 if args.traj_precision == "fp64" else FP32
    nc = noisy_ry_cz_ladder(n, depth)
    flat, placements = nc.Flatten()
    gates = len(flat.Operations)
    D = nc.MaxDraws()
    obs = [PauliString("".join("Z" if q == i else "I" for q in reversed(range(n)))) for i in range(n)]
    obs += [PauliString("".join("Z" if q in (i, i + 1) else "I" for q in reversed(range(n)))) for i in range(n - 1)]
    # ranks: each GPU runs its own T trajectories, the next slice of one seeded stream (weak
    # scaling); the timed region is bracketed by barriers and timed as the max over ranks
    dist, rank, world, local = dist_setup(args.gpus)
    stream = random_doubles(DEFAULT_DRAW_SEED, T * D, skip=rank * T * D)
    rows = stream.reshape(T, D)
    ctx = B200Context(B200BackendOptions(DeviceIndex=local, DeviceMemoryBudgetBytes=160 << 30,
                                         StagingMemoryBudgetBytes=1 << 30))
    sim = B200NoisySimulator(ctx, precision=prec)
    sim.RunBatch(nc, rows[:8], obs)  # warm-up: plans, kernel attributes
    clocks = ClockSampler(local)
    barrier_max(dist, 0.0, local)
    with clocks:
        t0 = time.perf_counter()
        res = sim.RunBatch(nc, rows, obs)
        wall = time.perf_counter() - t0
    wall = barrier_max(dist, wall, local)
    if rank != 0:
        ctx.Dispose()
        if dist is not None:
            dist.destroy_process_group()
        return
    # every trajectory drew once per placement, so the rows were the reference's draw order
    in_order = bool(np.all(res.consumed == D))
    dev = res.stats["device_seconds"]
    state_bytes = (8 if prec == FP32 else 16) << n
    per_traj = (2 * res.stats["passes"] + res.stats["mass_passes"]) * state_bytes
    peaks, peak_kind = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    achieved = per_traj * T / dev / 1e9
    # FP32 against FP64 on the same draws
    check = min(8, T)
    other = B200NoisySimulator(ctx, precision=FP64 if prec == FP32 else FP32).RunBatch(nc, rows[:check], obs)
    err = float(np.max(np.abs(other.values - res.values[:check])))
    # CPU baseline: the oracle (scalar port, one thread) on the first layer of one trajectory
    cpu = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as orc
        layer = noisy_ry_cz_ladder(n, 1)
        t1 = time.perf_counter()
        orc.trajectory(layer, stream[:layer.MaxDraws()])
        cpu_dt = (time.perf_counter() - t1) * depth
        cpu = {"value": 1.0 / cpu_dt, "unit": "trajectories/s", "cores": 1, "kind": "port",
               "sample": f"oracle NoisyCircuit.Execute restatement, first of {depth} layers of one {n}-qubit "
                         f"trajectory ({time.perf_counter() - t1:.2f} s), scaled to the full depth"}
    line = {
        "metric": "noise trajectories/s", "value": world * T / wall, "unit": "trajectories/s", "n_gpus": world,
        "steps": 1,
        "warmup": 1, "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if prec == FP32 else "f64", "data": "synthetic",
        "config": {"workload": f"noisy RY/CZ ladder, {n} qubits, depth {depth}, {gates} gates, {len(placements)} "
                               f"channel placements (depolarizing 1e-3 / 1e-2, damping 1e-3), {T} trajectories, "
                               f"{len(obs)} Z / ZZ observables", "draws": f"seeded System.Random stream, {D} per trajectory",
                   "reference_draw_order": in_order, "l2": "inputs larger than L2; no flush"},
        "device_trajectories_per_s": T / dev,
        "amp_updates_per_s": T * gates * (1 << n) / wall,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": None, "peak_source": peak_kind,
                     "model": "per trajectory: 2 x state per fused pass + 1 x state per joint-mass pass"},
        "stats": res.stats, "max_abs_error_vs_other_precision": err,
        "ambiguous_damping_draws": int(res.ambiguous.sum()), "clocks": clocks.summary(),
        "e2e": {"value": world * T / wall, "unit": "trajectories/s", "h2d_bytes_per_step": int(rows.nbytes) * world,
                "d2h_bytes_per_step": int(res.values.nbytes + res.masses.nbytes) * world},
        "cpu_baseline": cpu,
    }
    line["config"]["parallelism"] = f"trajectory partitions x{world}"
    print(json.dumps(line), flush=True)
    ctx.Dispose()
    if dist is not None:
        dist.destroy_process_group()


def serving_requests(count: int, rate: float, precision: int, seed: int, sessions, kinds: int = 3):
    """Poisson arrivals at `rate`; each request an expectation of a random brick circuit (Z_i and
    Z_i Z_i+1), 1000 shots of one, or a VQE step of a random session (TFIM chain, hardware-efficient
    ansatz of 2 layers); qubits uniform in [10, 28], brick depth uniform in [10, 100]."""
    import numpy as np

    from quantummatter_b200.observables import PauliString
    from quantummatter_b200.serving import ExpectationRequest, ShotsRequest, VqeStepRequest
    from quantummatter_b200.workloads import brick_circuit
    rng = np.random.default_rng(seed)
    t, arrivals, reqs = 0.0, [], []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        arrivals.append(t)
        kind = int(rng.integers(kinds))
        if kind == 2:
            reqs.append(VqeStepRequest(sessions[int(rng.integers(len(sessions)))]))
            continue
        n, depth = int(rng.integers(10, 29)), int(rng.integers(10, 101))
        c = brick_circuit(n, depth, seed=seed * 1000 + i)
        if kind == 0:
            obs = [PauliString("".join("Z" if q == j else "I" for q in reversed(range(n)))) for j in range(n)]
            obs += [PauliString("".join("Z" if q in (j, j + 1) else "I" for q in reversed(range(n)))) for j in range(n - 1)]
            reqs.append(ExpectationRequest(c, obs, precision))
        else:
            reqs.append(ShotsRequest(c, shots=1000, seed=i, precision=precision))
    return reqs, arrivals


def serving_sessions(count: int, precision: int, seed: int):
    import numpy as np

    from quantummatter_b200.serving import VqeSession
    from quantummatter_b200.workloads import hardware_efficient_ansatz, tfim_chain
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(10, 29))
        c = hardware_efficient_ansatz(n, 2)
        out.append(VqeSession(c, tfim_chain(n, seed=seed + i), rng.uniform(-np.pi, np.pi, c.ParameterCount),
                              step_size=0.05, precision=precision))
    return out


def serving_summary(responses, reqs, makespan: float) -> dict:
    import numpy as np

    from quantummatter_b200.serving import VqeStepRequest
    lat = np.array([r.latency for r in responses])
    evals = sum(1 + 2 * len(q.session.circuit.RotationParameterIndices) for q in reqs if isinstance(q, VqeStepRequest))
    per_kind = {}
    for kind in ("expectation", "shots", "vqe_step"):
        k = np.array([r.latency for r in responses if r.kind == kind])
        if k.size:
            per_kind[kind] = {"count": int(k.size), "p50_ms": float(np.percentile(k, 50) * 1e3),
                              "p99_ms": float(np.percentile(k, 99) * 1e3)}
    return {"requests": len(responses), "makespan_s": makespan, "requests_per_s": len(responses) / makespan,
            "energy_evals_per_s": evals / makespan, "energy_evals": evals,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_vqe_batch": float(np.mean([r.batch for r in responses if r.kind == "vqe_step"] or [1])),
            "per_kind": per_kind}


def run_serving_closed(args) -> None:
    """Closed-loop serving: one client thread per VQE session submits its next step only when the
    previous one returned (16 sessions: TFIM chains of 14, 16, 18 and 20 sites, 4 each, 2-layer
    hardware-efficient ansatz), beside `--background` clients that keep one expectation or
    1000-shot request each in flight (random brick circuits of 10-28 qubits).  The server runs
    at its own pace, so its throughput is capacity, not offered load.  The plain form runs the same
    VQE steps one circuit at a time in FP64."""
    import numpy as np

    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context
    from quantummatter_b200.serving import B200Server, VqeSession, VqeStepRequest, serve_plain
    from quantummatter_b200.workloads import hardware_efficient_ansatz, tfim_chain
    sizes = [int(x) for x in args.session_sizes.split(",")]
    steps = args.session_steps

    def sessions(prec):
        rng = np.random.default_rng(17)
        out = []
        for n in sizes:
            c = hardware_efficient_ansatz(n, 2)
            for k in range(args.sessions_per_size):
                out.append(VqeSession(c, tfim_chain(n, seed=100 * n + k), rng.uniform(-np.pi, np.pi, c.ParameterCount),
                                      step_size=0.05, precision=prec))
        return out

    def evals(s):
        return 1 + 2 * len(s.circuit.RotationParameterIndices)

    results = {}
    clocks = ClockSampler(0)
    with clocks:
        for name, prec in (("fp32", FP32), ("fp64", FP64)):
            ss = sessions(prec)
            background, _ = serving_requests(args.background * 40, 1.0, prec, seed=23, sessions=[], kinds=2)
            with B200Server(workers=args.workers, budget_bytes=args.serve_budget << 30,
                            context_budget_bytes=24 << 30, cache_bytes=8 << 30) as server:
                warm = sessions(prec)  # plans and kernels of every size, outside the timed region
                for f in [server.submit(VqeStepRequest(s)) for s in warm]:
                    f.result()
                for f in [server.submit(r) for r in background[:4]]:
                    f.result()
                responses, lock, stop = [], threading.Lock(), threading.Event()

                def vqe_client(s):
                    for _ in range(steps):
                        r = server.submit(VqeStepRequest(s)).result()
                        with lock:
                            responses.append(r)

                def background_client(k):
                    i = k
                    while not stop.is_set() and i < len(background):
                        r = server.submit(background[i]).result()
                        with lock:
                            responses.append(r)
                        i += args.background

                t0 = time.perf_counter()
                threads = [threading.Thread(target=vqe_client, args=(s,)) for s in ss]
                bg = [threading.Thread(target=background_client, args=(k,)) for k in range(args.background)]
                for t in threads + bg:
                    t.start()
                for t in threads:
                    t.join()
                makespan = time.perf_counter() - t0
                stop.set()
                for t in bg:
                    t.join()
                stats = server.stats()
            vq = [r for r in responses if r.kind == "vqe_step"]
            lat = np.array([r.latency for r in responses if r.finished - t0 <= makespan + 1e-9])
            vlat = np.array([r.latency for r in vq])
            results[name] = {"makespan_s": makespan, "vqe_steps": len(vq),
                             "energy_evals_per_s": steps * sum(evals(s) for s in ss) / makespan,
                             "requests_per_s": len(lat) / makespan,
                             "mean_vqe_batch": float(np.mean([r.batch for r in vq])),
                             "max_vqe_batch": int(max(r.batch for r in vq)),
                             "vqe_p50_ms": float(np.percentile(vlat, 50) * 1e3),
                             "vqe_p99_ms": float(np.percentile(vlat, 99) * 1e3),
                             "all_p50_ms": float(np.percentile(lat, 50) * 1e3),
                             "all_p99_ms": float(np.percentile(lat, 99) * 1e3),
                             "background_requests": len(responses) - len(vq),
                             "server": {k: stats[k] for k in ("jobs", "vqe_jobs", "vqe_steps", "max_batch",
                                                              "peak_reserved_bytes", "budget_bytes")}}
        # plain form: the same VQE steps, one circuit at a time, FP64, one request after another
        ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=24 << 30, StagingMemoryBudgetBytes=1 << 30))
        ss = sessions(FP64)
        serve_plain([VqeStepRequest(s) for s in sessions(FP64)[::args.sessions_per_size]], ctx)  # warm-up
        sample = ss[::args.sessions_per_size]  # one session per size, every step
        t0 = time.perf_counter()
        plain = []
        for _ in range(steps):
            plain += serve_plain([VqeStepRequest(s) for s in sample], ctx)
        plain_dt = time.perf_counter() - t0
        ctx.Dispose()
        plain_evals = steps * sum(evals(s) for s in sample) / plain_dt
        plat = np.array([r.latency for r in plain])
        results["plain_fp64"] = {"energy_evals_per_s": plain_evals, "seconds": plain_dt,
                                 "vqe_p50_ms": float(np.percentile(plat, 50) * 1e3),
                                 "vqe_p99_ms": float(np.percentile(plat, 99) * 1e3),
                                 "sample": f"one session per size ({len(sample)}), {steps} steps each"}
    line = {
        "metric": "served energy evals/s (closed loop)", "value": results["fp32"]["energy_evals_per_s"],
        "unit": "evals/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"closed loop: {len(sizes) * args.sessions_per_size} VQE sessions (TFIM chains of "
                               f"{sizes} sites, {args.sessions_per_size} each, 2-layer hardware-efficient ansatz), "
                               f"{steps} steps each, one step in flight per session; {args.background} background "
                               "clients with expectation / 1000-shot requests (brick circuits, 10-28 qubits)",
                   "workers": args.workers, "budget_gib": args.serve_budget},
        "p50_ms": results["fp32"]["vqe_p50_ms"], "p99_ms": results["fp32"]["vqe_p99_ms"],
        "fp32_over_plain_fp64": results["fp32"]["energy_evals_per_s"] / plain_evals,
        "fp64_over_plain_fp64": results["fp64"]["energy_evals_per_s"] / plain_evals,
        "results": results, "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def run_serving(args) -> None:
    """Serving: Poisson request streams at swept rates through the batching server (FP32 and FP64),
    and the plain form (one request at a time, FP64, unbatched) on the same stream."""
    from quantummatter_b200.backend import FP32, FP64, B200BackendOptions, B200Context
    from quantummatter_b200.serving import B200Server, serve_plain
    rates = [float(r) for r in args.rates.split(",")]
    results = {}
    clocks = ClockSampler(0)
    with clocks:
        for name, prec in (("fp32", FP32), ("fp64", FP64)):
            for rate in rates:
                sessions = serving_sessions(args.sessions, prec, seed=7)
                reqs, arrivals = serving_requests(args.requests, rate, prec, seed=11, sessions=sessions)
                with B200Server(workers=args.workers, budget_bytes=args.serve_budget << 30,
                                context_budget_bytes=24 << 30, cache_bytes=8 << 30) as server:
                    # warm-up: kernel attributes and plans of each kind
                    warm = serving_sessions(1, prec, seed=3)
                    wr, _ = serving_requests(3, 1.0, prec, seed=5, sessions=warm)
                    for f in [server.submit(r) for r in wr]:
                        f.result()
                    t0 = time.perf_counter()
                    futures = []
                    for req, at in zip(reqs, arrivals):
                        wait = t0 + at - time.perf_counter()
                        if wait > 0:
                            time.sleep(wait)
                        futures.append(server.submit(req))
                    responses = [f.result() for f in futures]
                    makespan = max(r.finished for r in responses) - t0
                results[f"{name}_rate{rate:g}"] = serving_summary(responses, reqs, makespan)
        # plain form at the lowest rate on the same stream (FP64)
        ctx = B200Context(B200BackendOptions(DeviceMemoryBudgetBytes=24 << 30, StagingMemoryBudgetBytes=1 << 30))
        sessions = serving_sessions(args.sessions, FP64, seed=7)
        reqs, arrivals = serving_requests(args.requests, rates[0], FP64, seed=11, sessions=sessions)
        warm = serving_sessions(1, FP64, seed=3)
        serve_plain(serving_requests(3, 1.0, FP64, seed=5, sessions=warm)[0], ctx)
        t0 = time.perf_counter()
        plain = serve_plain(reqs, ctx, arrivals)
        results[f"plain_fp64_rate{rates[0]:g}"] = serving_summary(plain, reqs, max(r.finished for r in plain) - t0)
        ctx.Dispose()
    top = results[f"fp32_rate{rates[-1]:g}"]
    same = results[f"fp64_rate{rates[0]:g}"]
    plain = results[f"plain_fp64_rate{rates[0]:g}"]
    line = {
        "metric": "served energy evals/s", "value": top["energy_evals_per_s"], "unit": "evals/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic", "scaling": "weak", "vs_baseline": None,
        "config": {"workload": "Poisson request stream: expectations of random brick circuits (depth 10-100), 1000 "
                               "shots, or VQE steps (TFIM chains, 2-layer hardware-efficient ansatz); qubits 10-28; "
                               f"admission budget {args.serve_budget} GiB at 16 * 2^n (FP64) or 8 * 2^n (FP32) bytes "
                               f"per request; {args.workers} workers; {args.requests} requests per rate",
                   "rates_per_s": rates, "sessions": args.sessions},
        "p99_ms": top["p99_ms"], "p50_ms": top["p50_ms"],
        f"fp64_p99_ms_rate{rates[0]:g}": same["p99_ms"], f"plain_fp64_p99_ms_rate{rates[0]:g}": plain["p99_ms"],
        "p99_vs_plain_fp64": same["p99_ms"] / plain["p99_ms"],
        "energy_evals_per_s_vs_plain_fp64": same["energy_evals_per_s"] / plain["energy_evals_per_s"],
        "results": results, "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--width", type=int, default=0, help="fusion width (block qubits); 1 = one launch per gate")
    ap.add_argument("--qubits", type=int, default=QUBITS)
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-side-runs", action="store_true",
                    help="skip the complex64 and batched-variational side runs of the default line")
    ap.add_argument("--workload", default="brick", choices=["brick", "vqe", "trajectories", "serving", "widths"])
    ap.add_argument("--widths", default="1,2,3,4,5,6,12", help="widths workload: fusion widths to sweep")
    ap.add_argument("--circuit", default="brick", choices=["brick", "qft", "grover"],
                    help="brick workload: the circuit (qft and grover: the algorithm builders at --qubits)")
    ap.add_argument("--sizes", default="16,18,20,22", help="vqe workload: qubit counts")
    ap.add_argument("--vectors", type=int, default=128, help="vqe workload: parameter vectors per size")
    ap.add_argument("--traj-qubits", type=int, default=24, help="trajectories workload: qubits")
    ap.add_argument("--traj-depth", type=int, default=30, help="trajectories workload: layers")
    ap.add_argument("--trajectories", type=int, default=1024, help="trajectories workload: trajectories")
    ap.add_argument("--traj-precision", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--rates", default="1,3", help="serving workload: arrival rates per second")
    ap.add_argument("--requests", type=int, default=40, help="serving workload: requests per rate")
    ap.add_argument("--sessions", type=int, default=12, help="serving workload: VQE sessions")
    ap.add_argument("--workers", type=int, default=4, help="serving workload: worker streams")
    ap.add_argument("--serve-budget", type=int, default=96, help="serving workload: admission budget, GiB")
    ap.add_argument("--serve-mode", default="open", choices=["open", "closed"],
                    help="serving workload: Poisson arrivals (open) or clients that wait for each result (closed)")
    ap.add_argument("--session-sizes", default="14,16,18,20", help="closed serving: VQE session sizes")
    ap.add_argument("--sessions-per-size", type=int, default=4, help="closed serving: sessions per size")
    ap.add_argument("--session-steps", type=int, default=4, help="closed serving: steps per session")
    ap.add_argument("--background", type=int, default=4, help="closed serving: expectation/shots clients")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "vqe":
        run_vqe(args)
        return
    if args.workload == "trajectories":
        run_trajectories(args)
        return
    if args.workload == "serving":
        run_serving_closed(args) if args.serve_mode == "closed" else run_serving(args)
        return
    if args.workload == "widths":
        run_widths(args)
        return

    dist, rank, world, local = dist_setup(args.gpus)
    import numpy as np

    from quantummatter_b200.backend import (FP32, FP64, B200BackendOptions, B200Context, B200StateVectorBackend,
                                            DeviceState, Plan, jit_info)
    from quantummatter_b200.algorithms import GroverSearch, QuantumFourierTransform
    from quantummatter_b200.workloads import brick_circuit

    qubits, depth = args.qubits, args.depth
    precision = FP32 if args.precision == "fp32" else FP64
    elem = 8 if precision == FP32 else 16
    if args.circuit == "qft":
        circuit = QuantumFourierTransform.CreateCircuit(qubits)
        described = f"quantum Fourier transform, {qubits} qubits (H, controlled phases, bit-reversal swaps)"
    elif args.circuit == "grover":
        inputs = (qubits + 2) // 2
        circuit = GroverSearch.CreateCircuit(inputs, (1 << inputs) // 3, iterations=2)
        qubits = circuit.QubitCount
        described = (f"Grover search, {inputs} input + {qubits - inputs} scratch qubits, 2 iterations "
                     f"(X, H, Toffoli ladders, CZ)")
    else:
        circuit = brick_circuit(qubits, depth)
        described = f"brick circuit, {qubits} qubits, depth {depth}, U3 + CNOT"
    gates = len(circuit.Operations)
    amps = 1 << qubits
    ctx = B200Context(B200BackendOptions(DeviceIndex=local, DeviceMemoryBudgetBytes=150 << 30,
                                         StagingMemoryBudgetBytes=80 << 30, EnableProfiling=True,
                                         FusionWidth=args.width))
    plan = Plan(ctx, circuit, precision, args.width)
    passes, launches, planned_bytes = plan.stats()
    state = DeviceState(ctx, qubits, precision)

    for _ in range(args.warmup):
        plan.execute(state)
    barrier_max(dist, 0.0, local)
    device_seconds = []
    jit_before = jit_info()["launches"]
    with ClockSampler(local) as clocks:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            prof = plan.execute(state, profile=True)
            device_seconds.append(prof.DeviceEvolutionSeconds)
        wall = time.perf_counter() - t_wall
    compiled = jit_info()["launches"] - jit_before == args.steps * launches and passes > 0
    total = sum(device_seconds)
    total_max = barrier_max(dist, total, local)
    ms_per_step = 1e3 * total_max / args.steps
    value = world * args.steps * gates * amps / total_max

    peaks, peak_kind = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    per_launch_s = total / (args.steps * launches)
    bytes_per_launch = planned_bytes / launches
    achieved_gbs = bytes_per_launch / per_launch_s / 1e9
    # the pass kernel that ran: compiled for each pass's op sequence (qm_pass) or the interpreter
    kernel_key = f"{'qm_pass' if compiled else 'k_fused'}_{args.precision}_k{plan_width(passes, qubits, precision, args.width)}_{qubits}q" \
        if passes else f"k_gate_{args.precision}_{qubits}q"
    traffic = profile_traffic(kernel_key)

    # arithmetic a dense 2x2 product would issue for the H, Rx, Ry and Unitary gates (16 real flops
    # per amplitude; permutations and diagonal phases free).  The compiled passes issue 8 per
    # amplitude for a general unitary (a scaled rotation between deferred phases), 4 for a real one.
    dense = sum(1 for op in circuit.Operations if int(op.Kind) in (0, 6, 7, 15))
    flops = dense * amps * 8 * 2
    # what the compiled passes issue, counting an FMA as 2 flops: at most 8 per amplitude for a
    # general 2x2 (Rx, U; 7 where the rotation's phase is known at compile time and applied by
    # three shears), 4 for a real one (H, Ry), against the FP64 peak of 64 FMA per clock per SM at
    # the sampled SM clock; the ncu pipe counter beside it is the measured side
    fp64_flops = amps * sum(8 if int(op.Kind) in (6, 15) else 4
                            for op in circuit.Operations if int(op.Kind) in (0, 6, 7, 15))
    e2e = None
    if not args.no_e2e and precision == FP64:
        backend = B200StateVectorBackend(context=ctx)
        host = ctx.host_array(amps)
        host.array[:] = 0
        host.array[0] = 1
        e2e_steps = max(2, args.steps // 2)
        backend.Execute(circuit, host.array)  # warm-up of the port (allocation of its device buffer)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            backend.Execute(circuit, host.array)
        dt = barrier_max(dist, time.perf_counter() - t0, local)
        e2e = {"value": world * e2e_steps * gates * amps / dt, "unit": "amp-updates/s",
               "h2d_bytes_per_step": elem * amps, "d2h_bytes_per_step": elem * amps,
               "ms_per_step": 1e3 * dt / e2e_steps, "path": "qm_execute_host (drop-in port), pinned host buffer"}
        host.free()
        backend.Dispose()

    fp64 = fp64_roofline(fp64_flops, args.steps, total, launches, clocks.summary())
    counter = profile_value("fp64_pipe_active", kernel_key)
    if counter is not None:
        fp64["pipe_active_counter"] = counter
        fp64["pipe_active_source"] = ("ncu sm__pipe_fp64_cycles_active of a 26-qubit capture of the same pass kind "
                                      "(profiles/qm_pass_fp64_brick26q_full.md)")
    side32 = side_vqe = None
    if rank == 0 and world == 1 and precision == FP64 and args.circuit == "brick" and not args.no_side_runs:
        # side runs never take the headline line down: a failure is reported in its place
        try:
            side32 = fp32_side_run(ctx, circuit, state, plan, steps=3)
        except Exception as e:  # noqa: BLE001
            side32 = {"error": f"{type(e).__name__}: {e}"}
        try:
            side_ctx = B200Context(B200BackendOptions(DeviceIndex=local, DeviceMemoryBudgetBytes=40 << 30,
                                                      StagingMemoryBudgetBytes=1 << 30))
            try:
                side_vqe = vqe_side_run(side_ctx)
            finally:
                side_ctx.Dispose()
        except Exception as e:  # noqa: BLE001
            side_vqe = {"error": f"{type(e).__name__}: {e}"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        state.Dispose()
        cpu = cpu_baseline(circuit, qubits, first_layer_gates(qubits) if args.circuit == "brick" else 8)

    if rank == 0:
        line = {
            "metric": f"amp-updates/s at {qubits}q", "value": value, "unit": "amp-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if precision == FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": f"{described}, {gates} gates, "
                                   f"{'complex64' if precision == FP32 else 'complex128'} state resident in HBM",
                       "qubits": qubits, "depth": depth, "gates": gates, "precision": args.precision,
                       "fusion": f"{passes} fused passes (block width {plan_width(passes, qubits, precision, args.width)})"
                       if passes else f"{launches} per-gate launches",
                       "l2": f"inputs larger than L2 ({elem * amps / 2**30:.0f} GiB state); no flush",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved_gbs / hbm_peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": kernel_key, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "launch_ms": 1e3 * per_launch_s,
                         "dense_2x2_equivalent_tflops": flops * args.steps / total / 1e12,
                         "fp64": fp64, "bound_frac": max(achieved_gbs / hbm_peak, fp64["frac"])},
            "gpu_launches": args.steps * launches,
            "clocks": clocks.summary(),
            "wall_s_timed": wall,
        }
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        if side32:
            line["fp32"] = side32
        if side_vqe:
            line["vqe_22q"] = side_vqe
        print(json.dumps(line), flush=True)
    plan.Dispose()
    try:
        state.Dispose()
    except Exception:
        pass
    ctx.Dispose()
    if dist is not None:
        dist.destroy_process_group()


def plan_width(passes: int, qubits: int, precision: int, width: int) -> int:
    if width:
        return width
    return min(12, qubits)


if __name__ == "__main__":
    main()
