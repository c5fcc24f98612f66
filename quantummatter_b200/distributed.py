"""Batch workloads over several GPUs: one process per GPU, units partitioned across ranks.

The single-state path does not shard (a 30-qubit FP64 state fits one B200), so a plain
evolution runs as independent replicas.  The batch workloads are independent units:
trajectories of a noisy circuit and parameter vectors of a VQE evaluation.  Each rank runs a
contiguous share of the units on its own GPU; the one exchange is an all-gather of the per-unit
results (a few KB), after which every rank holds the same results in unit order, so sums come
out in the same order, and with the same bits, as on one GPU.

Trajectories draw in the reference's order (one generator across all trajectories).  A rank
cannot know where its first trajectory starts in the stream until the earlier trajectories have
drawn, so every rank assumes the most draws per trajectory, all ranks exchange what each
trajectory consumed, and the trajectories after the first one that drew less run again from
the corrected offset: a loop of rounds that every rank takes in the same order.

The process group is torch.distributed (NCCL over NVLink between GPUs, gloo on the host for
tests); only host tensors of per-unit results cross it.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from .observables import PauliString


def partition(total: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of `total` units for `rank` (sizes differ by at most one)."""
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _all_gather_rows(dist, group, local: np.ndarray, total_rows: int, world: int) -> np.ndarray:
    """Concatenation, in rank order, of every rank's rows (row counts from `partition`)."""
    import torch
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    rows = [partition(total_rows, world, r) for r in range(world)]
    most = max(hi - lo for lo, hi in rows)
    buf = np.zeros((most, width), dtype=np.float64)
    buf[:local.shape[0]] = local.reshape(local.shape[0], width)
    backend = dist.get_backend(group)
    device = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    send = torch.from_numpy(buf).to(device)
    parts = [torch.empty_like(send) for _ in range(world)]
    dist.all_gather(parts, send, group=group)
    out = [parts[r].cpu().numpy()[:hi - lo] for r, (lo, hi) in enumerate(rows)]
    res = np.concatenate(out, axis=0)
    return res.reshape((total_rows,) + local.shape[1:]) if local.ndim > 1 else res.reshape(total_rows)


def trajectory_values(sim, circuit, observables: Sequence[PauliString], trajectories: int, stream: np.ndarray,
                      dist, group=None) -> dict:
    """Per-trajectory observable values of `trajectories` trajectories drawing in reference
    order from `stream` (trajectories * D values, D = circuit.MaxDraws()), computed across the
    ranks of `group`; every rank returns the full arrays."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    D = circuit.MaxDraws()
    nterms = len(observables)
    values = np.zeros((trajectories, nterms))
    masses = np.zeros(trajectories)
    consumed = np.zeros(trajectories)
    start, offset, rounds = 0, 0, 0
    while start < trajectories:
        rounds += 1
        count = trajectories - start
        lo, hi = partition(count, world, rank)
        rows = stream[offset + lo * D:offset + hi * D].reshape(hi - lo, D)
        if hi > lo:
            part = sim.RunBatch(circuit, rows, observables)
            pv = part.values if part.values is not None else np.zeros((hi - lo, nterms))
            pm, pc = part.masses, part.consumed.astype(np.float64)
        else:
            pv, pm, pc = np.zeros((0, nterms)), np.zeros(0), np.zeros(0)
        all_c = _all_gather_rows(dist, group, pc, count, world)
        all_v = _all_gather_rows(dist, group, pv, count, world) if nterms else np.zeros((count, 0))
        all_m = _all_gather_rows(dist, group, pm, count, world)
        short = np.nonzero(all_c != D)[0]
        keep = count if short.size == 0 else int(short[0]) + 1
        values[start:start + keep] = all_v[:keep]
        masses[start:start + keep] = all_m[:keep]
        consumed[start:start + keep] = all_c[:keep]
        offset += int(all_c[:keep].sum())
        start += keep
    return {"values": values, "masses": masses, "consumed": consumed.astype(np.int64), "rounds": rounds}


def vqe_batch(evaluator, circuit, hamiltonian, parameters: np.ndarray, dist, group=None,
              with_gradient: bool = True) -> tuple[np.ndarray, np.ndarray | None]:
    """Energies (and gradients) of every parameter vector, the vectors split across the ranks."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    params = np.atleast_2d(np.asarray(parameters, dtype=np.float64))
    vectors = params.shape[0]
    lo, hi = partition(vectors, world, rank)
    if hi > lo:
        r = evaluator.EvaluateBatch(circuit, hamiltonian, params[lo:hi], withGradient=with_gradient)
        e, g = r.Energies, r.Gradients
    else:
        e = np.zeros(0)
        g = np.zeros((0, params.shape[1])) if with_gradient else None
    energies = _all_gather_rows(dist, group, e, vectors, world)
    grads = _all_gather_rows(dist, group, g, vectors, world) if with_gradient else None
    return energies, grads
