"""Independent systems across GPUs: one process per GPU, each solving its
share of the systems in one batch (cf_batch_*), with no collective on the
data path.  The only exchange is the final gather of the per-system
statuses to rank 0.

A single system is never split: the reference rejects coupled interfaces
(src/metal4Foam/solvers/metalFoamSolver.C:89-99), so there is no halo to
exchange.  Systems are assigned by longest-processing-time-first bin
packing on the bytes of one SpMV of each system, the quantity that bounds
every phase of an iteration.

    shards = partition([spmv_bytes(s.n, s.nf) for s in systems], world)
    mine = shards[rank]
    records = solve_sharded(systems, rank, world, solve_fn)   # rank 0: all
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence

__all__ = ["spmv_bytes", "partition", "perf_record", "gather_records", "solve_sharded",
           "batch_solve_fn", "ShardError"]

PERF_FIELDS = ("converged", "nIterations", "nRestarts", "initialResidual", "finalResidual",
               "singular", "stagnated", "deflated", "normFactor")


class ShardError(RuntimeError):
    """A rank failed while solving its share; raised on rank 0 after the
    gather, naming the failed ranks and their systems."""


def spmv_bytes(n: int, nf: int, s: int = 4, sym: bool = True) -> int:
    """Bytes of one FP32 LDU SpMV with the reference's access pattern: diag,
    x, y and the face coefficients once, plus the five int32 addressing
    arrays (uppAddr, lowAddr, losort, ownStart, losortStart)."""
    return s * (3 * n + nf * (1 if sym else 2)) + 4 * (3 * nf + 2 * (n + 1))


def partition(weights: Sequence[float], nranks: int) -> List[List[int]]:
    """Longest-processing-time-first: systems in decreasing weight (ties by
    index) go to the least-loaded rank (ties by rank).  Deterministic, so
    every rank computes the same assignment without communicating.  The
    heaviest share is at most 4/3 of the optimum."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    loads = [0.0] * nranks
    shares: List[List[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (loads[k], k))
        shares[r].append(i)
        loads[r] += float(weights[i])
    return [sorted(s) for s in shares]


def perf_record(p) -> Dict[str, float]:
    """Plain-dict status of one solve (cf_performance or any object with the
    same attribute names; a missing flag reads as False)."""
    flags = ("converged", "singular", "stagnated", "deflated")
    return {f: (bool(getattr(p, f, False)) if f in flags else getattr(p, f)) for f in PERF_FIELDS}


def gather_records(indices: Sequence[int], records: Optional[Sequence[dict]], nsystems: int,
                   rank: int, world: int, error: Optional[str] = None,
                   group=None) -> Optional[List[dict]]:
    """Gather (index, record) pairs of every rank to rank 0 and return the
    records in global system order there (None on the other ranks).  Every
    rank calls it exactly once per solve, also when its own solve failed
    (error set): rank 0 then raises ShardError."""
    payload = {"rank": rank, "indices": list(indices),
               "records": list(records) if records is not None else None, "error": error}
    if world == 1:
        gathered = [payload]
    else:
        import torch.distributed as dist
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    failed = [g for g in gathered if g["error"] is not None]
    if failed:
        raise ShardError("; ".join(f"rank {g['rank']} (systems {g['indices']}): {g['error']}"
                                   for g in failed))
    out: List[Optional[dict]] = [None] * nsystems
    for g in gathered:
        if len(g["records"]) != len(g["indices"]):
            raise ShardError(f"rank {g['rank']} returned {len(g['records'])} records for "
                             f"{len(g['indices'])} systems")
        for i, rec in zip(g["indices"], g["records"]):
            if out[i] is not None:
                raise ShardError(f"system {i} solved on more than one rank")
            out[i] = dict(rec, rank=g["rank"])
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ShardError(f"systems {missing} were not solved on any rank")
    return out  # type: ignore[return-value]


def solve_sharded(systems: Sequence, rank: int, world: int,
                  solve_fn: Callable[[List[int]], Sequence], weights=None,
                  group=None) -> Optional[List[dict]]:
    """Solve this rank's share and gather every status to rank 0.

    ``solve_fn(indices)`` solves the systems with those global indices (an
    empty list is possible when there are more ranks than systems) and
    returns one performance object per index.  An exception in it is
    caught, reported through the gather and raised on rank 0 as ShardError,
    so the other ranks never wait on a rank that left."""
    if weights is None:
        weights = [spmv_bytes(s.n, s.nf) for s in systems]
    mine = partition(weights, world)[rank]
    records, error = None, None
    try:
        records = [perf_record(p) for p in solve_fn(mine)] if mine else []
    except Exception as e:  # reported on rank 0 after the gather
        error = f"{type(e).__name__}: {e}"
    return gather_records(mine, records, len(systems), rank, world, error, group)


def batch_solve_fn(systems: Sequence, psis: Sequence, sources: Sequence, options,
                   device: int = 0, reorder: str = "auto", stream_handle=None):
    """solve_fn for :func:`solve_sharded` on a GPU: the share becomes one
    cf_batch (host arrays; psis updated in place)."""
    from . import _lib

    def run(indices: List[int]):
        bt = _lib.Batch(device)
        try:
            if stream_handle is not None:
                bt.set_stream(stream_handle)
            for i in indices:
                bt.add_system(systems[i].addr)
            bt.finalize(reorder)
            for k, i in enumerate(indices):
                bt.set_coeffs(k, systems[i].diag, systems[i].upper)
            return bt.solve([psis[i] for i in indices], [sources[i] for i in indices], options)
        finally:
            bt.close()
    return run
