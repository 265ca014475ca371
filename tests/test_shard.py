"""Independent systems across ranks (metal4foam_b200.shard): the bin
packing, and the gather of statuses over world-size-2 gloo process groups
on the CPU, with the oracle's CPU restatement of the driver standing in for
each rank's GPU batch."""
import os
import socket

import numpy as np
import pytest

from metal4foam_b200 import mesh, shard


def small_systems():
    return [mesh.poisson2d(12, 10, seed=1), mesh.varcoeff3d((6, 5, 4), seed=2),
            mesh.varcoeff3d((9, 8), seed=3, permute=False), mesh.poisson2d(20, 7, seed=4),
            mesh.varcoeff3d((4, 4, 4), seed=5), mesh.varcoeff3d((7, 6, 5), seed=6)]


def test_spmv_bytes_matches_formula():
    # 128^3 varcoeff: 141.8 MB (FP32 symmetric), 192.0 MB (FP64)
    n, nf = 2097152, 6242304
    assert shard.spmv_bytes(n, nf) == 4 * (3 * n + nf) + 4 * (3 * nf + 2 * (n + 1))
    assert round(shard.spmv_bytes(n, nf) / 1e6, 1) == 141.8
    assert round(shard.spmv_bytes(n, nf, 8) / 1e6, 1) == 192.0


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8, 64])
def test_partition_properties(nranks):
    rng = np.random.default_rng(nranks)
    w = list(10 ** rng.uniform(3, 6, 48))
    parts = shard.partition(w, nranks)
    assert len(parts) == nranks
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(48))
    assert parts == shard.partition(w, nranks)          # deterministic
    loads = [sum(w[i] for i in p) for p in parts]
    lower = max(max(w), sum(w) / nranks)
    assert max(loads) <= sum(w) / nranks + max(w) + 1e-6   # list-scheduling bound
    assert max(loads) >= lower - 1e-6
    if nranks > 48:
        assert sum(1 for p in parts if not p) == nranks - 48


def test_partition_lpt_known_case():
    # LPT on {7,6,5,4,3,2} over 2 ranks: 7->0, 6->1, 5->1, 4->0, 3->0, 2->1
    assert shard.partition([7, 6, 5, 4, 3, 2], 2) == [[0, 3, 4], [1, 2, 5]]
    assert shard.partition([1, 1, 1], 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def test_partition_batched_configuration_balance():
    systems = mesh.batched_systems()
    w = [shard.spmv_bytes(s.n, s.nf) for s in systems]
    for nr in (2, 4, 8):
        loads = [sum(w[i] for i in p) for p in shard.partition(w, nr)]
        # the largest system alone bounds the heaviest share from below
        assert max(loads) <= max(max(w), sum(w) / nr) * 4 / 3 + 1


def fake_solve_fn(systems, oracle_mod, fail_on=None):
    def run(indices):
        if fail_on is not None and fail_on in indices:
            raise RuntimeError(f"injected failure on system {fail_on}")
        return [oracle_mod.metal_solve(systems[i], maxIter=2000) for i in indices]
    return run


def test_single_rank_gather_in_global_order(oracle):
    systems = small_systems()
    recs = shard.solve_sharded(systems, 0, 1, fake_solve_fn(systems, oracle))
    assert len(recs) == len(systems)
    for s, r in zip(systems, recs):
        ref = oracle.metal_solve(s, maxIter=2000)
        assert r["nIterations"] == ref.nIterations and r["converged"] and r["rank"] == 0


def free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _worker(rank, world, port, fail_on, out_path):
    import datetime
    import json

    import torch.distributed as dist

    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    systems = small_systems()
    result = {"rank": rank}
    try:
        recs = shard.solve_sharded(systems, rank, world,
                                   fake_solve_fn(systems, O, fail_on if rank == 1 else None))
        result["records"] = recs
    except shard.ShardError as e:
        result["shard_error"] = str(e)
    finally:
        dist.destroy_process_group()
    with open(out_path + f".{rank}", "w") as f:
        json.dump(result, f)


def run_two_ranks(tmp_path, fail_on):
    import json

    import torch.multiprocessing as mp
    out = str(tmp_path / "res")
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fail_on, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    return [json.load(open(out + f".{r}")) for r in range(2)]


def test_gloo_two_ranks_gather(tmp_path, oracle):
    res = run_two_ranks(tmp_path, None)
    assert res[1].get("records") is None and "shard_error" not in res[1]
    recs = res[0]["records"]
    systems = small_systems()
    parts = shard.partition([shard.spmv_bytes(s.n, s.nf) for s in systems], 2)
    assert all(parts)
    for i, (s, r) in enumerate(zip(systems, recs)):
        assert r["rank"] == (0 if i in parts[0] else 1)
        ref = oracle.metal_solve(s, maxIter=2000)
        assert r["nIterations"] == ref.nIterations
        assert r["finalResidual"] == ref.finalResidual and r["converged"]


def test_gloo_rank_failure_reported_on_rank0(tmp_path):
    """A rank whose solve raises still takes part in the gather; rank 0
    raises ShardError naming it, and no rank waits for ever."""
    systems = small_systems()
    parts = shard.partition([shard.spmv_bytes(s.n, s.nf) for s in systems], 2)
    victim = parts[1][0]
    res = run_two_ranks(tmp_path, victim)
    assert "rank 1" in res[0]["shard_error"]
    assert f"injected failure on system {victim}" in res[0]["shard_error"]
    assert "shard_error" not in res[1]
