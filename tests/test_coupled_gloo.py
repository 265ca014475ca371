"""The subdomains' communication over torch.distributed (metal4foam_b200.
coupled.TorchComm) on world-size-2 and -3 gloo process groups on the CPU: the
callbacks the subdomain solver calls -- the global sum/max and the halo
exchange -- driven with host buffers, and an FP64 matrix-vector product of
a decomposed system assembled from them (each rank: its internal product
via the oracle, the neighbour's values across the interface from the
exchange) equal to the unsplit product.  The same callbacks move device
buffers over NCCL on GPUs."""
import ctypes as C
import json
import os
import socket

import numpy as np
import pytest


def free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _system():
    from metal4foam_b200 import mesh
    return mesh.varcoeff3d((7, 6, 5), seed=11, permute=True)


def _worker(rank, world, port, out_path):
    import datetime

    import torch.distributed as dist

    from metal4foam_b200 import _lib, coupled, decompose
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    res = {"rank": rank}
    try:
        comm = coupled.TorchComm(on_device=False)
        cb = comm.comm
        # global sum and max of host doubles
        v = np.array([1.5 + rank, -2.0 * rank, 10.0 ** rank], np.float64)
        rc = cb.allreduce(None, v.ctypes.data, 3, 0, None)
        res["sum"] = [rc] + v.tolist()
        w = np.array([rank + 0.25, -rank], np.float64)
        rc = cb.allreduce(None, w.ctypes.data, 2, 1, None)
        res["max"] = [rc] + w.tolist()
        # one FP64 A x over the decomposed system
        s = _system()
        part = np.random.default_rng(3).integers(0, world, s.n).astype(np.int32)
        subs = decompose.decompose(s, part, world)
        me = subs[rank]
        x = np.random.default_rng(4).standard_normal(s.n)
        xl = np.ascontiguousarray(x[me.cells])
        nb, nfc, fc, cf = me.interface_arrays()
        send = [np.ascontiguousarray(xl[i.faceCells]) for i in me.interfaces]
        recv = [np.empty(len(i.faceCells)) for i in me.interfaces]
        sp = (C.c_void_p * len(send))(*[a.ctypes.data for a in send])
        rp = (C.c_void_p * len(recv))(*[a.ctypes.data for a in recv])
        rc = cb.exchange(None, len(nb), nb.ctypes.data, nfc.ctypes.data, 8, sp, rp, None)
        y = O.amul(me.system, xl)
        for itf, h in zip(me.interfaces, recv):
            for k in range(len(itf.faceCells)):
                y[itf.faceCells[k]] -= itf.coeffs[k] * h[k]
        ref = O.amul(s, x)[me.cells]
        res["exchange_rc"] = rc
        res["amul_err"] = float(np.max(np.abs(y - ref)) / np.max(np.abs(ref)))
        # FP32 halo too (the Krylov vectors), from every neighbour
        s32 = [a.astype(np.float32) for a in send]
        r32 = [np.empty(len(i.faceCells), np.float32) for i in me.interfaces]
        sp = (C.c_void_p * len(s32))(*[a.ctypes.data for a in s32])
        rp = (C.c_void_p * len(r32))(*[a.ctypes.data for a in r32])
        rc = cb.exchange(None, len(nb), nb.ctypes.data, nfc.ctypes.data, 4, sp, rp, None)
        ok = rc == 0 and len(me.interfaces) == world - 1
        for itf, got in zip(me.interfaces, r32):
            other = subs[itf.neighbour]
            back = next(i for i in other.interfaces if i.neighbour == rank)
            ok = ok and np.array_equal(got, x[other.cells][back.faceCells].astype(np.float32))
        res["exchange32_ok"] = bool(ok)
    finally:
        dist.destroy_process_group()
    with open(out_path + f".{rank}", "w") as f:
        json.dump(res, f)


@pytest.mark.parametrize("world", [2, 3])
def test_torch_comm_gloo_ranks(tmp_path, world):
    """2 ranks (one interface each) and 3 ranks (a random split: every rank
    has an interface with each of the two others)."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "res")
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = [json.load(open(out + f".{r}")) for r in range(world)]
    for r in res:
        assert r["sum"] == [0, sum(1.5 + k for k in range(world)),
                            sum(-2.0 * k for k in range(world)),
                            sum(10.0 ** k for k in range(world))]
        assert r["max"] == [0, world - 1 + 0.25, 0.0]
        assert r["exchange_rc"] == 0
        assert r["amul_err"] < 1e-13
        assert r["exchange32_ok"]
