"""Decomposed solves across processes: the cf_comm callbacks over
torch.distributed.

One process per subdomain (one per GPU), launched like any torch.distributed
job.  The subdomain solver (cf_subdomain_solve) calls back for every global
sum and every halo exchange; :class:`TorchComm` implements both with
torch.distributed collectives on the buffers the solver hands over:

* allreduce: ``all_reduce`` (SUM or MAX) in place;
* exchange: one ``isend``/``irecv`` pair per interface, all posted together
  (``batch_isend_irecv``) and completed before returning.

With NCCL the buffers are device memory on the subdomain's GPU and the
collectives are ordered on torch's current stream, which the subdomain is
told to use (:func:`solve_subdomain`).  With gloo the same callbacks move
host memory, which is how the host-side logic is exercised on CPU ranks.
A callback never lets an exception cross into the C library: it returns a
non-zero status, and the solve fails with CF_ERR_CUDA.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class _Cai:
    """A device buffer seen through __cuda_array_interface__."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def _view(ptr, count, elem_bytes, on_device, torch):
    """A torch tensor over `count` elements at `ptr` (no copy)."""
    if count == 0:
        return None
    if on_device:
        typestr = "<f8" if elem_bytes == 8 else "<f4"
        return torch.as_tensor(_Cai(ptr, count, typestr), device="cuda")
    ctype = C.c_double if elem_bytes == 8 else C.c_float
    arr = np.ctypeslib.as_array((ctype * int(count)).from_address(int(ptr)))
    return torch.from_numpy(arr)


class TorchComm:
    """cf_comm over a torch.distributed process group: every rank is one
    subdomain, subdomain numbers are group ranks.  `on_device`: the solver
    hands device buffers (NCCL); otherwise host buffers (gloo, or any
    backend without device support: the library stages the copies)."""

    def __init__(self, group=None, on_device: bool = True):
        import torch
        import torch.distributed as dist
        self.torch = torch
        self.dist = dist
        self.group = group
        self.on_device = on_device
        self.failed = None
        self._cb_allreduce = _lib.ALLREDUCE_FN(self._allreduce)
        self._cb_exchange = _lib.EXCHANGE_FN(self._exchange)
        self._cb_abort = _lib.ABORT_FN(self._abort)
        self.comm = _lib.Comm(None, self._cb_allreduce, self._cb_exchange, self._cb_abort,
                              0 if on_device else 1)

    def _allreduce(self, user, values, count, op, stream):
        try:
            t = _view(values, count, 8, self.on_device, self.torch)
            if t is not None:
                red = self.dist.ReduceOp.MAX if op == 1 else self.dist.ReduceOp.SUM
                self.dist.all_reduce(t, op=red, group=self.group)
            return 0
        except Exception as e:  # noqa: BLE001 -- no exception may cross the C ABI
            self.failed = e
            return 1

    def _exchange(self, user, nif, neighbour, nfaces, elem_bytes, send, recv, stream):
        try:
            nb = np.ctypeslib.as_array((C.c_int32 * nif).from_address(neighbour)) if nif else []
            nfc = np.ctypeslib.as_array((C.c_int32 * nif).from_address(nfaces)) if nif else []
            sp = (C.c_void_p * nif).from_address(send) if nif else []
            rp = (C.c_void_p * nif).from_address(recv) if nif else []
            ops = []
            for p in range(nif):
                if nfc[p] == 0:
                    continue
                peer = int(nb[p])
                if self.group is not None:
                    peer = self.dist.get_global_rank(self.group, peer)
                st = _view(sp[p], nfc[p], elem_bytes, self.on_device, self.torch)
                rt = _view(rp[p], nfc[p], elem_bytes, self.on_device, self.torch)
                ops.append(self.dist.P2POp(self.dist.isend, st, peer, self.group))
                ops.append(self.dist.P2POp(self.dist.irecv, rt, peer, self.group))
            if ops:
                for w in self.dist.batch_isend_irecv(ops):
                    w.wait()
            return 0
        except Exception as e:  # noqa: BLE001
            self.failed = e
            return 1

    def _abort(self, user):
        self.failed = self.failed or RuntimeError("this subdomain's solve failed")


def solve_subdomain(solver, sub_solver, psi, source, options, comm: TorchComm):
    """cf_subdomain_solve on torch's current stream (the stream the NCCL
    collectives are ordered on)."""
    import torch
    if comm.on_device:
        sub_solver.set_stream(torch.cuda.current_stream().cuda_stream)
    return sub_solver.solve(solver, psi, source, options, comm.comm)
