"""Transports for the halo exchange of a partitioned mesh.

The library packs the shared nodes into a send buffer and calls back into
the transport, which moves every neighbour's range of the buffer as
src/lib_sod2d/sources/mod_comms.f90:1049-1102 (mpi_base_comms_*_ncclSendRcv)
does: send buffer range i to rank ranksToComm(i), receive the same range of
the receive buffer from it.  The library then sums each shared node over its
ranks in ascending rank order.

- `DistHaloTransport`: torch.distributed point-to-point, one process per
  GPU (NCCL over NVLink on CUDA tensors; gloo on CPU tensors).  The
  library's stream must be torch's current stream, so that the sends follow
  the pack kernel and the sum kernel follows the receives.
- `LocalHaloGroup`: every part in one process, one host thread per part,
  used to run the partitioned path on a single device.  The exchange is a
  device-to-device copy between the parts' buffers; the threads meet at a
  barrier bounded by a timeout before and after the copies.  No kernel
  waits on another.

Both also provide allreduce(rank, tensor, kind) for the global reductions
of the explicit step (min / max of float32, sum of float64), the
reference's MPI_Allreduce calls.
"""
from __future__ import annotations

import threading

from .partition import HaloPlan


class DistHaloTransport:
    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group

    def _peer(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def allreduce(self, rank: int, t, kind: int) -> None:
        ops = (self.dist.ReduceOp.MIN, self.dist.ReduceOp.MAX, self.dist.ReduceOp.SUM)
        self.dist.all_reduce(t, op=ops[kind], group=self.group)

    def exchange(self, plan: HaloPlan, send, recv, width: int) -> None:
        dist = self.dist
        ops = []
        for nb, pos, size in zip(plan.ranksToComm.tolist(), plan.commsMemPosInLoc.tolist(),
                                 plan.commsMemSize.tolist()):
            a, b = (pos - 1) * width, (pos - 1 + size) * width
            ops.append(dist.P2POp(dist.irecv, recv[a:b], self._peer(nb), self.group))
            ops.append(dist.P2POp(dist.isend, send[a:b], self._peer(nb), self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class LocalHaloGroup:
    def __init__(self, plans: list[HaloPlan], timeout: float = 120.0):
        self.plans = {p.rank: p for p in plans}
        self.send = {}
        self.red = {}
        self.barrier = threading.Barrier(len(plans), timeout=timeout)

    def register(self, rank: int, send) -> None:
        self.send[rank] = send

    def allreduce(self, rank: int, t, kind: int) -> None:
        """min (0), max (1) or sum (2) over the parts, combined in ascending
        rank order so every part gets the same bits."""
        import torch
        self._sync(t)
        self.red[rank] = t.clone()
        self.barrier.wait()  # every part has posted its value
        vals = [self.red[r] for r in sorted(self.red)]
        acc = vals[0].clone()
        for v in vals[1:]:
            acc = torch.minimum(acc, v) if kind == 0 else (torch.maximum(acc, v) if kind == 1 else acc + v)
        t.copy_(acc)
        self._sync(t)
        self.barrier.wait()  # every part has read the others' values

    def _sync(self, t) -> None:
        if t.is_cuda:
            import torch
            torch.cuda.synchronize(t.device)

    def exchange(self, plan: HaloPlan, send, recv, width: int) -> None:
        self._sync(send)
        self.barrier.wait()  # every part has packed
        for nb, pos, size in zip(plan.ranksToComm.tolist(), plan.commsMemPosInLoc.tolist(),
                                 plan.commsMemSize.tolist()):
            pa, pb = self.plans[nb].range_of(plan.rank)
            if pb - pa != size:
                raise RuntimeError(f"halo plans of ranks {plan.rank} and {nb} disagree")
            recv[(pos - 1) * width:(pos - 1 + size) * width].copy_(self.send[nb][pa * width:pb * width])
        self._sync(recv)
        self.barrier.wait()  # every part has read its neighbours' buffers

    def run(self, fns) -> list:
        """Run fns[r]() in one thread per part; re-raise the first error."""
        out, errs = [None] * len(fns), []

        def body(r):
            try:
                out[r] = fns[r]()
            except BaseException as e:  # noqa: BLE001 - reported to the caller below
                errs.append(e)
                self.barrier.abort()

        th = [threading.Thread(target=body, args=(r,)) for r in range(len(fns))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        if errs:
            raise errs[0]
        return out
