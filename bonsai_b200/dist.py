"""Host side of a row-sharded fit over torch.distributed ranks (one GPU each).

Which rows a rank holds (`shard_range`), the fit's initial score as ONE
float serial sum of the labels in row order, chained through the ranks so it
equals a one-process fit's bit for bit (`chained_label_sum`), and the NCCL id
rank 0 makes for the others (`share_comm_id`). The device side is
`bonsai_b200.Comm` + `Booster(..., comm=...)`.
"""

from __future__ import annotations

import numpy as np

from . import Comm, init_score_from_sum, label_sum, shard_range

__all__ = ["shard_range", "chained_label_sum", "share_comm_id", "sharded_init_score",
           "open_comm"]


def _device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def chained_label_sum(labels_shard, world: int, rank: int) -> np.float32:
    """std::accumulate over the fit's labels in row order, the shards holding
    consecutive ranges: rank r continues rank r - 1's running float sum over
    its own labels and passes it on; the last rank's total goes to all."""
    if world == 1:
        return label_sum(labels_shard)
    import torch
    import torch.distributed as dist
    dev = _device()
    run = torch.zeros(1, dtype=torch.float32, device=dev)
    if rank > 0:
        dist.recv(run, src=rank - 1)
    s = label_sum(labels_shard, float(run.item()))
    if rank + 1 < world:
        dist.send(torch.tensor([s], dtype=torch.float32, device=dev), dst=rank + 1)
    total = torch.tensor([s], dtype=torch.float32, device=dev)
    dist.broadcast(total, src=world - 1)
    return np.float32(total.item())


def sharded_init_score(labels_shard, n_rows: int, objective: str, world: int,
                       rank: int) -> np.float32:
    """The fit's initial score, identical on every rank and to a one-process
    fit's (bb_booster_create's float serial sum, then mean or log-odds)."""
    return init_score_from_sum(chained_label_sum(labels_shard, world, rank), n_rows, objective)


def share_comm_id(world: int, rank: int, make=Comm.unique_id) -> bytes:
    """Rank 0's NCCL unique id, on every rank."""
    if world == 1:
        return make()
    import torch.distributed as dist
    box = [make() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0)
    return box[0]


def open_comm(world: int, rank: int) -> Comm:
    """This rank's member of an NCCL communicator over the job's ranks."""
    return Comm.nccl(share_comm_id(world, rank), world, rank)
