"""Replica runs on several GPUs: one process per GPU, each running the whole
BFS of its own copy of the graph, then one exchange of results.

The reference splits ONE search across GPUs by state ownership
(multigpubfs/launch.py:350-378, one `graph-rank` process per GPU) and, after
the run, requires every rank to report the same layer table
(multigpubfs/launch.py:398-405).  This engine's path does not shard one
search (a layer's visited test needs the whole bitmap or table), so `--gpus N`
runs N independent replicas; what the ranks still share is that check and the
timing rule: the job's time is the slowest rank's device time.

Everything here is host logic over `torch.distributed`; it runs on NCCL with
CUDA tensors in the benchmark and on gloo with CPU tensors in the tests.
"""
from __future__ import annotations

import hashlib
import struct

TABLE_WORDS = 4  # depth, total (mod 2^62), two 62-bit halves of a SHA-256 of the table


class ReplicaMismatch(RuntimeError):
    """Ranks disagree on the layer table (LAYER_CONSENSUS_MISMATCH)."""


def table_digest(layer_sizes) -> list[int]:
    """Fixed-size signature of a layer table: equal tables give equal words."""
    raw = b"".join(struct.pack("<Q", int(s)) for s in layer_sizes)
    h = hashlib.sha256(raw).digest()
    mask = (1 << 62) - 1
    return [len(layer_sizes), sum(int(s) for s in layer_sizes) & mask,
            int.from_bytes(h[:8], "little") & mask, int.from_bytes(h[8:16], "little") & mask]


def exchange(layer_sizes, device_seconds: float, successors: int, *, device=None, group=None) -> dict:
    """All ranks call this once, in the same order, after their timed runs.

    Returns the job view every rank agrees on: the slowest rank's device time,
    the successors all ranks processed, and the world size.  Raises
    ReplicaMismatch on every rank if any two ranks' tables differ."""
    import torch
    import torch.distributed as dist

    dev = device if device is not None else torch.device("cpu")
    world = dist.get_world_size(group)
    mine = torch.tensor(table_digest(layer_sizes), dtype=torch.int64, device=dev)
    every = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(every, mine, group=group)
    t = torch.tensor([float(device_seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    s = torch.tensor([int(successors)], dtype=torch.int64, device=dev)
    dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    rows = [tuple(int(x) for x in e.cpu().tolist()) for e in every]
    if any(r != rows[0] for r in rows):
        bad = [k for k, r in enumerate(rows) if r != rows[0]]
        raise ReplicaMismatch(f"LAYER_CONSENSUS_MISMATCH: ranks {bad} differ from rank 0")
    return {"world": world, "device_seconds_max": float(t.item()), "successors_total": int(s.item())}
