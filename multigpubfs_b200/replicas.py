"""Runs on several GPUs, one process per GPU, with no collective on the data
path: N replicas of one single-graph BFS (their tables checked against each
other once, after the runs), or a batched sweep whose instances are split
between the ranks by work and whose tables are gathered to rank 0.

The reference splits ONE search across GPUs by state ownership
(multigpubfs/launch.py:350-378, one `graph-rank` process per GPU) and, after
the run, requires every rank to report the same layer table
(multigpubfs/launch.py:398-405).  The owner-partitioned split of one search
is multigpubfs_b200.sharded (the bench's `s13-lrx-sharded`); the single-graph
workloads here run N independent replicas of the fused engine, and what the
ranks share is that table check and the timing rule: the job's time is the
slowest rank's device time.

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


# ---------------------------------------------------------------------------
# Batched sweeps on several GPUs: the instances are independent, so each rank
# takes a share of them and runs it as its own waves, with no exchange on the
# data path; rank 0 gathers the tables afterwards.

def partition_instances(work, world: int) -> list[int]:
    """Owner rank of every instance, balancing the summed `work` (e.g. the
    exact successor count g * |G| of each instance) over `world` ranks: the
    largest instances first, each to the least-loaded rank (ties: lower rank,
    lower instance index), so the split is deterministic on every rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    owner = [0] * len(work)
    for i in sorted(range(len(work)), key=lambda k: (-int(work[k]), k)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += int(work[i])
    return owner


def gather_tables(ids, tables, count: int, *, device=None, group=None):
    """All ranks call this once, in the same order.  `ids` are the instance
    indices this rank ran and `tables` their layer tables.  Rank 0 returns the
    `count` tables ordered by instance index; the other ranks return None.
    Raises on rank 0 if an instance is missing or reported twice."""
    import torch
    import torch.distributed as dist

    dev = device if device is not None else torch.device("cpu")
    world = dist.get_world_size(group)
    flat = []
    for i, t in zip(ids, tables):
        flat += [int(i), len(t)] + [int(x) for x in t]
    size = torch.tensor([len(flat)], dtype=torch.int64, device=dev)
    sizes = [torch.empty_like(size) for _ in range(world)]
    dist.all_gather(sizes, size, group=group)
    longest = max(int(s.item()) for s in sizes)
    mine = torch.full((max(longest, 1),), -1, dtype=torch.int64, device=dev)
    if flat:
        mine[:len(flat)] = torch.tensor(flat, dtype=torch.int64, device=dev)
    every = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(every, mine, group=group)
    if dist.get_rank(group) != 0:
        return None
    out = [None] * count
    for r, buf in enumerate(every):
        words = buf[:int(sizes[r].item())].cpu().tolist()
        k = 0
        while k < len(words):
            i, n = words[k], words[k + 1]
            if not 0 <= i < count or out[i] is not None:
                raise RuntimeError(f"GATHER_INSTANCE {i} from rank {r}")
            out[i] = words[k + 2:k + 2 + n]
            k += 2 + n
    missing = [i for i, t in enumerate(out) if t is None]
    if missing:
        raise RuntimeError(f"GATHER_MISSING {missing[:8]}")
    return out
