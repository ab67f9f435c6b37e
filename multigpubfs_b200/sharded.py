"""One BFS split across ranks by state ownership: each rank (one process per
GPU) owns a slice of the Lehmer bitmap and the part of every layer that falls
in it, and the ranks exchange routed children once per layer chunk.

Partition (mgbfs2_shard_geometry): prefix block s -- the states whose first
`prefix` Lehmer digits give s, (n - prefix)! consecutive ranks -- belongs to
rank s mod world, which stores it as local block s // world.  Per layer,
every rank:

1. route: expands its frontier, chunk by chunk, and writes each child to its
   owner's buckets (mgbfs2_shard_route; owner-major, block-minor);
2. exchange: an all-to-all of the per-(owner, block) counts, then an
   all-to-all of the words with those counts as split sizes;
3. accept: claims what it received in its slice (mgbfs2_shard_accept); the
   winners are its part of the next layer;
4. the layer size is the all-reduced sum of the winners; the search ends at 0.

Every rank takes the same collectives in the same order: the number of chunks
of a layer is the all-reduced maximum, and a rank with fewer sends empty
buckets.  Reference: the owner route / exchange / accept loop of
crates/mgbfs-runtime/src/generic_distributed_native.rs:199-285, the grouped
send/recv of its NCCL transport (nccl_transport.cpp:670-778) and the count
all-gather and error all-reduce (:295-297).

`ShardedBfs` drives any number of local shards through an exchange:
`DistExchange` (one shard per process, torch.distributed: NCCL with CUDA
tensors, gloo with CPU tensors) or `LocalExchange` (every rank's shard in one
process, the exchange done by copies; on one GPU this runs the partitioned
path with all of its kernels).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

from . import native
from .graph_definition import GraphDefinition


@dataclass(frozen=True)
class Geometry:
    degree: int
    world: int
    prefix: int
    blocks_per_owner: int
    slice_bits: int

    @property
    def block_bits(self) -> int:
        return math.factorial(self.degree - self.prefix)

    @property
    def buckets(self) -> int:
        return self.world * self.blocks_per_owner


def geometry(degree: int, world: int) -> Geometry:
    """The partition of `degree`-symbol states over `world` ranks (host only)."""
    lib = native.load()
    k, b, s = C.c_uint32(), C.c_uint32(), C.c_uint64()
    native.check(lib.mgbfs2_shard_geometry(degree, world, C.byref(k), C.byref(b), C.byref(s)),
                 "mgbfs2_shard_geometry")
    return Geometry(degree, world, k.value, b.value, s.value)


def lehmer_digits(state):
    """Lehmer digits of a permutation of distinct labels (their sorted order
    gives the codes)."""
    order = {v: i for i, v in enumerate(sorted(state))}
    codes = [order[v] for v in state]
    out = []
    for i, c in enumerate(codes):
        out.append(c - sum(1 for x in codes[:i] if x < c))
    return out


def owner_of(state, geo: Geometry) -> tuple[int, int]:
    """(owner rank, bit in the owner's slice) of a state."""
    d = lehmer_digits(state)
    n = len(d)
    block = 0
    for i in range(geo.prefix):
        block = block * (n - i) + d[i]
    tail = 0
    for i in range(geo.prefix, n):
        tail = tail * (n - i) + d[i]
    return block % geo.world, (block // geo.world) * geo.block_bits + tail


def pack_state(state) -> int:
    order = {v: i for i, v in enumerate(sorted(state))}
    word = 0
    for i, v in enumerate(state):
        word |= order[v] << (4 * i)
    return word


def _check_graph(graph: GraphDefinition):
    if graph.action["kind"] != "permutation":
        raise ValueError("SHARDED_REQUIRES_PERMUTATION_ACTION")
    n = len(graph.start)
    if not 2 <= n <= 16 or len(set(graph.start)) != n:
        raise ValueError("SHARDED_REQUIRES_DISTINCT_LABELS_UP_TO_16")


class DeviceShard:
    """One rank's part of the search on a GPU: its bitmap slice, its frontier
    and the buffers of the route and accept calls."""

    def __init__(self, graph: GraphDefinition, rank: int, world: int, device, *, frontier_capacity=None,
                 chunk_parents: int = 1 << 25):
        import torch
        _check_graph(graph)
        self.lib = native.require_device()
        self.torch = torch
        self.rank, self.world = rank, world
        self.device = torch.device(device) if not isinstance(device, torch.device) else device
        self.n = len(graph.start)
        self.geo = geometry(self.n, world)
        gens = graph.action["generators"]
        self.gens = len(gens)
        self.perms = (C.c_uint32 * (self.gens * self.n))(*[int(x) for g in gens for x in g])
        dev = self.device
        self.slice = torch.zeros((self.geo.slice_bits + 63) // 64, dtype=torch.int64, device=dev)
        if frontier_capacity is None:
            free, _ = torch.cuda.mem_get_info(dev)
            frontier_capacity = min(self.geo.slice_bits, max(1024, free // 8 // 8))
        self.capacity = int(frontier_capacity)
        self.front = torch.empty(self.capacity, dtype=torch.int64, device=dev)
        self.next = torch.empty(self.capacity, dtype=torch.int64, device=dev)
        self.count = 0
        # Chunks start at multiples of 32 entries: the route call needs a
        # 16-byte aligned frontier, and whole warps of parents coalesce.
        self.chunk_parents = max(32, (int(chunk_parents) + 31) // 32 * 32)
        self.out = torch.empty(0, dtype=torch.int64, device=dev)
        self.bucket_counts = torch.zeros(self.geo.buckets, dtype=torch.int64, device=dev)
        self.next_count = torch.zeros(1, dtype=torch.int64, device=dev)
        self.error = torch.zeros(1, dtype=torch.int32, device=dev)
        self.scratch = torch.empty(int(self.lib.mgbfs2_shard_scratch_bytes()), dtype=torch.uint8, device=dev)
        self.appended = 0
        self.launches = 0
        self.start = list(graph.start)
        self.reset()

    def reset(self) -> None:
        """Clears the slice and puts the start state on its owner."""
        self.slice.zero_()
        self.count = self.appended = 0
        owner, bit = owner_of(self.start, self.geo)
        if owner == self.rank:
            self.front[0] = _signed(pack_state(self.start))
            self.count = 1
            self.slice[bit >> 6] = _signed(1 << (bit & 63))

    def chunks(self) -> int:
        return (self.count + self.chunk_parents - 1) // self.chunk_parents

    def route(self, c: int):
        """Routes chunk `c` of the frontier (empty past the last chunk).
        Returns (words, bucket counts), both on the device."""
        lo = min(self.count, c * self.chunk_parents)
        hi = min(self.count, lo + self.chunk_parents)
        need = (hi - lo) * self.gens
        if self.out.numel() < need:
            self.out = self.torch.empty(need, dtype=self.torch.int64, device=self.device)
        stream = native.stream_handle()
        native.check(self.lib.mgbfs2_shard_route(
            self.n, self.gens, self.perms, self.front.data_ptr() + 8 * lo if hi > lo else None, hi - lo,
            self.world, self.out.data_ptr() if need else None, self.out.numel(), self.bucket_counts.data_ptr(),
            self.error.data_ptr(), self.scratch.data_ptr(), self.scratch.numel(), stream), "mgbfs2_shard_route")
        self.launches += 4 if hi > lo else 1  # count, layout, route, publish
        return self.out, self.bucket_counts

    def accept(self, words, counts) -> None:
        """Claims received words (source-major, `counts` per source and local
        block) in the slice; winners are appended to the next layer."""
        room = self.capacity - self.appended
        stream = native.stream_handle()
        # With nothing received any device buffer will do: no word is read.
        incoming = words.data_ptr() if words.numel() else self.next.data_ptr()
        native.check(self.lib.mgbfs2_shard_accept(
            self.n, self.world, self.rank, incoming, counts.data_ptr(), self.slice.data_ptr(),
            self.next.data_ptr() + 8 * self.appended, room, self.next_count.data_ptr(), self.error.data_ptr(),
            self.scratch.data_ptr(), self.scratch.numel(), stream), "mgbfs2_shard_accept")
        self.launches += 3  # layout, accept, publish
        got = int(self.next_count.item())
        if got > room or int(self.error.item()):
            raise RuntimeError(f"SHARD_ACCEPT_FAILED: rank {self.rank}, winners {got}, room {room}, "
                               f"error bits {int(self.error.item()):#x}")
        self.appended += got

    def finish(self) -> int:
        """Ends the layer: the appended winners become the frontier."""
        self.front, self.next = self.next, self.front
        self.count, self.appended = self.appended, 0
        return self.count

    def frontier_words(self):
        """This rank's part of the current layer, packed words without the
        parent-edge tags."""
        words = self.front[:self.count]
        return words if self.n == 16 else words & ((1 << (4 * self.n)) - 1)


def _signed(x: int) -> int:
    return x - (1 << 64) if x >= 1 << 63 else x


class LocalExchange:
    """Every rank's shard in one process: the all-to-all is done by copies."""

    def __init__(self, world: int):
        self.world = world

    def max(self, values):
        return max(values)

    def sum(self, values):
        return sum(values)

    def exchange(self, sends):
        import torch
        world = self.world
        blocks = len(sends[0][1]) // world
        counts = [c.view(world, blocks).cpu() for _, c in sends]          # [source][owner, block]
        totals = [c.sum(dim=1).tolist() for c in counts]                  # [source][owner]
        offsets = [[sum(t[:o]) for o in range(world)] for t in totals]
        out = []
        for o in range(world):
            parts = [sends[r][0][offsets[r][o]:offsets[r][o] + totals[r][o]] for r in range(world)]
            words = torch.cat(parts) if parts else sends[0][0][:0]
            cnt = torch.cat([sends[r][1].view(world, blocks)[o] for r in range(world)])
            out.append((words, cnt))
        return out


class DistExchange:
    """One shard per process over torch.distributed (NCCL with CUDA tensors,
    gloo with CPU tensors)."""

    def __init__(self, group=None, device=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.device = device

    def _reduce(self, value: int, op) -> int:
        import torch
        t = torch.tensor([int(value)], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(t, op=op, group=self.group)
        return int(t.item())

    def max(self, values):
        (v,) = values
        return self._reduce(v, self.dist.ReduceOp.MAX)

    def sum(self, values):
        (v,) = values
        return self._reduce(v, self.dist.ReduceOp.SUM)

    def exchange(self, sends):
        import torch
        ((words, counts),) = sends
        world = self.world
        blocks = counts.numel() // world
        recv_counts = torch.empty_like(counts)
        self.dist.all_to_all_single(recv_counts, counts, group=self.group)
        send_split = counts.view(world, blocks).sum(dim=1).tolist()
        recv_split = recv_counts.view(world, blocks).sum(dim=1).tolist()
        incoming = torch.empty(sum(recv_split), dtype=words.dtype, device=words.device)
        self.dist.all_to_all_single(incoming, words[:sum(send_split)], output_split_sizes=recv_split,
                                    input_split_sizes=send_split, group=self.group)
        return [(incoming, recv_counts)]


class ShardedBfs:
    """Drives local shards (all ranks' in one process, or this rank's) layer
    by layer through an exchange.  `run()` returns the global layer table,
    the same on every rank."""

    def __init__(self, shards, exchange):
        self.shards = list(shards)
        self.exchange = exchange

    def layer(self) -> int:
        chunks = self.exchange.max([s.chunks() for s in self.shards])
        for c in range(chunks):
            sends = [s.route(c) for s in self.shards]
            for s, (words, counts) in zip(self.shards, self.exchange.exchange(sends)):
                s.accept(words, counts)
        return self.exchange.sum([s.finish() for s in self.shards])

    def run(self, max_layers=None) -> list[int]:
        sizes = [self.exchange.sum([s.count for s in self.shards])]
        while sizes[-1] and (max_layers is None or len(sizes) < max_layers):
            size = self.layer()
            if size:
                sizes.append(size)
            else:
                break
        return sizes


def run_emulated(graph: GraphDefinition, world: int, device=0, **shard_options) -> list[int]:
    """All `world` ranks' shards on one GPU in this process."""
    shards = [DeviceShard(graph, r, world, device, **shard_options) for r in range(world)]
    return ShardedBfs(shards, LocalExchange(world)).run()


def run_distributed(graph: GraphDefinition, group=None, device=None, **shard_options) -> list[int]:
    """This rank's shard, the others' in the other processes of `group`."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    shard = DeviceShard(graph, rank, world, dev, **shard_options)
    return ShardedBfs([shard], DistExchange(group, dev)).run()
