"""The owner-partitioned BFS (multigpubfs_b200.sharded) on CPU: the partition
rule of mgbfs2_shard_geometry against a restatement, and the multi-rank
driver (ShardedBfs over DistExchange) on two and three gloo ranks, with a CPU
shard that restates the route and accept contract of mgbfs2_shard_route /
mgbfs2_shard_accept (bucket order, split sizes, slice bits) in Python.  The
layer tables are checked against the oracle."""
import itertools
import math
import multiprocessing as mp
import os
import socket
import traceback

import pytest

from multigpubfs_b200 import sharded
from oracle import graph_oracle as G


def _expected_geometry(n, world):
    prefix = 2 if n >= 4 else 1
    blocks = math.perm(n, prefix)
    per = -(-blocks // world)
    if world * per > 256:
        return None
    return prefix, per, per * math.factorial(n - prefix)


@pytest.mark.parametrize("n", [2, 3, 4, 7, 10, 13, 15, 16])
@pytest.mark.parametrize("world", [1, 2, 3, 5, 8, 16, 40])
def test_geometry_matches_the_partition_rule(n, world):
    want = _expected_geometry(n, world)
    if want is None:
        with pytest.raises(Exception):
            sharded.geometry(n, world)
        return
    g = sharded.geometry(n, world)
    assert (g.prefix, g.blocks_per_owner, g.slice_bits) == want
    assert g.buckets <= 256


@pytest.mark.parametrize("n,world", [(4, 1), (4, 5), (5, 2), (6, 3), (6, 7)])
def test_every_state_has_one_owner_bit(n, world):
    geo = sharded.geometry(n, world)
    seen = set()
    for p in itertools.permutations(range(n)):
        owner, bit = sharded.owner_of(list(p), geo)
        assert 0 <= owner < world and 0 <= bit < geo.slice_bits
        seen.add((owner, bit))
    assert len(seen) == math.factorial(n)


def _unpack(word, n):
    return tuple((word >> (4 * i)) & 15 for i in range(n))


class CpuShard:
    """Python restatement of one rank's device shard (same interface as
    sharded.DeviceShard): route writes children owner-major and block-minor
    with per-(owner, block) counts; accept claims source-major received words
    and checks each lies in the block the counts put it in."""

    def __init__(self, gens, n, rank, world, chunk_parents):
        import torch
        self.torch = torch
        self.gens, self.n, self.rank, self.world = gens, n, rank, world
        self.geo = sharded.geometry(n, world)
        self.chunk_parents = chunk_parents
        start = list(range(n))
        owner, bit = sharded.owner_of(start, self.geo)
        self.bits = {bit} if owner == rank else set()
        self.front = [tuple(start)] if owner == rank else []
        self.next = []
        self.count = len(self.front)

    def _block(self, state):
        owner, bit = sharded.owner_of(list(state), self.geo)
        return owner, bit // self.geo.block_bits

    def chunks(self):
        return -(-self.count // self.chunk_parents)

    def route(self, c):
        per = self.geo.blocks_per_owner
        buckets = [[] for _ in range(self.world * per)]
        for s in self.front[c * self.chunk_parents:(c + 1) * self.chunk_parents]:
            for g in self.gens:
                child = tuple(s[g[i]] for i in range(self.n))
                owner, block = self._block(child)
                buckets[owner * per + block].append(sharded.pack_state(child))
        words = self.torch.tensor([w for b in buckets for w in b], dtype=self.torch.int64)
        counts = self.torch.tensor([len(b) for b in buckets], dtype=self.torch.int64)
        return words, counts

    def accept(self, words, counts):
        per = self.geo.blocks_per_owner
        ws, cs = words.tolist(), counts.tolist()
        assert len(cs) == self.world * per and sum(cs) == len(ws)
        at = 0
        for src in range(self.world):
            for block in range(per):
                for w in ws[at:at + cs[src * per + block]]:
                    state = _unpack(w, self.n)
                    owner, bit = sharded.owner_of(list(state), self.geo)
                    assert owner == self.rank and bit // self.geo.block_bits == block
                    if bit not in self.bits:
                        self.bits.add(bit)
                        self.next.append(state)
                at += cs[src * per + block]

    def finish(self):
        self.front, self.next = self.next, []
        self.count = len(self.front)
        return self.count


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, gens, n, chunk, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
        shard = CpuShard(gens, n, rank, world, chunk)
        bfs = sharded.ShardedBfs([shard], sharded.DistExchange(None, "cpu"))
        if mode == "exit":
            bfs.layer()
            if rank == 1:
                os._exit(0)  # leaves between layers, with no collective in flight
        out.put((rank, "ok", bfs.run()))
    except Exception as exc:  # noqa: BLE001 - reported to the parent
        out.put((rank, "error", f"{type(exc).__name__}: {exc}\n{traceback.format_exc()[-600:]}"))


def _run(gens, n, world, chunk=1 << 30, mode="normal"):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, gens, n, chunk, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world - (1 if mode == "exit" else 0)):
        rank, kind, payload = out.get(timeout=180)
        results[rank] = (kind, payload)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return results


@pytest.mark.timeout(300)
@pytest.mark.parametrize("world,chunk", [(2, 1 << 30), (3, 7)])
def test_ranks_split_one_bfs_and_agree_on_the_oracle_table(world, chunk):
    n = 6
    gens = G.lrx_generators(n)
    expect = G.layer_sizes(G.permutation_graph(gens, list(range(n))))
    res = _run(gens, n, world, chunk)
    for rank in range(world):
        kind, got = res[rank]
        assert kind == "ok", got
        assert got == expect


@pytest.mark.timeout(300)
def test_directed_graph_splits_exactly():
    n = 6
    gens = [[1, 2, 0, 3, 4, 5], [0, 1, 2, 4, 5, 3], [5, 0, 1, 2, 3, 4]]
    expect = G.layer_sizes(G.permutation_graph(gens, list(range(n))))
    res = _run(gens, n, 2, 5)
    assert res[0] == ("ok", expect) and res[1] == ("ok", expect)


@pytest.mark.timeout(120)
def test_rank_that_leaves_between_layers_ends_the_next_exchange_with_an_error():
    res = _run(G.lrx_generators(5), 5, 2, mode="exit")
    kind, payload = res[0]
    assert kind == "error", payload


def test_unaligned_frontier_is_refused_before_any_launch():
    """The route kernels read parents two at a time (16-byte loads): an
    unaligned frontier pointer is refused on the host, with no device call.
    The pointers here are never dereferenced."""
    import ctypes as C

    from multigpubfs_b200 import native
    lib = native.load()
    perms = (C.c_uint32 * 5)(1, 2, 3, 4, 0)
    counts = C.c_void_p(0x10000)
    rc = lib.mgbfs2_shard_route(5, 1, perms, C.c_void_p(0x10008), 3, 2, C.c_void_p(0x20000), 64, counts, None,
                                C.c_void_p(0x30000), 1 << 20, None)
    assert rc == 1
    rc = lib.mgbfs2_expand_layer_bitmap(5, 1, perms, C.c_void_p(0x10008), 3, C.c_void_p(0x20000),
                                        C.c_void_p(0x40000), 64, C.c_void_p(0x50000), None, C.c_void_p(0x30000),
                                        1 << 20, None)
    assert rc == 1
