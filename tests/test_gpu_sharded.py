"""The owner-partitioned path on the GPU: every rank's shard in one process
(the all-to-all done by copies), through mgbfs2_shard_route and
mgbfs2_shard_accept; the layer tables must equal the oracle's for every world
size, with large and tiny route chunks; each rank's frontier holds only the
states it owns; a word sent to the wrong rank is refused; and one NCCL rank
runs the same loop through torch.distributed."""
import os
import socket

import pytest

from oracle import graph_oracle as G
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _graph(gens, start):
    from multigpubfs_b200 import GraphDefinition
    return GraphDefinition.from_dict(G.permutation_graph(gens, start))


@pytest.mark.parametrize("world", [1, 2, 3, 5, 8])
def test_lrx_split_over_ranks_matches_the_reference_table(world):
    from multigpubfs_b200 import sharded
    expect = golden("lrx_layers.json")["layers"]["10"]
    assert sharded.run_emulated(_graph(G.lrx_generators(10), list(range(10))), world) == expect


@pytest.mark.parametrize("world,chunk", [(2, 1000), (4, 37), (7, 1 << 25)])
def test_chunked_routes_and_other_graphs(world, chunk):
    from multigpubfs_b200 import sharded
    cases = [
        (G.coxeter_generators(8), list(range(8))),
        ([[1, 2, 0, 3, 4, 5, 6, 7, 8], [0, 1, 2, 4, 5, 6, 7, 8, 3], [8, 0, 1, 2, 3, 4, 5, 6, 7]], list(range(9))),
        (G.lrx_generators(9), [3, 1, 4, 0, 5, 8, 2, 6, 7]),
    ]
    for gens, start in cases:
        expect = G.layer_sizes(G.permutation_graph(gens, start))
        got = sharded.run_emulated(_graph(gens, start), world, chunk_parents=chunk)
        assert got == expect, (gens, start)


def test_each_rank_keeps_only_the_states_it_owns():
    import numpy as np
    from multigpubfs_b200 import sharded
    world, n = 3, 8
    g = _graph(G.lrx_generators(n), list(range(n)))
    shards = [sharded.DeviceShard(g, r, world, 0) for r in range(world)]
    bfs = sharded.ShardedBfs(shards, sharded.LocalExchange(world))
    for _ in range(12):
        bfs.layer()
    geo = shards[0].geo
    total = 0
    for r, s in enumerate(shards):
        words = s.frontier_words().cpu().numpy().astype(np.uint64)
        total += len(words)
        for w in words[:500]:
            state = [int(w >> np.uint64(4 * i)) & 15 for i in range(n)]
            assert sharded.owner_of(state, geo)[0] == r
    assert total == golden("lrx_layers.json")["layers"]["8"][12]


def test_a_word_sent_to_the_wrong_rank_is_not_claimed():
    import torch
    from multigpubfs_b200 import sharded
    n, world = 7, 2
    g = _graph(G.lrx_generators(n), list(range(n)))
    shard = sharded.DeviceShard(g, 0, world, 0)
    state = next(p for p in ([(i + k) % n for i in range(n)] for k in range(n))
                 if sharded.owner_of(p, shard.geo)[0] == 1)
    owner, bit = sharded.owner_of(state, shard.geo)
    block = bit // shard.geo.block_bits
    words = torch.tensor([sharded.pack_state(state)], dtype=torch.int64, device="cuda")
    counts = torch.zeros(shard.geo.buckets, dtype=torch.int64, device="cuda")
    counts[block] = 1  # from source 0, as if it were in rank 0's block
    before = shard.slice.clone()
    with pytest.raises(RuntimeError, match="SHARD_ACCEPT_FAILED"):
        shard.accept(words, counts)
    assert int(shard.error.item()) & 128  # BAD_REFERENCE
    assert torch.equal(shard.slice, before) and shard.appended == 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_nccl_rank_runs_the_distributed_loop():
    import torch
    import torch.distributed as dist
    from multigpubfs_b200 import sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        got = sharded.run_distributed(_graph(G.lrx_generators(9), list(range(9))))
    finally:
        dist.destroy_process_group()
    assert got == golden("lrx_layers.json")["layers"]["9"]
