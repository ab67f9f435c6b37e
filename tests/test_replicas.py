"""The N>1 replica path (multigpubfs_b200.replicas) on CPU: two gloo ranks on
127.0.0.1, as the multi-GPU benchmark runs them on NCCL.  Failures are made on
the host (a differing table, a rank that exits before the exchange)."""
import multiprocessing as mp
import os
import socket
import traceback

import pytest

from multigpubfs_b200 import replicas

LRX5 = [1, 3, 6, 11, 19, 25, 23, 17, 11, 4]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, tables, seconds, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
        if mode == "exit" and rank == 1:
            os._exit(0)  # leaves between steps, with nothing in flight
        got = replicas.exchange(tables[rank], seconds[rank], 3 * sum(tables[rank]))
        out.put((rank, "ok", got))
    except replicas.ReplicaMismatch as exc:
        out.put((rank, "mismatch", str(exc)))
    except Exception as exc:  # noqa: BLE001 - reported to the parent
        out.put((rank, "error", f"{type(exc).__name__}: {exc}\n{traceback.format_exc()[-400:]}"))


def _run(tables, seconds, mode="normal", world=2):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, tables, seconds, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    expected = world - (1 if mode == "exit" else 0)
    for _ in range(expected):
        rank, kind, payload = out.get(timeout=120)
        results[rank] = (kind, payload)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return results


def test_table_digest_distinguishes_tables():
    assert replicas.table_digest(LRX5) == replicas.table_digest(list(LRX5))
    assert replicas.table_digest(LRX5) != replicas.table_digest(LRX5[:-1] + [5])
    assert replicas.table_digest([1, 2]) != replicas.table_digest([2, 1])


def test_two_ranks_agree_and_take_the_slowest_time():
    res = _run([LRX5, LRX5], [0.25, 0.5])
    for rank in (0, 1):
        kind, got = res[rank]
        assert kind == "ok", got
        assert got == {"world": 2, "device_seconds_max": 0.5, "successors_total": 2 * 3 * 120}


def test_layer_consensus_mismatch_raises_on_every_rank():
    other = LRX5[:-2] + [10, 5]
    res = _run([LRX5, other], [0.1, 0.1])
    assert res[0][0] == "mismatch" and res[1][0] == "mismatch"
    assert "LAYER_CONSENSUS_MISMATCH" in res[0][1]


@pytest.mark.timeout(120)
def test_rank_that_exits_ends_the_exchange_with_an_error():
    res = _run([LRX5, LRX5], [0.1, 0.1], mode="exit")
    kind, payload = res[0]
    assert kind == "error", payload


# ---------------------------------------------------------------------------
# Batched sweep split by instance: partition, gather to rank 0, and a rank
# that leaves between steps.

def test_partition_balances_work_deterministically():
    work = [7, 1, 9, 3, 3, 5, 2, 2]
    owner = replicas.partition_instances(work, 3)
    assert owner == replicas.partition_instances(list(work), 3)
    loads = [sum(w for w, o in zip(work, owner) if o == r) for r in range(3)]
    assert sum(loads) == sum(work) and max(loads) - min(loads) <= max(work)
    assert replicas.partition_instances(work, 1) == [0] * len(work)
    # The sweep itself: exact successor counts g * |G| from the host statics.
    from multigpubfs_b200 import native, workloads
    graphs = workloads.sweep(512)
    _, states = native.graph_statics([(g["action"]["generators"], g["start"]) for g in graphs])
    work = [len(g["action"]["generators"]) * int(s) for g, s in zip(graphs, states)]
    for world in (2, 4, 8):
        owner = replicas.partition_instances(work, world)
        loads = [sum(w for w, o in zip(work, owner) if o == r) for r in range(world)]
        assert max(loads) <= 1.02 * sum(work) / world  # within 2 % of an even split


SWEEP_TABLES = {0: [1, 3, 6], 1: [1, 2], 2: [1, 4, 9, 2], 3: [1], 4: [1, 5, 5]}


def _sweep_rank(rank, world, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
        work = [sum(t) for _, t in sorted(SWEEP_TABLES.items())]
        owner = replicas.partition_instances(work, world)
        ids = [i for i, o in enumerate(owner) if o == rank]
        if mode == "exit" and rank == 1:
            os._exit(0)  # leaves between steps, with nothing in flight
        if mode == "duplicate" and rank == 1:
            ids = ids + [0]  # rank 1 also claims instance 0
        tables = [SWEEP_TABLES[i] for i in ids]
        got = replicas.gather_tables(ids, tables, len(SWEEP_TABLES))
        out.put((rank, "ok", (ids, got)))
    except Exception as exc:  # noqa: BLE001 - reported to the parent
        out.put((rank, "error", f"{type(exc).__name__}: {exc}"))


def _run_sweep(mode="normal", world=2):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sweep_rank, args=(r, world, port, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = {}
    for _ in range(world - (1 if mode == "exit" else 0)):
        rank, kind, payload = out.get(timeout=120)
        results[rank] = (kind, payload)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return results


def test_two_ranks_split_the_sweep_and_rank0_gathers_every_table():
    res = _run_sweep()
    kind0, (ids0, got0) = res[0]
    kind1, (ids1, got1) = res[1]
    assert kind0 == kind1 == "ok"
    assert sorted(ids0 + ids1) == sorted(SWEEP_TABLES) and not set(ids0) & set(ids1)
    assert got0 == [SWEEP_TABLES[i] for i in sorted(SWEEP_TABLES)] and got1 is None


def test_gather_rejects_an_instance_reported_twice():
    res = _run_sweep(mode="duplicate")
    assert res[0][0] == "error" and "GATHER_INSTANCE" in res[0][1]


@pytest.mark.timeout(120)
def test_sweep_rank_that_exits_ends_the_gather_with_an_error():
    res = _run_sweep(mode="exit")
    kind, payload = res[0]
    assert kind == "error", payload
