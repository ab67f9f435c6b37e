"""torch-tensor wrappers of the kernel-level C-ABI entry points.

Each call launches on torch's current CUDA stream over caller-owned device
tensors; nothing here allocates inside libmgbfs2.
"""
from __future__ import annotations

import ctypes as C

from . import native


def _lib():
    return native.require_device()


def _error_word(device):
    import torch
    return torch.zeros(1, dtype=torch.int32, device=device)


def successors_i64(graph, parents):
    """All successors of int64 parents [count, elements] -> [count, generators, elements]."""
    import torch
    lib = _lib()
    a = graph.action
    parents = parents.to(torch.int64).contiguous()
    count, width = parents.shape
    gens = graph.generator_count
    dev = parents.device
    children = torch.empty((count, gens, width), dtype=torch.int64, device=dev)
    err = _error_word(dev)
    if a["kind"] == "permutation":
        perms = torch.tensor(a["generators"], dtype=torch.int32, device=dev).contiguous()
        rc = lib.mgbfs2_successors_i64(0, width, width, 1, gens, parents.data_ptr(), count, perms.data_ptr(), None,
                                       None, children.data_ptr(), err.data_ptr(), native.stream_handle())
    else:
        mats = torch.tensor([g["matrix"] for g in a["generators"]], dtype=torch.int64, device=dev).contiguous()
        mods = torch.tensor([g["modulo"] for g in a["generators"]], dtype=torch.int64, device=dev).to(torch.int32)
        rc = lib.mgbfs2_successors_i64(1, width, a["rows"], a["cols"], gens, parents.data_ptr(), count, None,
                                       mats.data_ptr(), mods.contiguous().data_ptr(), children.data_ptr(),
                                       err.data_ptr(), native.stream_handle())
    native.check(rc, "mgbfs2_successors_i64")
    torch.cuda.current_stream().synchronize()
    if int(err.item()):
        raise native.NativeError(native.DEVICE_STATUS, "mgbfs2_successors_i64", f"device error bits {int(err.item())}")
    return children


def successors_packed(degree, bits, generators, parents):
    """Packed successors: parents uint64-as-int64 [count] -> [count, generators]."""
    import torch
    lib = _lib()
    flat = (C.c_uint32 * (degree * len(generators)))(*[x for g in generators for x in g])
    count = parents.numel()
    out = torch.empty((count, len(generators)), dtype=torch.int64, device=parents.device)
    native.check(lib.mgbfs2_successors_packed(degree, bits, len(generators), flat, parents.data_ptr(), count,
                                              out.data_ptr(), native.stream_handle()), "mgbfs2_successors_packed")
    return out


def rank_packed(degree, bits, counts, words):
    """Exact lexicographic multiset rank of packed words; (ranks, error_bits)."""
    import torch
    lib = _lib()
    arr = (C.c_uint32 * len(counts))(*counts)
    ranks = torch.empty_like(words)
    err = _error_word(words.device)
    native.check(lib.mgbfs2_rank_packed(degree, bits, len(counts), arr, words.data_ptr(), words.numel(),
                                        ranks.data_ptr(), err.data_ptr(), native.stream_handle()),
                 "mgbfs2_rank_packed")
    return ranks, err


def bitmap_claim(ranks, bitmap, domain, warp=True):
    import torch
    lib = _lib()
    won = torch.zeros(ranks.numel(), dtype=torch.uint8, device=ranks.device)
    err = _error_word(ranks.device)
    native.check(lib.mgbfs2_bitmap_claim(ranks.data_ptr(), ranks.numel(), bitmap.data_ptr(), domain, won.data_ptr(),
                                         1 if warp else 0, err.data_ptr(), native.stream_handle()),
                 "mgbfs2_bitmap_claim")
    return won, err


def hash_insert(keys, table):
    import torch
    lib = _lib()
    inserted = torch.zeros(keys.numel(), dtype=torch.uint8, device=keys.device)
    err = _error_word(keys.device)
    native.check(lib.mgbfs2_hash_insert(keys.data_ptr(), keys.numel(), table.data_ptr(), table.numel(),
                                        inserted.data_ptr(), err.data_ptr(), native.stream_handle()),
                 "mgbfs2_hash_insert")
    return inserted, err


def sort_unique_tiles(keys, key_bits, tile=4096):
    import torch
    lib = _lib()
    tiles = (keys.numel() + tile - 1) // tile
    out = torch.empty(max(tiles * tile, 1), dtype=torch.int64, device=keys.device)
    counts = torch.zeros(max(tiles, 1), dtype=torch.int32, device=keys.device)
    native.check(lib.mgbfs2_sort_unique_tiles(keys.data_ptr(), keys.numel(), tile, key_bits, out.data_ptr(),
                                              counts.data_ptr(), native.stream_handle()),
                 "mgbfs2_sort_unique_tiles")
    return out, counts


def expand_layer_bitmap(degree, generators, frontier, bitmap, next_capacity, scratch=None):
    """One bucketed BFS layer: frontier (packed words, int64 tensor) against
    `bitmap` (int64 tensor of ceil(degree!/64) words, updated in place).
    Returns (next words [count], error bits)."""
    import torch
    lib = _lib()
    flat = (C.c_uint32 * (degree * len(generators)))(*[x for g in generators for x in g])
    count = frontier.numel()
    need = lib.mgbfs2_expand_layer_scratch_bytes(degree, len(generators), count)
    if scratch is None:
        scratch = torch.empty(need, dtype=torch.uint8, device=frontier.device)
    nxt = torch.empty(max(next_capacity, 1), dtype=torch.int64, device=frontier.device)
    out_count = torch.zeros(1, dtype=torch.int64, device=frontier.device)
    err = _error_word(frontier.device)
    native.check(lib.mgbfs2_expand_layer_bitmap(degree, len(generators), flat, frontier.data_ptr(), count,
                                                bitmap.data_ptr(), nxt.data_ptr(), next_capacity,
                                                out_count.data_ptr(), err.data_ptr(), scratch.data_ptr(),
                                                scratch.numel(), native.stream_handle()),
                 "mgbfs2_expand_layer_bitmap")
    n = int(out_count.item())
    return nxt[:min(n, next_capacity)], int(err.item())


def bucket_keys(keys, shift, shards, capacity):
    import torch
    lib = _lib()
    buckets = torch.zeros((shards, capacity), dtype=torch.int64, device=keys.device)
    counts = torch.zeros(shards, dtype=torch.int64, device=keys.device)
    err = _error_word(keys.device)
    native.check(lib.mgbfs2_bucket_keys(keys.data_ptr(), keys.numel(), shift, shards, buckets.data_ptr(), capacity,
                                        counts.data_ptr(), err.data_ptr(), native.stream_handle()),
                 "mgbfs2_bucket_keys")
    return buckets, counts, err
