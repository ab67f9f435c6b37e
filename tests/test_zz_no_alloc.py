"""The allocation-free layer entry point, mgbfs2_expand_layer_bitmap_static.

It exists for callers that cannot allocate device memory per call (a host
that reserves the whole GPU in its own pool, or a search loop that must not
stall or fail in an allocator in the middle of a BFS): its scratch is a fixed
32 MiB array inside the library.  This file checks it through the C ABI
against the caller-scratch entry point, mgbfs2_expand_layer_bitmap, on two
calls in a row (the shared array keeps the first call's contents), and the
size limit.  It is collected last so that a failure here leaves every other
test already run; it must also pass alone in a fresh process.
"""
import ctypes as C
import math

import pytest

from oracle import graph_oracle as G
from oracle import packed_oracle as P

pytestmark = pytest.mark.gpu

STATIC_LIMIT = 4191328  # count * generators per call


def _call(lib, static, n, gens, frontier, bitmap, capacity, scratch=None):
    import torch
    from multigpubfs_b200 import native
    flat = (C.c_uint32 * (n * len(gens)))(*[x for g in gens for x in g])
    nxt = torch.full((capacity,), -1, dtype=torch.int64, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = native.stream_handle()
    if static:
        rc = lib.mgbfs2_expand_layer_bitmap_static(n, len(gens), flat, frontier.data_ptr(), frontier.numel(),
                                                   bitmap.data_ptr(), nxt.data_ptr(), capacity, count.data_ptr(),
                                                   err.data_ptr(), stream)
    else:
        rc = lib.mgbfs2_expand_layer_bitmap(n, len(gens), flat, frontier.data_ptr(), frontier.numel(),
                                            bitmap.data_ptr(), nxt.data_ptr(), capacity, count.data_ptr(),
                                            err.data_ptr(), scratch.data_ptr(), scratch.numel(), stream)
    torch.cuda.synchronize()
    k = int(count.item())
    return rc, nxt[:min(k, capacity)], k, int(err.item())


def test_static_layer_matches_caller_scratch_on_two_calls():
    import torch
    from multigpubfs_b200 import native
    lib = native.require_device()
    n = 10
    gens = G.lrx_generators(n)
    # Walk S10 LRX to layer 20 with the caller-scratch entry point, then expand
    # layers 20 and 21 with both entry points from identical inputs.
    bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
    bitmap[0] = 1
    frontier = torch.tensor([P.pack(list(range(n)), 4)], dtype=torch.int64, device="cuda")
    for _ in range(20):
        scratch = torch.empty(lib.mgbfs2_expand_layer_scratch_bytes(n, 3, frontier.numel()), dtype=torch.uint8,
                              device="cuda")
        rc, frontier, _, err = _call(lib, False, n, gens, frontier, bitmap, 3 * frontier.numel(), scratch)
        assert rc == 0 and err == 0
        frontier = frontier.clone()
    ref_bitmap, static_bitmap = bitmap.clone(), bitmap.clone()
    ref_frontier, static_frontier = frontier.clone(), frontier.clone()
    from tests.conftest import golden
    expect = golden("lrx_layers.json")["layers"]["10"]
    for depth in (20, 21):
        cap = 3 * ref_frontier.numel()
        scratch = torch.empty(lib.mgbfs2_expand_layer_scratch_bytes(n, 3, ref_frontier.numel()), dtype=torch.uint8,
                              device="cuda")
        rc_r, ref_next, k_r, err_r = _call(lib, False, n, gens, ref_frontier, ref_bitmap, cap, scratch)
        rc_s, static_next, k_s, err_s = _call(lib, True, n, gens, static_frontier, static_bitmap, cap)
        assert rc_r == 0 and rc_s == 0 and err_r == 0 and err_s == 0
        assert k_s == k_r == expect[depth + 1]
        # Same set of new states (frontier order is not deterministic), same bitmap.
        assert torch.equal(torch.sort(static_next).values, torch.sort(ref_next).values)
        assert torch.equal(static_bitmap, ref_bitmap)
        ref_frontier, static_frontier = ref_next.clone(), static_next.clone()


def test_static_layer_full_bfs_and_limit():
    import torch
    from multigpubfs_b200 import native
    lib = native.require_device()
    n = 8
    gens = G.coxeter_generators(n)
    bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
    bitmap[0] = 1
    frontier = torch.tensor([P.pack(list(range(n)), 4)], dtype=torch.int64, device="cuda")
    sizes = [1]
    while frontier.numel():
        rc, frontier, k, err = _call(lib, True, n, gens, frontier, bitmap, len(gens) * frontier.numel())
        assert rc == 0 and err == 0
        frontier = frontier.clone()
        if k:
            sizes.append(k)
    assert sizes == G.coxeter_layers(n)
    # Beyond the stated maximum the call is refused before any launch.
    too_many = STATIC_LIMIT // len(gens) + 1
    big = torch.zeros(too_many, dtype=torch.int64, device="cuda")
    rc, _, _, _ = _call(lib, True, n, gens, big, bitmap, 1)
    assert rc == 4  # MGBFS2_CAPACITY
    at_limit = torch.full((STATIC_LIMIT // len(gens),), P.pack(list(range(n)), 4), dtype=torch.int64, device="cuda")
    rc, _, k, err = _call(lib, True, n, gens, at_limit, bitmap, 1)
    assert rc == 0 and k == 0 and err == 0  # every successor already visited


def test_static_layer_allocates_nothing():
    """The defining property: after a first call on the device (which loads the
    kernels and resolves the array's address), further calls change neither
    the device's free memory nor torch's allocator.  Every buffer is made
    before the measured calls."""
    import torch
    from multigpubfs_b200 import native
    lib = native.require_device()
    n = 9
    gens = G.lrx_generators(n)
    flat = (C.c_uint32 * (n * len(gens)))(*[x for g in gens for x in g])
    bitmap = torch.zeros((math.factorial(n) + 63) // 64, dtype=torch.int64, device="cuda")
    frontier = torch.tensor([P.pack(list(range(n)), 4)], dtype=torch.int64, device="cuda")
    nxt = torch.empty(1 << 16, dtype=torch.int64, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = native.stream_handle()

    def layer(src, k):
        rc = lib.mgbfs2_expand_layer_bitmap_static(n, len(gens), flat, src.data_ptr(), k, bitmap.data_ptr(),
                                                   nxt.data_ptr(), nxt.numel(), count.data_ptr(), err.data_ptr(),
                                                   stream)
        assert rc == 0

    layer(frontier, 1)  # warm-up: module load and symbol address
    bitmap.zero_()
    bitmap[0] = 1
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    torch_before = torch.cuda.memory_allocated()
    layer(frontier, 1)
    layer(frontier, 1)  # the start's children are visited now: nothing new
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == torch_before
    assert free_after == free_before
    assert int(count.item()) == 0 and int(err.item()) == 0
