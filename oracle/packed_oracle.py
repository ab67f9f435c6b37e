"""ctypes front end of the C oracle (``bfs_oracle.c``).

TEST INFRASTRUCTURE ONLY (see ``graph_oracle.py``): imported by tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs, never by the
product package.  Layer sizes from here are checked against the pure-Python
restatement and the reference-generated golden vectors in tests/golden/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
_LIB = None


def build() -> Path:
    """Compile liboracle.so in place (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return HERE / "liboracle.so"


def library():
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        lib.oracle_packed_bfs.restype = C.c_int
        lib.oracle_packed_bfs.argtypes = [
            C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint64, C.c_int,
            C.c_uint64, C.c_int, C.POINTER(C.c_uint64), C.c_uint32, C.POINTER(C.c_uint32),
            C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_uint64),
            C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_uint64)]
        lib.oracle_lehmer_rank.restype = C.c_int
        lib.oracle_lehmer_rank.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64),
                                           C.c_uint64, C.POINTER(C.c_uint64)]
        _LIB = lib
    return _LIB


def codes_of(start):
    """Dense symbol codes: the i-th smallest distinct label -> i."""
    order = sorted(set(start))
    index = {v: i for i, v in enumerate(order)}
    return [index[v] for v in start], order


def bits_for(distinct: int) -> int:
    bits = 4
    while (1 << bits) < distinct:
        bits *= 2
    return bits


def pack(codes, bits):
    w = 0
    for i, c in enumerate(codes):
        w |= c << (i * bits)
    return w


def unpack(word, n, bits):
    mask = (1 << bits) - 1
    return [(word >> (i * bits)) & mask for i in range(n)]


def packed_bfs(generators, start, *, use_bitmap=None, max_states=None, threads=0,
               max_layers=1 << 16, sample=0, partial=False):
    """Exact layer sizes of the permutation graph (child[i] = state[g[i]]).

    Returns (layer_sizes, last_layer_states, previous_layer_states), the two
    sample lists holding up to ``sample`` decoded states each, sorted.  With
    ``partial`` a search stopped by ``max_layers`` returns its first layers."""
    n = len(start)
    codes, labels = codes_of(start)
    bits = bits_for(len(labels))
    if n * bits > 64:
        raise ValueError("ORACLE_STATE_WIDTH")
    distinct = len(labels) == n
    if use_bitmap is None:
        use_bitmap = distinct and n <= 12
    if use_bitmap and not distinct:
        raise ValueError("ORACLE_BITMAP_NEEDS_DISTINCT")
    if max_states is None:
        import math
        max_states = math.factorial(n)
    lib = library()
    flat = (C.c_uint32 * (len(generators) * n))(*[x for g in generators for x in g])
    layers = (C.c_uint64 * max_layers)()
    count = C.c_uint32()
    last = (C.c_uint64 * max(sample, 1))()
    prev = (C.c_uint64 * max(sample, 1))()
    last_n = C.c_uint64()
    prev_n = C.c_uint64()
    rc = lib.oracle_packed_bfs(n, bits, len(generators), flat, pack(codes, bits), int(bool(use_bitmap)),
                               max_states, threads, layers, max_layers, C.byref(count),
                               last, sample, C.byref(last_n), prev, sample, C.byref(prev_n))
    if rc == 4 and partial:
        # Layer limit: layers 0..max_layers-1 were recorded and all expanded.
        return [int(layers[i]) for i in range(count.value)], [], []
    if rc:
        raise RuntimeError(f"ORACLE_STATUS_{rc}")
    sizes = [int(layers[i]) for i in range(count.value)]

    def decode(buf, k):
        out = [[labels[c] for c in unpack(int(buf[i]), n, bits)] for i in range(min(k, sample))]
        return sorted(out)
    return sizes, decode(last, last_n.value), decode(prev, prev_n.value)


def lehmer_ranks(words, n, bits=4):
    lib = library()
    arr = (C.c_uint64 * len(words))(*words)
    out = (C.c_uint64 * len(words))()
    rc = lib.oracle_lehmer_rank(n, bits, arr, len(words), out)
    if rc:
        raise RuntimeError(f"ORACLE_STATUS_{rc}")
    return [int(x) for x in out]


def default_threads() -> int:
    return len(os.sched_getaffinity(0))
