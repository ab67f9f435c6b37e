"""ctypes front end of the reference's own standalone GPU library
(gpu/cayley_bfs.cu and its neighbours, built for sm_100a into
``_ref/libmgbfs_ref_gpu.so`` by ``make -C oracle ref-gpu`` from the reference
sources where they lie).

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's same-box
reference leg, never by the product package.  Its S_8..S_10
adjacent-transposition BFS (mgbfs_cayley_create / reset / step,
gpu/multigpubfs_cuda.h) is the reference's GPU code path timed beside this
engine's on the same B200, and its layer tables are a cross-check.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_ref" / "libmgbfs_ref_gpu.so"
_LIB = None


def available() -> bool:
    return LIBRARY.exists()


def library():
    global _LIB
    if _LIB is None:
        lib = C.CDLL(str(LIBRARY))
        lib.mgbfs_cayley_create.restype = C.c_int
        lib.mgbfs_cayley_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]
        lib.mgbfs_cayley_reset.restype = C.c_int
        lib.mgbfs_cayley_reset.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
        lib.mgbfs_cayley_step.restype = C.c_int
        lib.mgbfs_cayley_step.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_size_t),
                                          C.POINTER(C.c_float), C.c_char_p, C.c_size_t]
        lib.mgbfs_cayley_destroy.restype = None
        lib.mgbfs_cayley_destroy.argtypes = [C.c_void_p]
        _LIB = lib
    return _LIB


class CayleyBfs:
    """One reference context for S_n (8 <= n <= 10) under the n-1 adjacent
    transpositions: a 32-bit-word Lehmer bitmap and two frontiers of n! states
    (so its bounded append never overflows)."""

    def __init__(self, n: int):
        import math
        self.lib = library()
        self.n = n
        self.handle = C.c_void_p()
        err = C.create_string_buffer(256)
        rc = self.lib.mgbfs_cayley_create(n, math.factorial(n), C.byref(self.handle), err, len(err))
        if rc:
            raise RuntimeError(f"mgbfs_cayley_create: {rc} {err.value.decode()}")

    def run(self, variant: int = 0, layout: int = 0):
        """Whole BFS from the identity, one step per layer (the reference's
        host loop).  Returns (layer sizes, summed kernel ms, wall seconds)."""
        err = C.create_string_buffer(256)
        t = time.perf_counter()
        rc = self.lib.mgbfs_cayley_reset(self.handle, err, len(err))
        if rc:
            raise RuntimeError(f"mgbfs_cayley_reset: {rc} {err.value.decode()}")
        sizes, kernel_ms = [1], 0.0
        count, ms = C.c_size_t(), C.c_float()
        while True:
            rc = self.lib.mgbfs_cayley_step(self.handle, variant, layout, C.byref(count), C.byref(ms), err, len(err))
            if rc:
                raise RuntimeError(f"mgbfs_cayley_step: {rc} {err.value.decode()}")
            kernel_ms += ms.value
            if not count.value:
                break
            sizes.append(count.value)
        return sizes, kernel_ms, time.perf_counter() - t

    def close(self):
        if self.handle:
            self.lib.mgbfs_cayley_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
