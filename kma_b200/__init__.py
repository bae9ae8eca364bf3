"""kma_b200 -- B200-native KMA device heap.

The product is libkma_b200.so (CUDA, sm_100a) with the C ABI of
include/kma.h and the device API of include/kma_device.cuh.  This package
is its host-side mirror: ``Heap`` (kma_create/kma_destroy), ``Workload``
(the stress programs), and the heap inspector in ``kma_b200.inspect``.
"""
from ._lib import (KMA_FLAG_BADFREE, KMA_FLAG_TIMEOUT, MODE_PLAIN, MODE_WARP, WL_C1, WL_C2,
                   KmaError, lib)
from .heap import Heap, Workload, bench_atomics, sbid_by_size, size_by_sbid, slots_by_size

__all__ = ["Heap", "Workload", "KmaError", "lib", "bench_atomics", "size_by_sbid",
           "slots_by_size", "sbid_by_size", "MODE_PLAIN", "MODE_WARP", "WL_C1", "WL_C2",
           "KMA_FLAG_TIMEOUT", "KMA_FLAG_BADFREE"]
