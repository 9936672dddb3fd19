"""Thread-parallel map for the oracle (test infrastructure only).

The oracle's heavy steps (sparse G products, FFTs, the SARA filter banks)
run in NumPy/SciPy code that releases the GIL, so independent channels,
blocks and wavelet bases map onto host threads.  Results are returned in
input order and every reduction over them stays in that order, so the
oracle's outputs do not depend on the thread count.  Nested calls (a mapped
function that maps again) run sequentially inside the worker.
"""
from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

_local = threading.local()
_pool = None
_lock = threading.Lock()


def n_threads() -> int:
    env = os.environ.get("FHS_ORACLE_THREADS")
    if env:
        return max(1, int(env))
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return os.cpu_count() or 1


def _get_pool():
    global _pool
    with _lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(max_workers=n_threads(), thread_name_prefix="oracle")
        return _pool


def _run(fn, item):
    _local.inside = True
    try:
        return fn(item)
    finally:
        _local.inside = False


def pmap(fn, items):
    """[fn(i) for i in items], on the oracle's thread pool."""
    items = list(items)
    if len(items) <= 1 or n_threads() == 1 or getattr(_local, "inside", False):
        return [fn(i) for i in items]
    return list(_get_pool().map(lambda i: _run(fn, i), items))
