"""CPU oracle for the exact dual regional-extrema route (test infrastructure).

Imported only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``.  The product library never loads it.
"""
from .oracle import extrema, extrema_batch, max_threads, tile_fragments  # noqa: F401
