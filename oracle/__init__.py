"""CPU oracle of the distributed-scatterer chain — TEST INFRASTRUCTURE ONLY.

Imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` as the checker; never by the product path.
"""
