"""CPU oracle for the pseudoskeleton path: TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package, and only as the checker or the timed CPU baseline; the library never routes
through it.
"""
