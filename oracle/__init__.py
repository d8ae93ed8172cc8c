"""FP64 CPU oracle of the reference's fan-beam DD path -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker.  The product path never imports it.
"""
