"""CPU oracle of the reference algorithms - TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm use this package, and only as the checker or the timed CPU baseline.  The
product (gm1_b200) never imports, links or calls it.
"""
