"""CPU oracle of the hot path — TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py as the checker; never by the vipe_b200 package.  See the header of
each module for the reference code it restates.
"""
