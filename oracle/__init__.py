"""Oracle package (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package.  The product (spikesorting_fullpursuit_b200) never does.
"""
