"""Stand-in for the `mkl` module (TEST INFRASTRUCTURE ONLY).

The reference package imports `mkl` at import time (utils/parallel_funs.py:5)
only to set thread counts; those calls do nothing here.
"""


def set_num_threads(n):
    return None


def get_max_threads():
    return 1
