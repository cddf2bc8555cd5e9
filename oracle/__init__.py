"""CPU oracle and rebuilt-reference wrappers: test and baseline infrastructure only.

Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py
may import this package.  The product (piv_xcorr2d_v1.0_b200/) never does.
"""
