"""Test and benchmark infrastructure (not the product).

* ``exact``    - exact Fraction restatement of the reference's CGAL bvh-peel
                 route; the parity oracle.
* ``fastpeel`` - ctypes wrapper of ``fast_peel.cpp``, a C++/OpenMP restatement
                 of the reference's finite-precision fast-bvh-peel CPU path;
                 the timed CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
