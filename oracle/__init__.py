"""Test infrastructure (the checker), never the product.

* ``kutta_oracle``: a CPU restatement in C of the reference's solve path
  (aggregation AMG setup, V-cycle, PCG / BiCGStab / Jacobi drivers, scalar
  guards) and an FP64 CG oracle; each function cites the reference file:line it
  follows.
* ``ref``: the reference's own CPU path compiled from its sources
  (``build_ref.sh`` -> ``_ref/libkutta_ref.so``), used to pin the restatement.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package.
"""
