"""ORACLE -- test infrastructure, not product code.

CPU restatement (numpy, float64/complex128) of GPAW's FD hot-path kernels,
used only by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py as the checker.  The product (gpaw_b200) never imports this package.

Each function cites the reference file:line it restates.  The restatement is
pinned two ways (tests/test_oracle_*.py):
  * against GPAW's own C extension built from the reference sources by
    oracle/Makefile into oracle/_ref/ (when that build is present), and
  * against golden vectors under tests/golden/ generated from that build by
    tests/golden/make_golden.py, plus the known-answer tests of the
    reference's test suite (gpaw/test/fd_ops/*, gpaw/test/lfc/*,
    gpaw/test/gpu/test_xc_gpu.py).
"""
