"""The oracle: CPU restatements of the reference's algorithms for the law-step path, used ONLY as the checker.

Test infrastructure. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import anything here;
the product (online-physics-cuda_b200/) never does. Every function cites the reference file:line it restates
(paths within NotTruecCoder/online-physics-cuda).

Pinning: tests/test_oracle_pin.py checks these restatements against golden outputs of the reference's own CPU solver
(tests/golden/, made by tests/golden/make_golden.py from the reference's lawc built by oracle/Makefile), bit for bit
where the reference's arithmetic is restated op for op.
"""
