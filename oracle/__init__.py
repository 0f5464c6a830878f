"""CPU oracle for the quict_b200 parity tests -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker / the timed CPU
baseline.  The product (``quict_b200``) never imports it.

Contents
  sv.py        FP64 numpy restatement of QuICT's state-vector semantics
               (big-endian tensordot application, measurement, sampling rules)
  dm.py        FP64 density-matrix restatement (rho <- sum K rho K^dagger)
               and QuICT's noise-channel Kraus operators
  observe.py   expectation values and parameter-shift gradients (FP64)
  ref_port.py  numba restatement of the reference CPU kernels'
               index-walk algorithm (QuICT/ops/linalg/cpu_calculator.py),
               used as the timed CPU baseline ("port")

Parity pinning: tests/golden/ holds fixtures generated by running the
reference itself (tests/golden/make_golden.py); tests/test_oracle_golden.py
checks this oracle against them.
"""
