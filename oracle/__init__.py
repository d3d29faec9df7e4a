"""CPU oracle for the B200 vector engine -- TEST INFRASTRUCTURE ONLY.

This package restates the reference's CPU engine (ve/openmp driven by core/jitk) so that the
tests, `__graft_entry__.smoke()` and the `cpu_baseline` leg of bench.py can check the CUDA engine
against it. Nothing in bohrium_b200/ imports it, and the product never runs it.

  jitk.py        the reference fuser (simplify, pre-fuser, greedy DAG contraction,
                 collapse_redundant_axes, identity blocks) restated in Python
  ve_openmp.py   the reference's C99/OpenMP code generator and executor restated: every fused
                 kernel becomes C source compiled with gcc -O3 -march=native -fopenmp and run on the
                 host cores
  kernel_deps.h  device-independent helpers of the generated C (Philox2x32-10 of BH_RANDOM)
  Makefile       builds oracle/_ref/ from the reference's own sources (the vendored Random123
                 header) to pin kernel_deps.h

Parity pins: the Philox restatement is checked against oracle/_ref (the reference's own header,
compiled in place by oracle/Makefile) and against the known-answer vector (counter 0, key 42) ->
(624017136, 4231775638); operation semantics are checked against NumPy, the witness the
reference's own test-suite uses (test/python/run.py:42-59), in tests/test_oracle.py; golden
vectors generated with the reference header live in tests/golden/.
"""
