"""B200 (sm_100a) bordered cyclic reduction for BABD systems.

``bcr`` is the ctypes front-end over the C ABI of ``libalglin_b200.so``
(``include/alglin_b200.h``): ``BorderedCR`` mirrors ``alglin::BorderedCR<double>``
and ``Batch`` solves many independent systems together.  ``synth`` generates the
seeded synthetic BABD systems used by the tests and the benchmark.
"""
