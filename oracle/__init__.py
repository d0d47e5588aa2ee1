"""CPU oracle for the graph-tensor-network hot path.

TEST INFRASTRUCTURE ONLY. This package is a plain-FP64 numpy restatement of
LuchnikovI/dequantizer's algorithms (tensor_ops.py, mappings/*.py, the
tensor-valued TensorGraph methods and the emulators). Only ``tests/``,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` import it,
and only as the checker or as the timed CPU baseline. The product package
``dequantizer_b200`` never imports it and has no CPU fallback.

Pinning: the reference is pure Python on JAX, and JAX cannot be installed in
this environment, so it cannot be run to produce golden vectors, and the
reference ships none. The oracle is pinned instead by the reference's own
known-answer tests, restated in tests/test_oracle_known_answers.py:
  * dequantizer/src/mappings/utils_testing.py:20-100 (random-tree GHZ gauge
    fixing: Vidal distance, truncation to d, messages = I/d, rho = I/d);
  * dequantizer/src/graph/tensor_graph.py:1075-1177 (GHZ preparation and
    uncomputation on a 4x4 lattice);
  * dequantizer/src/quantum_emulator/test_bp_quantum_emulator.py:21-108 (BP
    emulator vs the dense exact emulator on the heavy cube, small heavy hex and
    a random tree);
  * dequantizer/src/graph/test_unit.py:8-36 (GHZ core, bloated GHZ).
Bitwise/LAPACK-level parity with JAX and JAX-PRNG stream parity are unpinned.
"""
