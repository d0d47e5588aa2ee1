"""CPU oracle for the graph-tensor-network hot path.

TEST INFRASTRUCTURE ONLY. This package is a plain-FP64 numpy restatement of
LuchnikovI/dequantizer's algorithms (tensor_ops.py, mappings/*.py, the
tensor-valued TensorGraph methods and the emulators). Only ``tests/``,
``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py`` import it,
and only as the checker or as the timed CPU baseline. The product package
``dequantizer_b200`` never imports it and has no CPU fallback.

Pinning, two ways.
Golden vectors of the reference's own code: tests/golden/make_golden.py runs
the reference's dequantizer/src/tensor_ops.py as it is. JAX is absent, so it
runs under a stand-in whose jax.numpy forwards to numpy, with JAX's
immutable-array meaning of in-place operators. It records inputs and outputs
of pass_through_node, edge_svd, absorb_by_node, vidal_dist, canonicalize,
_decompose_gate, _apply_half_gate and simple_update
(tests/golden/tensor_ops_golden.npz), and tests/test_golden_reference.py
holds every oracle function to them (1e-12, 1e-10 where SVD vectors enter).
The same script runs the reference's maps (BP in its four schedules, Vidal
gauge and distance, symmetric gauge, lambdas2messages, message distance,
density matrices) on three deterministic graphs (tests/golden/maps_golden.npz);
It also records the TensorGraph gate methods on a lattice and a run of the
reference's BPQuantumEmulator (initial messages drawn as this package's
emulator draws them). tests/test_golden_maps.py holds the oracle's maps,
traversals, methods and emulator to these records.
The reference's own known-answer tests, restated in
tests/test_oracle_known_answers.py:
  * dequantizer/src/mappings/utils_testing.py:20-100 (random-tree GHZ gauge
    fixing: Vidal distance, truncation to d, messages = I/d, rho = I/d);
  * dequantizer/src/graph/tensor_graph.py:1075-1177 (GHZ preparation and
    uncomputation on a 4x4 lattice);
  * dequantizer/src/quantum_emulator/test_bp_quantum_emulator.py:21-108 (BP
    emulator vs the dense exact emulator on the heavy cube, small heavy hex and
    a random tree);
  * dequantizer/src/graph/test_unit.py:8-36 (GHZ core, bloated GHZ).
Parity with JAX's own LAPACK calls and with the JAX PRNG stream is unpinned.
"""
