"""Pins the FP64 oracle to the reference's own known-answer tests (CPU).

* random_tree_ghz_gauge_fixing_test -- dequantizer/src/mappings/utils_testing.py:20-100
* ghz_state_preparation_test        -- dequantizer/src/graph/tensor_graph.py:1075-1177
* _bp_quantum_emulator_test         -- dequantizer/src/quantum_emulator/test_bp_quantum_emulator.py:21-108
* test_gen_ghz_core / bloated GHZ   -- dequantizer/src/graph/test_unit.py:8-36
The reference has no golden numeric vectors; these physics-level answers
(messages = I/d, rho = I/d, agreement with the dense state vector) are the
assertions it makes, with its tolerances.
"""

import numpy as np
import pytest

from dequantizer_b200 import graph as G
from dequantizer_b200.graph import Edge, Node
from dequantizer_b200.initializers import (_gen_ghz_core, get_message_random_nonnegative_initializer,
                                           get_tensor_bloated_ghz_initializer, get_tensor_std_state_initializer)
from oracle import maps as OM
from oracle.emulator import BPQuantumEmulator, ExactQuantumEmulator
from tests.helpers import heavy_cube, random_ising_q2_gate, random_q1_gate, small_heavy_hex


def _bp_until(bp, tensors, messages, acc):
    dist = np.finfo(np.float32).max
    while dist > acc:
        new = bp(tensors, messages)
        dist = OM.messages_frob_distance(new, messages)
        messages = new
    return messages


def test_random_tree_ghz_gauge_fixing():
    acc, d = 1e-8, 3
    tree = G.get_random_tree_tensor_graph(20, d, [3, 4, 5], 42)
    trav = list(tree.get_traversal_iterator())
    bp = OM.get_belief_propagation_map(trav)
    tensors = OM.init_tensors(tree, get_tensor_bloated_ghz_initializer(42))
    messages = tree.init_messages(get_message_random_nonnegative_initializer(43))
    messages = _bp_until(bp, tensors, messages, acc)
    new_t, lam = OM.get_vidal_gauge_fixing_map(trav, acc)(tensors, messages)
    assert OM.get_vidal_gauge_distance_map(trav, acc)(new_t, lam) < acc
    tt, tl = OM.truncate(tree, new_t, lam, acc)
    for el in tree.get_traversal_iterator():
        if isinstance(el, Edge):
            assert el.dimension == d
        else:
            assert all(x == d for x in el.bond_shape)
    tensors = OM.get_symmetric_gauge_fixing_map(trav, acc)(tt, tl)
    messages = tree.init_messages(get_message_random_nonnegative_initializer(44))
    messages = _bp_until(bp, tensors, messages, acc)
    for m in messages.values():
        assert (np.abs(m - np.eye(d) / d) < acc).all()
    for el in tree.get_traversal_iterator():
        if isinstance(el, Node):
            dens = OM.get_one_side_density_matrix(el, tensors, messages)
            assert np.linalg.norm(dens - np.eye(d) / d) < acc


HADAMARD = np.array([[1, 1], [1, -1]], dtype=np.complex128)
CNOT = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=np.complex128).reshape(2, 2, 2, 2)
GHZ_CNOTS = [((0, 0), (0, 1)), ((0, 1), (0, 2)), ((0, 2), (0, 3)), ((0, 0), (1, 0)), ((0, 1), (1, 1)),
             ((0, 2), (1, 2)), ((0, 3), (1, 3)), ((1, 0), (2, 0)), ((2, 0), (2, 1)), ((2, 1), (2, 2)),
             ((2, 2), (2, 3)), ((2, 3), (3, 3)), ((3, 3), (3, 2)), ((2, 1), (3, 1)), ((2, 0), (3, 0))]


def test_ghz_state_preparation():
    lattice = G.get_nd_lattice([4, 4], 2, 1)
    tensors = OM.init_tensors(lattice, get_tensor_std_state_initializer())
    OM.apply1(lattice, (0, 0), tensors, HADAMARD)
    for a, b in GHZ_CNOTS:
        OM.apply2(lattice, a, b, tensors, CNOT, 1e-8)
    trav = list(lattice.get_traversal_iterator())
    bp = OM.get_belief_propagation_map(trav)
    messages = _bp_until(bp, tensors, lattice.init_messages(get_message_random_nonnegative_initializer(42)), 1e-8)
    for i in range(4):
        for j in range(4):
            dens = OM.get_one_side_density_matrix(lattice.get_node((i, j)), tensors, messages)
            assert np.isclose(dens, np.eye(2) / 2).all()
    for a, b in reversed(GHZ_CNOTS):
        OM.apply2(lattice, a, b, tensors, CNOT, 1e-8)
    OM.apply1(lattice, (0, 0), tensors, HADAMARD)
    messages = _bp_until(bp, tensors, lattice.init_messages(get_message_random_nonnegative_initializer(43)), 1e-8)
    tensors, lmbds = OM.get_vidal_gauge_fixing_map(trav, 1e-8)(tensors, messages)
    tensors, lmbds = OM.truncate(lattice, tensors, lmbds, 1e-8)
    tensors = OM.get_symmetric_gauge_fixing_map(trav, 1e-8)(tensors, lmbds)
    messages = _bp_until(bp, tensors, lattice.init_messages(get_message_random_nonnegative_initializer(44)), 1e-8)
    for i in range(4):
        for j in range(4):
            node = lattice.get_node((i, j))
            for dim, nb in zip(node.bond_shape, node.neighbors):
                assert nb.dimension == dim == 1
            dens = OM.get_one_side_density_matrix(node, tensors, messages)
            assert np.isclose(dens - np.array([[1, 0], [0, 0]]), 0, atol=1e-8).all()


def emulator_vs_exact(graph, layers, accuracy, seed=42):
    """test_bp_quantum_emulator.py:21-95 with seeded numpy randomness; the
    uniform samples of measure() are shared by both emulators."""
    rng = np.random.default_rng(seed)
    trav = list(graph.get_traversal_iterator())
    exact = ExactQuantumEmulator(graph)
    bp = BPQuantumEmulator(graph, seed, 1024, graph.edges_number, belief_propagation_accuracy=1e-6)
    nodes = [el for el in trav if isinstance(el, Node)]
    state = {n.id: int(rng.integers(0, 2)) for n in nodes}
    exact.set_to_product_state(state)
    bp.set_to_product_state(state)
    for nid, s in state.items():
        correct = np.zeros((2, 2))
        correct[s, s] = 1.0
        assert np.isclose(bp.dens_q1(nid), correct, atol=1e-8).all()
        assert np.isclose(exact.dens_q1(nid), correct, atol=1e-8).all()
        assert bp.measure(nid, float(rng.uniform())) == s
    for _ in range(layers):
        for el in trav:
            if isinstance(el, Node):
                g = random_q1_gate(rng)
                exact.apply_q1(g, el.id)
                bp.apply_q1(g, el.id)
            else:
                g = random_ising_q2_gate(rng)
                exact.apply_q2(g, *el.id)
                bp.apply_q2(g, *el.id)
    worst = 0.0
    for el in nodes:
        worst = max(worst, float(np.linalg.norm(exact.dens_q1(el.id) - bp.dens_q1(el.id))))
    assert worst < accuracy, worst
    for el in nodes:
        assert np.linalg.norm(exact.dens_q1(el.id) - bp.dens_q1(el.id)) < accuracy
        u = float(rng.uniform())
        assert exact.measure(el.id, u) == bp.measure(el.id, u)
    return worst


def test_emulator_heavy_cube():
    emulator_vs_exact(heavy_cube(), 2, 3e-3)


@pytest.mark.slow
def test_emulator_small_heavy_hex():
    emulator_vs_exact(small_heavy_hex(), 4, 1e-4)


def test_emulator_random_tree():
    emulator_vs_exact(G.get_random_tree_tensor_graph(15, 2, 14 * [1], 42), 4, 1e-4)


def test_gen_ghz_core():
    for modes in range(2, 6):
        for d in range(1, 4):
            core = _gen_ghz_core(d, modes)
            assert abs(np.abs(core).sum() - d) < 1e-5
            for i in range(d):
                assert abs(core[modes * (i,)] - 1.0) < 1e-5


def test_bloated_ghz_initializer():
    g = G.TensorGraph()
    for _ in range(4):
        g.add_node(3)
    g.add_edge((0, 1), 5)
    g.add_edge((1, 2), 4)
    g.add_edge((1, 3), 6)
    t = OM.init_tensors(g, get_tensor_bloated_ghz_initializer(42))
    res = np.tensordot(t[0], t[1], axes=[0, 0])
    res = np.tensordot(t[2], res, axes=[0, 1])
    res = np.tensordot(t[3], res, axes=[0, 2])
    true = _gen_ghz_core(3, 4)
    assert res.shape == true.shape
    diff = np.linalg.norm(res - true) / max(np.linalg.norm(res), np.linalg.norm(true))
    assert diff < 1e-3
