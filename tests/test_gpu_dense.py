"""GPU dense state-vector emulator against the oracle's exact emulator
(exact_quantum_emulator.py restated): random circuits of one- and two-qubit
gates on 10 qubits, state, density matrices and measurement outcomes with
shared samples to 1e-12; and the BP emulator against it on a tree (exact for
BP) to 1e-8."""

import numpy as np
import pytest
import torch

from dequantizer_b200 import BPQuantumEmulator
from dequantizer_b200 import graph as G
from dequantizer_b200.dense import DenseStateEmulator
from dequantizer_b200.graph import Node
from oracle.emulator import ExactQuantumEmulator
from tests.helpers import random_ising_q2_gate, random_q1_gate, to_np

pytestmark = pytest.mark.gpu


def _random_unitary(rng, d):
    z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    q, _ = np.linalg.qr(z)
    return q


def test_dense_matches_oracle_exact_emulator():
    g = G.get_random_regular_graph(10, 3, 2, 1, 4)
    rng = np.random.default_rng(1)
    dev, ref = DenseStateEmulator(g), ExactQuantumEmulator(G.get_random_regular_graph(10, 3, 2, 1, 4))
    nodes = [el.id for el in g.get_traversal_iterator() if isinstance(el, Node)]
    assert dev.node2pos == ref.node2pos
    start = {nid: int(rng.integers(0, 2)) for nid in nodes}
    dev.set_to_product_state(start)
    ref.set_to_product_state(start)
    edges = list(g.edges)
    for _ in range(40):
        if rng.uniform() < 0.4:
            u = _random_unitary(rng, 2)
            nid = nodes[int(rng.integers(0, len(nodes)))]
            dev.apply_q1(u, nid)
            ref.apply_q1(u, nid)
        else:
            u = _random_unitary(rng, 4).reshape(2, 2, 2, 2)
            a, b = edges[int(rng.integers(0, len(edges)))]
            if rng.uniform() < 0.5:
                a, b = b, a
            dev.apply_q2(u, a, b)
            ref.apply_q2(u, a, b)
    assert np.abs(to_np(dev.state) - ref.state).max() < 1e-12
    for nid in nodes:
        assert np.abs(to_np(dev.dens_q1(nid)) - ref.dens_q1(nid)).max() < 1e-12
    for nid in nodes[:5]:
        s = float(rng.uniform())
        assert dev.measure(nid, s) == ref.measure(nid, s)
    assert np.abs(to_np(dev.state) - ref.state).max() < 1e-12


def test_bp_emulator_matches_dense_on_a_tree():
    def make():
        return G.get_random_tree_tensor_graph(12, 2, 11 * [1], 7)

    g_bp, g_dense = make(), make()
    rng = np.random.default_rng(3)
    bp = BPQuantumEmulator(g_bp, 1, 64, g_bp.edges_number, belief_propagation_accuracy=1e-10)
    dense = DenseStateEmulator(g_dense)
    trav = list(g_bp.get_traversal_iterator())
    for _ in range(3):
        for el in trav:
            if isinstance(el, Node):
                q = random_q1_gate(rng)
                bp.apply_q1(q, el.id)
                dense.apply_q1(q, el.id)
            else:
                q = random_ising_q2_gate(rng)
                bp.apply_q2(q, *el.id)
                dense.apply_q2(q, *el.id)
    for el in trav:
        if isinstance(el, Node):
            assert np.abs(to_np(bp.dens_q1(el.id)) - to_np(dense.dens_q1(el.id))).max() < 1e-8
