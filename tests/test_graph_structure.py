"""Graph structure tests (CPU), restating dequantizer/src/tests/test_tensor_graph.py:10-23
(small_graph_test tensor_graph.py:637-795, lattice_3d_test :798-1041,
random_tree_test :1044-1072) on dequantizer_b200.graph."""

import numpy as np
import pytest

from dequantizer_b200 import graph as G
from dequantizer_b200.graph import Edge, MessageID, Node, TensorGraph
from dequantizer_b200.initializers import (get_message_random_nonnegative_initializer,
                                           get_tensor_random_normal_initializer)
from oracle.maps import init_tensors


def test_small_graph():
    g = TensorGraph()
    ids = [g.add_node(d) for d in (2, 5, 3, 4, 6)]
    g.add_edge((0, 1), 2)
    g.add_edge((2, 0), 4)
    g.add_edge((1, 2), 5)
    g.add_edge((4, 2, 3), 6)
    n = [g.get_node(i) for i in range(5)]
    e = [g.get_edge(k) for k in [(0, 1), (2, 0), (1, 2), (4, 2, 3)]]
    tensors = init_tensors(g, get_tensor_random_normal_initializer(42))
    messages = g.init_messages(get_message_random_nonnegative_initializer(43))
    assert g.nodes_number == 5 and g.edges_number == 4
    assert ids == [0, 1, 2, 3, 4]
    assert [x.dimension for x in n] == [2, 5, 3, 4, 6]
    assert [x.degree for x in n] == [2, 2, 3, 1, 1]
    assert [x.degree for x in e] == [2, 2, 2, 3]
    assert [x.bond_shape for x in n] == [(2, 4), (2, 5), (4, 5, 6), (6,), (6,)]
    assert n[0].neighbors == [e[0], e[1]] and n[1].neighbors == [e[0], e[2]]
    assert n[2].neighbors == [e[1], e[2], e[3]] and n[3].neighbors == [e[3]] and n[4].neighbors == [e[3]]
    assert [x.dimension for x in e] == [2, 4, 5, 6]
    assert e[0].neighbors == [n[0], n[1]] and e[1].neighbors == [n[2], n[0]]
    assert e[2].neighbors == [n[1], n[2]] and e[3].neighbors == [n[4], n[2], n[3]]
    assert [tensors[i].shape for i in range(5)] == [(2, 4, 2), (2, 5, 5), (4, 5, 6, 3), (6, 4), (6, 6)]
    expect = {(0, (0, 1)): 2, (0, (2, 0)): 4, (1, (0, 1)): 2, (1, (1, 2)): 5, (2, (2, 0)): 4, (2, (1, 2)): 5,
              (2, (4, 2, 3)): 6, (3, (4, 2, 3)): 6, (4, (4, 2, 3)): 6}
    for (nid, eid), d in expect.items():
        assert messages[MessageID(nid, eid)].shape == (d, d)
        assert messages[MessageID(eid, nid)].shape == (d, d)
    m = messages[MessageID((4, 2, 3), 4)]
    assert (np.linalg.eigvalsh(m) > -1e-5).all()
    assert len(messages) == 18
    g.add_node()
    for start, order in ((e[1], "dfs"), (n[2], "bfs")):
        seen = set(g.get_traversal_iterator(start, order))
        assert seen.issuperset(n) and seen.issuperset(e) and len(seen) == 9


def test_errors_match_reference():
    g = TensorGraph()
    g.add_node(2, 1)
    with pytest.raises(KeyError):
        g.add_node(2, 1)
    with pytest.raises(KeyError):
        g.add_edge((1, 7), 2)
    g.add_node(2, 2)
    g.add_edge((1, 2), 2)
    with pytest.raises(KeyError):
        g.add_edge((1, 2), 3)
    with pytest.raises(KeyError):
        next(g.get_traversal_iterator(ordering="random"))
    assert list(TensorGraph().get_traversal_iterator()) == []


def test_3d_lattice():
    sizes, bond, phys = (4, 5, 6), 4, 3
    lat = G.get_nd_lattice(list(sizes), phys, bond)
    tensors = init_tensors(lat, get_tensor_random_normal_initializer(43))
    messages = lat.init_messages(get_message_random_nonnegative_initializer(44))
    x, y, z = sizes
    for corner in [(0, 0, 0), (x - 1, 0, 0), (0, y - 1, 0), (x - 1, y - 1, 0), (0, 0, z - 1), (x - 1, 0, z - 1),
                   (0, y - 1, z - 1), (x - 1, y - 1, z - 1)]:
        assert tensors[corner].shape == (bond,) * 3 + (phys,)
    for i in range(1, x - 2):
        for c in [(i, 0, 0), (i, y - 1, 0), (i, 0, z - 1), (i, y - 1, z - 1)]:
            assert tensors[c].shape == (bond,) * 4 + (phys,)
    for i in range(1, x - 2):
        for j in range(1, y - 2):
            for k in range(1, z - 2):
                assert tensors[(i, j, k)].shape == (bond,) * 6 + (phys,)
    n_edges = (x - 1) * y * z + x * (y - 1) * z + x * y * (z - 1)
    elems = list(lat.get_traversal_iterator())
    assert sum(isinstance(el, Node) for el in elems) == x * y * z == len(tensors)
    assert sum(isinstance(el, Edge) for el in elems) == n_edges
    assert len(messages) == 4 * n_edges


def test_random_tree():
    tree = G.get_random_tree_tensor_graph(20, 3, [3, 4, 5, 6], 44)
    assert tree.nodes_number == 20 and tree.edges_number == 19
    elems = list(tree.get_traversal_iterator())
    assert sum(isinstance(el, Node) for el in elems) == 20
    assert sum(isinstance(el, Edge) for el in elems) == 19
    assert all(el.dimension == 3 for el in elems if isinstance(el, Node))


def test_eagle_lattices():
    g = G.get_heavy_hex_ibm_eagle_lattice()
    assert g.nodes_number == 127 and g.edges_number == 144
    degs = sorted(n.degree for n in g.nodes.values())
    assert max(degs) == 3 and min(degs) == 1
    inf = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    assert inf.nodes_number == 5 and inf.edges_number == 6


@pytest.mark.parametrize("n", [16, 100, 1024])
def test_random_regular_pairing_model(n):
    pairs = G.random_regular_pairs(n, 3, 0)
    assert len(pairs) == 3 * n // 2
    assert all(a != b for a, b in pairs)
    assert len({(min(a, b), max(a, b)) for a, b in pairs}) == len(pairs)
    deg = np.bincount(np.array(pairs).reshape(-1), minlength=n)
    assert (deg == 3).all()


def test_edge_coloring_is_proper():
    g = G.get_heavy_hex_ibm_eagle_lattice()
    classes = G.greedy_edge_coloring(g)
    assert sum(len(c) for c in classes) == 144
    assert len(classes) == 3
    for c in classes:
        ends = [n for eid in c for n in eid]
        assert len(ends) == len(set(ends))
