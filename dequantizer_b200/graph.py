"""Host-side structure of a tensor graph: nodes, edges, message IDs, traversal.

This module holds connectivity and shape bookkeeping only. Every numerical
operation on the tensors attached to the graph (BP sweeps, gauge fixing, gate
application, truncation) runs on the GPU through ``dequantizer_b200._lib``.

It mirrors the reference's graph API:

* ``MessageID``          -- dequantizer/src/graph/element.py:17-33
* ``Element``            -- dequantizer/src/graph/element.py:39-80
* ``Node``               -- dequantizer/src/graph/node.py:7-47
* ``Edge``               -- dequantizer/src/graph/edge.py:7-22
* ``TensorGraph``        -- dequantizer/src/graph/tensor_graph.py:31-170
* lattice generators     -- dequantizer/src/graph/tensor_graph.py:470-631

The tensor-valued ``TensorGraph`` methods (``init_tensors``, ``truncate``,
``apply1``, ``apply2``, ``apply2_to_vidal_canonical``) live in
``dequantizer_b200.tensor_graph_ops`` and are attached to the class there, so
that this module stays importable without the CUDA library.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from collections import deque
from dataclasses import dataclass
from typing import Callable, Dict, Hashable, Iterator, List, Optional, Set, Tuple, Union

import numpy as np

NodeID = Hashable
EdgeID = Tuple[Hashable, ...]
ElementID = Union[NodeID, EdgeID]


@dataclass(unsafe_hash=True, frozen=True)
class MessageID:
    """Directed message key (src element -> dst element).

    Ordered by ``repr`` like the reference (element.py:22-33), so dicts keyed by
    message IDs can be sorted deterministically."""

    src: ElementID
    dst: ElementID

    def __lt__(self, other: "MessageID") -> bool:
        return repr(self) < repr(other)

    def __gt__(self, other: "MessageID") -> bool:
        return repr(self) > repr(other)

    def __le__(self, other: "MessageID") -> bool:
        return repr(self) <= repr(other)

    def __ge__(self, other: "MessageID") -> bool:
        return repr(self) >= repr(other)


class Element(ABC):
    """A node or an edge of a tensor graph (element.py:39-80)."""

    def __init__(self, dimension: int, element_id: ElementID):
        self._id = element_id
        self._dimension = dimension

    @property
    def id(self) -> ElementID:
        return self._id

    @property
    def dimension(self) -> int:
        return self._dimension

    @dimension.setter
    def dimension(self, value: int):
        self._dimension = int(value)

    @abstractmethod
    def _add_element(self, element: "Element"):
        ...

    @property
    @abstractmethod
    def neighbors(self) -> List["Element"]:
        ...

    @property
    @abstractmethod
    def degree(self) -> int:
        ...

    def __repr__(self) -> str:
        return f"{type(self).__name__}({self._id!r})"


MessageDir = Tuple[Element, Element]


class Node(Element):
    """A tensor site. ``dimension`` is the physical dimension; the tensor has
    shape ``(*bond_shape, dimension)`` with bonds in neighbour insertion order
    (node.py:19-27)."""

    def __init__(self, dimension: int, node_id: NodeID):
        super().__init__(dimension, node_id)
        self._bond_shape: Tuple[int, ...] = ()
        self._neighbors: List[Element] = []
        self._indices: Dict[EdgeID, int] = {}

    @property
    def degree(self) -> int:
        return len(self._bond_shape)

    def _add_element(self, element: Element):
        if not isinstance(element.id, tuple):
            raise NotImplementedError("A node can only be connected to an edge.")
        self._neighbors.append(element)
        self._indices[element.id] = len(self._neighbors) - 1
        self._bond_shape = self._bond_shape + (element.dimension,)

    @property
    def neighbors(self) -> List[Element]:
        return self._neighbors

    @property
    def bond_shape(self) -> Tuple[int, ...]:
        return self._bond_shape

    @bond_shape.setter
    def bond_shape(self, value: Tuple[int, ...]):
        self._bond_shape = tuple(int(v) for v in value)

    @property
    def indices(self) -> Dict[EdgeID, int]:
        return self._indices


class Edge(Element):
    """A bond; its ID is the tuple of the node IDs it connects (edge.py:7-22)."""

    def __init__(self, dimension: int, edge_id: EdgeID):
        super().__init__(dimension, edge_id)
        self._neighbors: List[Element] = []

    def _add_element(self, node: Element):
        self._neighbors.append(node)

    @property
    def degree(self) -> int:
        return len(self._neighbors)

    @property
    def neighbors(self) -> List[Element]:
        return self._neighbors


class TensorGraph:
    """Connectivity of a graph tensor network (tensor_graph.py:31-170).

    Besides the reference's API it keeps a version counter that increases on
    every structural or shape change, so device-side packings can tell when
    they are stale."""

    def __init__(self):
        self._default_starting_node: Optional[Node] = None
        self._nodes: Dict[NodeID, Node] = {}
        self._edges: Dict[EdgeID, Edge] = {}
        self._nodes_number = 0
        self._edges_number = 0
        self.structure_version = 0

    @property
    def nodes_number(self) -> int:
        return self._nodes_number

    @property
    def edges_number(self) -> int:
        return self._edges_number

    @property
    def nodes(self) -> Dict[NodeID, Node]:
        return self._nodes

    @property
    def edges(self) -> Dict[EdgeID, Edge]:
        return self._edges

    def add_node(self, phys_dim: int = 2, node_id: Optional[NodeID] = None) -> NodeID:
        # A falsy id (None or 0) takes the running node count, as in
        # tensor_graph.py:62.
        new_id = node_id or self._nodes_number
        if new_id in self._nodes:
            raise KeyError(f"Node with ID {new_id} already exists.")
        self._nodes[new_id] = Node(phys_dim, new_id)
        if self._nodes_number == 0:
            self._default_starting_node = self._nodes[new_id]
        self._nodes_number += 1
        self.structure_version += 1
        return new_id

    def add_edge(self, edge_id: EdgeID, dimension: int):
        if edge_id in self._edges:
            raise KeyError(f"Edge with ID {edge_id} already exists.")
        new_edge = Edge(dimension, edge_id)
        for node_id in edge_id:
            node = self._nodes.get(node_id)
            if node is None:
                raise KeyError(
                    f"Node with ID {node_id} does not exists in the graph, but "
                    f"presents in the given edge ID {edge_id}"
                )
        for node_id in edge_id:
            node = self._nodes[node_id]
            new_edge._add_element(node)
            node._add_element(new_edge)
        self._edges[edge_id] = new_edge
        self._edges_number += 1
        self.structure_version += 1

    def get_node(self, node_id: NodeID) -> Optional[Node]:
        return self._nodes.get(node_id)

    def does_node_exist(self, node_id: NodeID) -> bool:
        return node_id in self._nodes

    def does_edge_exist(self, edge_id: EdgeID) -> bool:
        return edge_id in self._edges

    def get_edge(self, edge_id: EdgeID) -> Optional[Edge]:
        return self._edges.get(edge_id)

    def find_edge(self, node_id1: NodeID, node_id2: NodeID) -> Optional[Edge]:
        """Edge between two nodes in either orientation (tensor_graph.py:309-311)."""
        return self.get_edge((node_id2, node_id1)) or self.get_edge((node_id1, node_id2))

    def get_traversal_iterator(
        self,
        starting_element: Optional[Union[Node, Edge]] = None,
        ordering: str = "bfs",
    ) -> Iterator[Union[Node, Edge]]:
        """Yields nodes and edges in BFS or DFS order (tensor_graph.py:136-170).

        Like the reference this is a generator, so an unknown ``ordering``
        raises ``KeyError`` on the first ``next``."""
        if ordering == "bfs":
            pop_left = True
        elif ordering == "dfs":
            pop_left = False
        else:
            raise KeyError(f"Nodes / edges ordering method {ordering} is unknown.")
        stack: deque = deque()
        visited: Set[ElementID] = set()
        if starting_element is None:
            if self._default_starting_node is None:
                return
            stack.append(self._default_starting_node)
        else:
            stack.append(starting_element)
        while stack:
            element = stack.popleft() if pop_left else stack.pop()
            if element.id not in visited:
                yield element
                visited.add(element.id)
                for new_element in element.neighbors:
                    stack.append(new_element)

    def init_messages(self, initializer: Callable[[MessageDir], object]) -> Dict[MessageID, object]:
        """Messages for every (node -> edge) and (edge -> node) pair, in BFS
        order (tensor_graph.py:205-223)."""
        messages: Dict[MessageID, object] = {}
        for element in self.get_traversal_iterator():
            if isinstance(element, Node):
                for edge in element.neighbors:
                    messages[MessageID(src=element.id, dst=edge.id)] = initializer((element, edge))
            else:
                for node in element.neighbors:
                    messages[MessageID(src=element.id, dst=node.id)] = initializer((element, node))
        return messages

    def to_product(self):
        """Sets every bond dimension to 1 (tensor_graph.py:450-456)."""
        for node in self._nodes.values():
            node.bond_shape = len(node.bond_shape) * (1,)
        for edge in self._edges.values():
            edge.dimension = 1
        self.structure_version += 1

    def refresh_bond_shapes(self):
        """Recomputes every node's bond shape from its edges' dimensions."""
        for node in self._nodes.values():
            node.bond_shape = tuple(e.dimension for e in node.neighbors)
        self.structure_version += 1


# --------------------------------------------------------------------------
# Lattice / graph generators
# --------------------------------------------------------------------------


def get_random_tree_tensor_graph(
    nodes_number: int,
    phys_dimension: int,
    bond_dimensions: List[int],
    key: int,
) -> TensorGraph:
    """Random tree with integer node labels (tensor_graph.py:470-498).

    ``key`` seeds numpy's PCG64 generator (JAX's threefry stream is not
    reproducible without JAX); the construction follows the reference: attach
    a uniformly drawn disconnected node to a uniformly drawn connected node,
    with a uniformly drawn bond dimension."""
    rng = np.random.default_rng(key)
    tree = TensorGraph()
    connected = [0]
    disconnected = list(range(1, nodes_number))
    tree.add_node(phys_dimension, 0)
    for _ in range(1, nodes_number):
        connected_id = connected[int(rng.integers(0, len(connected)))]
        disconnected_id = disconnected[int(rng.integers(0, len(disconnected)))]
        tree.add_node(phys_dimension, disconnected_id)
        dim = bond_dimensions[int(rng.integers(0, len(bond_dimensions)))]
        tree.add_edge((connected_id, disconnected_id), dim)
        disconnected.remove(disconnected_id)
        connected.append(disconnected_id)
    return tree


def get_nd_lattice(
    lattice_sizes: List[int],
    phys_dimension: int,
    bond_dimension: int,
    open_boundary: bool = True,
) -> TensorGraph:
    """N-dimensional hypercubic lattice with tuple node labels
    (tensor_graph.py:511-539); node and edge insertion order as there."""
    nodes_number = int(np.prod(lattice_sizes))
    lattice = TensorGraph()
    ids: List[List[int]] = []
    for i in range(nodes_number):
        node_id = []
        for size in lattice_sizes:
            node_id.append(i % size)
            i //= size
        lattice.add_node(phys_dimension, tuple(node_id))
        ids.append(node_id)
    for j in ids:
        for pos in range(len(j)):
            next_j = j.copy()
            next_j[pos] += 1
            if lattice.does_node_exist(tuple(next_j)):
                lattice.add_edge((tuple(j), tuple(next_j)), bond_dimension)
            elif not open_boundary:
                next_j[pos] = 0
                lattice.add_edge((tuple(j), tuple(next_j)), bond_dimension)
    return lattice


# Heavy-hex rows and bridges of the 127-qubit Eagle layout
# (tensor_graph.py:547-613): seven chains of consecutive labels and 48
# degree-2 bridge qubits, each listed as (upper, bridge, lower).
_EAGLE_ROWS = [(0, 13), (18, 32), (37, 51), (56, 70), (75, 89), (94, 108), (113, 126)]
_EAGLE_BRIDGES = [
    (0, 14, 18), (4, 15, 22), (8, 16, 26), (12, 17, 30),
    (20, 33, 39), (24, 34, 43), (28, 35, 47), (32, 36, 51),
    (37, 52, 56), (41, 53, 60), (45, 54, 64), (49, 55, 68),
    (58, 71, 77), (62, 72, 81), (66, 73, 85), (70, 74, 89),
    (75, 90, 94), (79, 91, 98), (83, 92, 102), (87, 93, 106),
    (96, 109, 114), (100, 110, 118), (104, 111, 122), (108, 112, 126),
]


def get_heavy_hex_ibm_eagle_lattice() -> TensorGraph:
    """127-node / 144-edge heavy-hex lattice, bond dimension 1."""
    lattice = TensorGraph()
    for _ in range(127):
        lattice.add_node()
    for first, last in _EAGLE_ROWS:
        for i in range(first, last):
            lattice.add_edge((i, i + 1), 1)
    for upper, bridge, lower in _EAGLE_BRIDGES:
        lattice.add_edge((upper, bridge), 1)
        lattice.add_edge((bridge, lower), 1)
    return lattice


def get_heavy_hex_ibm_eagle_lattice_infinite() -> TensorGraph:
    """Five-node unit cell of the infinite heavy-hex lattice
    (tensor_graph.py:621-631)."""
    lattice = TensorGraph()
    for _ in range(5):
        lattice.add_node(2)
    for e in [(0, 1), (1, 2), (2, 3), (2, 4), (3, 0), (4, 0)]:
        lattice.add_edge(e, 1)
    return lattice


def random_regular_pairs(nodes_number: int, degree: int, seed: int) -> List[Tuple[int, int]]:
    """Edges of a random ``degree``-regular simple graph by the pairing
    (configuration) model: shuffle ``nodes_number * degree`` stubs, pair them,
    and redraw the whole pairing whenever it has a self-loop or a multi-edge.

    This stands in for ``networkx.random_regular_graph`` used at
    examples/quantum_annealing/quantum_annealing/src/energy_function.py:226."""
    if (nodes_number * degree) % 2:
        raise ValueError("nodes_number * degree must be even.")
    rng = np.random.default_rng(seed)
    stubs = np.repeat(np.arange(nodes_number), degree)
    for _ in range(100000):
        perm = rng.permutation(stubs)
        a, b = perm[0::2], perm[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        keys = lo.astype(np.int64) * nodes_number + hi
        if np.unique(keys).size != keys.size:
            continue
        return [(int(x), int(y)) for x, y in zip(a, b)]
    raise RuntimeError("pairing model did not produce a simple graph")


def get_random_regular_graph(
    nodes_number: int, degree: int, phys_dimension: int, bond_dimension: int, seed: int
) -> TensorGraph:
    """Random regular tensor graph on integer labels from the pairing model."""
    graph = TensorGraph()
    for i in range(nodes_number):
        graph.add_node(phys_dimension, i)
    for u, v in random_regular_pairs(nodes_number, degree, seed):
        graph.add_edge((u, v), bond_dimension)
    return graph


def greedy_edge_coloring(graph: TensorGraph) -> List[List[EdgeID]]:
    """Splits the (two-node) edges into classes of node-disjoint edges.

    Edges are coloured in insertion order with colours 0..D-1, D the maximum
    degree. When no colour is free at both ends, the alternating a/b path
    from one end (a free at u, b free at v) is recoloured b/a, which frees a
    at v (Kempe chain). On bipartite graphs (heavy-hex, trees, open lattices)
    this always succeeds, so D classes suffice (Konig's edge-colouring
    theorem); when the path closes on an odd cycle a new colour is opened."""
    at: Dict[NodeID, Dict[int, EdgeID]] = {nid: {} for nid in graph.nodes}
    colour: Dict[EdgeID, int] = {}
    n_colours = max((n.degree for n in graph.nodes.values()), default=0)

    def other(eid, x):
        a, b = eid
        return b if x == a else a

    for eid, edge in graph.edges.items():
        if edge.degree != 2:
            raise NotImplementedError("edge colouring needs edges of degree 2")
        u, v = eid
        free_u = [c for c in range(n_colours) if c not in at[u]]
        free_v = [c for c in range(n_colours) if c not in at[v]]
        common = [c for c in free_u if c not in at[v]]
        if common:
            c = common[0]
        elif free_u and free_v:
            a, b = free_u[0], free_v[0]
            path, x, want = [], v, a
            while want in at[x]:
                e = at[x][want]
                path.append(e)
                x = other(e, x)
                want = b if want == a else a
            if x == u or any(u in e for e in path):
                c = n_colours
                n_colours += 1
            else:
                for e in path:
                    for y in e:
                        del at[y][colour[e]]
                for e in path:
                    colour[e] = b if colour[e] == a else a
                    for y in e:
                        at[y][colour[e]] = e
                c = a
        else:
            c = n_colours
            n_colours += 1
        colour[eid] = c
        at[u][c] = eid
        at[v][c] = eid
    classes: List[List[EdgeID]] = [[] for _ in range(n_colours)]
    for eid in graph.edges:
        classes[colour[eid]].append(eid)
    return [c for c in classes if c]
