"""FP64 numpy restatement of dequantizer/src/mappings/*.py and of the
tensor-valued TensorGraph methods (dequantizer/src/graph/tensor_graph.py:180-446).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Connectivity comes from ``dequantizer_b200.graph`` -- pure host bookkeeping
(node/edge lists, traversal order) with no arithmetic, checked on its own
against the reference's structure tests. Every number here is computed by
numpy from the restated reference algorithm.
"""

from typing import Dict, List

import numpy as np

from dequantizer_b200.graph import Edge, MessageID, Node, TensorGraph
from . import tensor_ops as ops


def get_belief_propagation_map(traverser, is_synchronous: bool = False):
    """mappings/belief_propagation.py:24-64: one sweep over the traversal list.

    Asynchronous mode (default) reads messages already updated earlier in the
    same sweep; synchronous mode reads only the input dict."""

    def bp_map(tensors, messages):
        updated: Dict[MessageID, np.ndarray] = {}
        for element in traverser:
            incoming = []
            for nb in element.neighbors:
                mid = MessageID(src=nb.id, dst=element.id)
                if is_synchronous:
                    incoming.append(messages[mid])
                else:
                    m = updated.get(mid)
                    incoming.append(messages[mid] if m is None else m)
            if isinstance(element, Node):
                out = ops.pass_through_node(tensors[element.id], incoming)
            else:
                out = ops.pass_through_edge(incoming)
            for nb, m in zip(element.neighbors, out):
                updated[MessageID(src=element.id, dst=nb.id)] = m
        return updated

    return bp_map


def messages_frob_distance(lhs, rhs) -> float:
    """mappings/messages_distance.py:14-22: mean Frobenius distance."""
    assert len(lhs) == len(rhs)
    dist = 0.0
    for key, arr in lhs.items():
        dist += float(np.linalg.norm(arr - rhs[key]))
    return dist / len(lhs)


def get_vidal_gauge_fixing_map(traverser, eps: float):
    """mappings/vidal_gauge.py:21-63: edge_svd on every edge, then absorb the
    orthogonalisers into every node."""

    def vg_map(tensors, messages):
        lambdas = {}
        gauged = {}
        orth = {}
        nodes = []
        for element in traverser:
            if isinstance(element, Edge):
                incoming = [messages[MessageID(src=nb.id, dst=element.id)] for nb in element.neighbors]
                local, lmbd = ops.edge_svd(incoming, eps)
                lambdas[element.id] = lmbd
                for g, nb in zip(local, element.neighbors):
                    orth[MessageID(src=element.id, dst=nb.id)] = g
            else:
                nodes.append(element)
        for node in nodes:
            mats = [orth[MessageID(src=nb.id, dst=node.id)] for nb in node.neighbors]
            gauged[node.id] = ops.absorb_by_node(tensors[node.id], mats)
        return gauged, lambdas

    return vg_map


def get_vidal_gauge_distance_map(traverser, eps: float):
    """mappings/vidal_distance.py:17-42: summed vidal_dist over nodes / 2|E|."""

    def vd_map(tensors, lambdas) -> float:
        dist = 0.0
        n_edges = 0
        for element in traverser:
            if isinstance(element, Node):
                lams = [lambdas[nb.id] for nb in element.neighbors]
                dist += ops.vidal_dist(tensors[element.id], lams, eps)
            else:
                n_edges += 1
        return dist / (2 * n_edges)

    return vd_map


def get_symmetric_gauge_fixing_map(traverser, eps: float):
    """mappings/symmetric_gauge.py:17-39."""

    def sg_map(tensors, lambdas):
        out = {}
        for element in traverser:
            if isinstance(element, Node):
                lams = [lambdas[nb.id] for nb in element.neighbors]
                out[element.id] = ops.canonicalize(tensors[element.id], lams, eps)
        return out

    return sg_map


def lambdas2messages(lambdas):
    """mappings/symmetric_gauge.py:50-61: diag(lambda) in both directions."""
    messages = {}
    for edge_id, lmbd in lambdas.items():
        m = np.diag(lmbd).astype(np.complex128)
        for node_id in edge_id:
            messages[MessageID(src=edge_id, dst=node_id)] = m
            messages[MessageID(src=node_id, dst=edge_id)] = m
    return messages


def get_one_side_density_matrix(node: Node, tensors, messages) -> np.ndarray:
    """mappings/density_matrix.py:16-37."""
    degree = node.degree
    tensor = tensors[node.id]
    assert degree == tensor.ndim - 1
    conj_tensor = np.transpose(tensor.conj(), [degree, *range(degree)]).reshape((tensor.shape[-1], -1))
    for nb in node.neighbors:
        tensor = np.tensordot(tensor, messages[MessageID(nb.id, node.id)], axes=[0, 1])
    tensor = tensor.reshape((tensor.shape[0], -1))
    dens = np.tensordot(tensor, conj_tensor, axes=[1, 1])
    return dens / np.trace(dens)


# ---------------------------------------------------------------------------
# TensorGraph tensor-valued methods (tensor_graph.py:180-446)
# ---------------------------------------------------------------------------


def init_tensors(graph: TensorGraph, initializer) -> Dict:
    """tensor_graph.py:180-195 (BFS order, shape-checked)."""
    out = {}
    for element in graph.get_traversal_iterator():
        if isinstance(element, Node):
            t = np.asarray(initializer(element))
            expected = (*element.bond_shape, element.dimension)
            if t.shape != expected:
                raise ValueError(f"Expected tensor of shape {expected} got tensor of shape {t.shape}.")
            out[element.id] = t.astype(np.complex128)
    return out


def truncate(graph: TensorGraph, tensors, lambdas, accuracy, max_rank=None):
    """tensor_graph.py:235-258: cut every bond to its rank, slice tensors."""
    new_lambdas = {}
    new_tensors = {}
    for edge_id, lmbd in lambdas.items():
        rank = ops.find_rank(lmbd, accuracy, max_rank)
        new_lambdas[edge_id] = lmbd[:rank]
        graph.get_edge(edge_id).dimension = int(min(rank, lmbd.shape[0]))
    for node_id, node in graph.nodes.items():
        t = tensors[node_id]
        shape = [nb.dimension for nb in node.neighbors]
        node.bond_shape = tuple(shape)
        new_tensors[node_id] = t[tuple(slice(0, s) for s in shape) + (slice(None),)]
    return new_tensors, new_lambdas


def apply1(graph: TensorGraph, node_id, tensors, gate):
    """tensor_graph.py:268-275."""
    t = np.tensordot(tensors[node_id], gate, axes=[-1, 1])
    tensors[node_id] = t / np.linalg.norm(t)
    return tensors


def _edge_and_nodes(graph: TensorGraph, id1, id2, gate):
    if gate.ndim != 4:
        raise ValueError("Gate must be a tensor of rank 4.")
    if gate.shape[3] != gate.shape[1] or gate.shape[2] != gate.shape[0]:
        raise ValueError("Input - output dimensions must match with each other.")
    edge = graph.find_edge(id1, id2)
    if edge is None:
        raise ValueError(f"Neither edge with ID {(id2, id1)} nor with ID {(id1, id2)} is found in the tensor graph.")
    if edge.degree != 2:
        raise NotImplementedError("apply2 is implemented only for two qubits.")
    return edge, graph.get_node(id1), graph.get_node(id2)


def apply2_to_vidal_canonical(graph, id1, id2, tensors, lambdas, gate, threshold, accuracy, max_rank=None):
    """tensor_graph.py:294-375."""
    edge, n1, n2 = _edge_and_nodes(graph, id1, id2, gate)
    i1 = n1.indices[edge.id]
    i2 = n2.indices[edge.id]
    h1, h2 = ops.decompose_gate(gate, threshold)
    l1 = [lambdas[nb.id] for nb in n1.neighbors]
    l2 = [lambdas[nb.id] for nb in n2.neighbors]
    t1, t2, lmbd, err, entropy = ops.simple_update(
        tensors[n1.id], tensors[n2.id], l1, l2, h1, h2, i1, i2, threshold, accuracy, max_rank
    )
    tensors[n1.id] = t1
    tensors[n2.id] = t2
    edge.dimension = lmbd.shape[0]
    n1.bond_shape = t1.shape[:-1]
    n2.bond_shape = t2.shape[:-1]
    lambdas[edge.id] = lmbd
    return tensors, lambdas, err, entropy


def apply2(graph, id1, id2, tensors, gate, threshold):
    """tensor_graph.py:387-446: untruncated gate-halves application."""
    edge, n1, n2 = _edge_and_nodes(graph, id1, id2, gate)
    i1 = n1.indices[edge.id]
    i2 = n2.indices[edge.id]
    h1, h2 = ops.decompose_gate(gate, threshold)
    t1, t2 = ops.apply_gate_halves(tensors[n1.id], tensors[n2.id], i1, i2, h1, h2)
    tensors[n1.id] = t1
    tensors[n2.id] = t2
    edge.dimension = h1.shape[0] * edge.dimension
    n1.bond_shape = t1.shape[:-1]
    n2.bond_shape = t2.shape[:-1]
    return tensors
