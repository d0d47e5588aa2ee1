"""Shared test helpers: seeded inputs and gauge-invariant comparisons."""

import string

import numpy as np

from dequantizer_b200.graph import Edge, MessageID, Node, TensorGraph


def random_tensors(graph: TensorGraph, seed: int, dims=None):
    """Independent complex normal node tensors (numpy), one generator per graph."""
    rng = np.random.default_rng(seed)
    out = {}
    for nid, node in graph.nodes.items():
        shape = tuple(node.bond_shape) + (node.dimension,)
        z = rng.standard_normal(shape + (2,))
        out[nid] = z[..., 0] + 1j * z[..., 1]
    return out


def random_messages(graph: TensorGraph, seed: int):
    """Independent random PSD messages for every directed (node, edge) pair."""
    rng = np.random.default_rng(seed)
    out = {}
    for eid, edge in graph.edges.items():
        c = edge.dimension
        for nd in edge.neighbors:
            for key in (MessageID(nd.id, eid), MessageID(eid, nd.id)):
                z = rng.standard_normal((c, c, 2))
                a = z[..., 0] + 1j * z[..., 1]
                out[key] = a @ a.conj().T
    return out


def to_np(x):
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def rel_err(a, b):
    a, b = to_np(a), to_np(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def contract_network(graph: TensorGraph, tensors, lambdas=None) -> np.ndarray:
    """Full contraction of a small network into a state vector over the
    physical indices (node insertion order); lambdas, when given, sit on the
    bonds. Used to compare gauge-fixed results gauge-invariantly."""
    letters = iter(string.ascii_letters)
    bond_letter = {eid: next(letters) for eid in graph.edges}
    operands, subs = [], []
    out = ""
    for nid, node in graph.nodes.items():
        s = "".join(bond_letter[e.id] for e in node.neighbors)
        p = next(letters)
        out += p
        operands.append(to_np(tensors[nid]))
        subs.append(s + p)
    if lambdas is not None:
        for eid in graph.edges:
            operands.append(to_np(lambdas[eid]).astype(np.complex128))
            subs.append(bond_letter[eid])
    expr = ",".join(subs) + "->" + out
    return np.einsum(expr, *operands, optimize=True).reshape(-1)


def state_fidelity(a: np.ndarray, b: np.ndarray) -> float:
    return float(abs(np.vdot(a, b)) / (np.linalg.norm(a) * np.linalg.norm(b)))


def two_site(t1, t2, i1, i2, lam) -> np.ndarray:
    """Theta = sum_j t1[.., j, ..] lam_j t2[.., j, ..] (bond-invariant)."""
    t1, t2, lam = to_np(t1), to_np(t2), to_np(lam).astype(np.complex128)
    a = np.moveaxis(t1, i1, -1) * lam
    b = np.moveaxis(t2, i2, -1)
    return np.tensordot(a, b, axes=[[-1], [-1]])


def heavy_cube() -> TensorGraph:
    """20-node cube with extra qubits on edges
    (quantum_emulator/graph_generators.py:9-37)."""
    g = TensorGraph()
    for _ in range(20):
        g.add_node()
    for e in [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7), (7, 0), (12, 13), (13, 14), (14, 15),
              (15, 16), (16, 17), (17, 18), (18, 19), (19, 12), (0, 8), (2, 9), (4, 10), (6, 11), (8, 12),
              (9, 14), (10, 16), (11, 18)]:
        g.add_edge(e, 1)
    return g


def small_heavy_hex() -> TensorGraph:
    """Two-cell heavy hex, 21 nodes (quantum_emulator/graph_generators.py:43-61)."""
    g = TensorGraph()
    for _ in range(21):
        g.add_node()
    for i in range(4):
        g.add_edge((i, i + 1), 1)
    for i in range(5, 11):
        g.add_edge((i, i + 1), 1)
    for i in range(12, 16):
        g.add_edge((i, i + 1), 1)
    for e in [(0, 17), (17, 7), (4, 18), (18, 11), (5, 19), (19, 12), (10, 20), (20, 16)]:
        g.add_edge(e, 1)
    return g


def random_q1_gate(rng) -> np.ndarray:
    z = rng.standard_normal((2, 2, 2))
    q, _ = np.linalg.qr(z[..., 0] + 1j * z[..., 1])
    return q


def random_ising_q2_gate(rng) -> np.ndarray:
    return np.diag(np.exp(1j * rng.standard_normal(4))).reshape((2, 2, 2, 2))
