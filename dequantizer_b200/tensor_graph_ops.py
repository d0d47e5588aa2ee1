"""Tensor-valued TensorGraph methods, run on the GPU.

Mirrors dequantizer/src/graph/tensor_graph.py:
* init_tensors              -- :180-195
* truncate                  -- :235-258
* apply1                    -- :268-275
* apply2_to_vidal_canonical -- :294-375
* apply2                    -- :387-446

Like the reference these methods replace entries of the dict they are given
(and return it) and update the graph's bond-dimension bookkeeping
(Edge.dimension, Node.bond_shape). Replaced tensors are new device tensors;
the previous ones are never written to.
"""

from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .gates import decompose_gates
from .graph import Edge, Node, TensorGraph
from .layout import GraphLayout
from .maps import as_device, as_device_real

EMPTY = torch.empty(0)


def _find_rank(lmbd: np.ndarray, accuracy, rank) -> int:
    """Rank rule of tensor_ops.py:7-17 (host-side, on a copied spectrum)."""
    if accuracy is None:
        return int(lmbd.shape[0] if rank is None else rank)
    scale = np.sqrt((lmbd**2).sum())
    return int(lmbd.shape[0] - (np.sqrt(np.cumsum(lmbd[::-1] ** 2)) / scale < accuracy).sum())


def init_tensors(self: TensorGraph, initializer) -> Dict:
    out = {}
    for element in self.get_traversal_iterator():
        if isinstance(element, Node):
            t = initializer(element)
            expected = (*element.bond_shape, element.dimension)
            shape = tuple(t.shape)
            if shape != expected:
                raise ValueError(f"Expected tensor of shape {expected} got tensor of shape {shape}.")
            out[element.id] = as_device(t)
    return out


def init_messages_device(self: TensorGraph, initializer) -> Dict:
    return {k: as_device(v) for k, v in TensorGraph.init_messages(self, initializer).items()}


def truncate(self: TensorGraph, tensors: Dict, core_edge_tensors: Dict, accuracy, max_rank: Optional[int] = None):
    new_lambdas = {}
    new_tensors = {}
    for edge_id, lmbd in core_edge_tensors.items():
        lam = as_device_real(lmbd)
        if accuracy is None:
            rank = _find_rank(np.zeros(lam.shape[0]), None, max_rank)
        else:
            rank = _find_rank(lam.cpu().numpy(), accuracy, max_rank)
        rank = min(rank, lam.shape[0])
        new_lambdas[edge_id] = lam[:rank]
        self.get_edge(edge_id).dimension = rank
    for node_id, node in self.nodes.items():
        t = as_device(tensors[node_id])
        shape = [nb.dimension for nb in node.neighbors]
        node.bond_shape = tuple(shape)
        new_tensors[node_id] = t[tuple(slice(0, s) for s in shape) + (slice(None),)].contiguous()
    self.structure_version += 1
    return new_tensors, new_lambdas


def apply1(self: TensorGraph, node_id, tensors: Dict, gate) -> Dict:
    node = self.get_node(node_id)
    t = as_device(tensors[node_id])
    g = as_device(gate)
    d = t.shape[-1]
    if tuple(g.shape) != (d, d):
        raise ValueError(f"gate of shape {tuple(g.shape)} does not act on a physical dimension {d}")
    layout = GraphLayout([node], list(node.neighbors), list(t.shape[:-1]), phys=[d])
    T = t.reshape(-1).clone()
    gp = torch.zeros(_lib.MAX_PHYS * _lib.MAX_PHYS, dtype=torch.complex128, device=T.device)
    gp[: d * d] = g.reshape(-1)
    idx = torch.zeros(1, dtype=torch.int32, device=T.device)
    _lib.call("dqz_apply1", layout.gptr, T.data_ptr(), idx.data_ptr(), gp.data_ptr(), 1, _lib.stream_handle())
    tensors[node_id] = T.view(tuple(t.shape))
    return tensors


def _edge_nodes(self: TensorGraph, id1, id2, gate) -> Tuple[Edge, Node, Node, np.ndarray]:
    g = gate.detach().cpu().numpy() if isinstance(gate, torch.Tensor) else np.asarray(gate)
    if g.ndim != 4:
        raise ValueError("Gate must be a tensor of rank 4.")
    if g.shape[3] != g.shape[1] or g.shape[2] != g.shape[0]:
        raise ValueError("Input - output dimensions must match with each other.")
    edge = self.find_edge(id1, id2)
    if edge is None:
        raise ValueError(
            f"Neither edge with ID {(id2, id1)} nor with ID {(id1, id2)} is found in the tensor graph."
        )
    if edge.degree != 2:
        raise NotImplementedError("apply2 is implemented only for two qubits.")
    return edge, self.get_node(id1), self.get_node(id2), g


def apply2(self: TensorGraph, controlling_node_id, controlled_node_id, tensors: Dict, gate, threshold) -> Dict:
    edge, n1, n2, g = _edge_nodes(self, controlling_node_id, controlled_node_id, gate)
    i1, i2 = n1.indices[edge.id], n2.indices[edge.id]
    flat, ranks, _ = decompose_gates(np.transpose(g, (0, 1, 2, 3))[None], float(threshold))
    r = int(ranks[0])
    t1, t2 = as_device(tensors[n1.id]), as_device(tensors[n2.id])
    dev = t1.device
    shapes, outs = [], []
    for t, idx in ((t1, i1), (t2, i2)):
        k = t.dim() - 1
        row = np.zeros(_lib.MAX_DEGREE + 4, dtype=np.int32)
        row[:4] = (k, t.shape[-1], idx, r)
        row[4 : 4 + k] = t.shape[:-1]
        shapes.append(row)
        new_shape = list(t.shape)
        new_shape[idx] *= r
        outs.append(tuple(new_shape))
    in_arena = torch.cat([t1.reshape(-1), t2.reshape(-1)])
    sizes = [int(np.prod(s)) for s in outs]
    out_arena = torch.empty(sum(sizes), dtype=torch.complex128, device=dev)
    in_off = torch.tensor([0, t1.numel()], dtype=torch.int64, device=dev)
    out_off = torch.tensor([0, sizes[0]], dtype=torch.int64, device=dev)
    shape_t = torch.from_numpy(np.stack(shapes)).to(dev)
    halves = torch.from_numpy(flat.reshape(2, -1)).to(dev)
    _lib.call("dqz_apply_half_gates", in_arena.data_ptr(), out_arena.data_ptr(), in_off.data_ptr(),
              out_off.data_ptr(), shape_t.data_ptr(), halves.data_ptr(), 2, _lib.stream_handle())
    tensors[n1.id] = out_arena[: sizes[0]].view(outs[0])
    tensors[n2.id] = out_arena[sizes[0] :].view(outs[1])
    edge.dimension = r * edge.dimension
    n1.bond_shape = outs[0][:-1]
    n2.bond_shape = outs[1][:-1]
    self.structure_version += 1
    return tensors


def simple_update_shapes(dims1, d1, i1, dims2, d2, i2, r, max_rank):
    """Host-side shape rule of tensor_ops.py:318-389: returns
    (rows1, rows2, cols, new bond dimension, full rank kk)."""
    chi = dims1[i1]
    m1 = d1 * int(np.prod([c for j, c in enumerate(dims1) if j != i1]))
    m2 = d2 * int(np.prod([c for j, c in enumerate(dims2) if j != i2]))
    k = chi * r
    kk = min(min(m1, k), min(m2, k))
    new = kk if max_rank is None else min(int(max_rank), kk)
    return m1, m2, k, new, kk


def apply2_to_vidal_canonical(
    self: TensorGraph,
    controlling_node_id,
    controlled_node_id,
    tensors: Dict,
    lambdas: Dict,
    gate,
    threshold,
    accuracy,
    max_rank: Optional[int] = None,
):
    edge, n1, n2, g = _edge_nodes(self, controlling_node_id, controlled_node_id, gate)
    eps = float(threshold)
    flat, ranks, _ = decompose_gates(g[None], eps)
    r = int(ranks[0])
    t1, t2 = as_device(tensors[n1.id]), as_device(tensors[n2.id])
    dims1, dims2 = list(t1.shape[:-1]), list(t2.shape[:-1])
    i1, i2 = n1.indices[edge.id], n2.indices[edge.id]
    m1, m2, k, new_chi, kk = simple_update_shapes(dims1, t1.shape[-1], i1, dims2, t2.shape[-1], i2, r,
                                                  None if accuracy is not None else max_rank)
    if k > _lib.MAX_CHI:
        raise NotImplementedError(f"bond dimension x gate rank = {k} above {_lib.MAX_CHI} is not supported")
    # mini layout: the two nodes and every edge touching them
    edges, seen = [], set()
    for nd in (n1, n2):
        for e in nd.neighbors:
            if e.id not in seen:
                seen.add(e.id)
                edges.append(e)
    chi = []
    for e in edges:
        if e is edge:
            chi.append(dims1[i1])
        elif e.id in n1.indices and e in n1.neighbors:
            chi.append(dims1[n1.indices[e.id]])
        else:
            chi.append(dims2[n2.indices[e.id]])
    s1_new = t1.numel() // dims1[i1] * new_chi
    s2_new = t2.numel() // dims2[i2] * new_chi
    cap_e = [max(c, new_chi) if e is edge else c for e, c in zip(edges, chi)]
    layout = GraphLayout(
        [n1, n2], edges, chi, phys=[t1.shape[-1], t2.shape[-1]],
        node_capacity=[max(t1.numel(), s1_new), max(t2.numel(), s2_new)], edge_capacity=cap_e,
    )
    dev = layout.device
    T = layout.pack_tensors([t1, t2])
    lam = layout.pack_lambdas([as_device_real(lambdas[e.id]) for e in edges])
    e_idx = torch.tensor([layout.edge_index[edge.id]], dtype=torch.int32, device=dev)
    first = 1 if edge.neighbors[0] is n1 else 0
    ctrl = torch.tensor([first], dtype=torch.uint8, device=dev)
    halves = torch.from_numpy(flat.reshape(-1)).to(dev)
    rk = torch.tensor([r], dtype=torch.int32, device=dev)
    err = torch.empty(1, dtype=torch.float64, device=dev)
    ent = torch.empty(1, dtype=torch.float64, device=dev)
    rows, cols = max(m1, m2), k
    scratch = torch.empty(
        max(_lib.lib().dqz_simple_update_scratch_bytes(1, rows, cols), 1), dtype=torch.uint8, device=dev
    )
    run_rank = new_chi if accuracy is None else kk
    _lib.call("dqz_simple_update", layout.gptr, T.data_ptr(), lam.data_ptr(), e_idx.data_ptr(), ctrl.data_ptr(),
              halves.data_ptr(), rk.data_ptr(), 1, eps, int(run_rank), rows, cols, err.data_ptr(), ent.data_ptr(),
              scratch.data_ptr(), _lib.stream_handle())
    ei = layout.edge_index[edge.id]
    layout.edge_chi[ei] = run_rank
    ts = layout.unpack_tensors(T)
    lam_e = lam[layout.edge_lam_off[ei] : layout.edge_lam_off[ei] + run_rank]
    err_v, ent_v = err[0], ent[0]
    if accuracy is not None:
        full = lam_e.cpu().numpy()
        rank = min(_find_rank(full, accuracy, max_rank), full.shape[0])
        nrm = np.linalg.norm(full)
        err_v = torch.tensor(float(np.linalg.norm(full[rank:] / nrm)), dtype=torch.float64, device=dev)
        sl1 = [slice(None)] * t1.dim()
        sl1[i1] = slice(0, rank)
        sl2 = [slice(None)] * t2.dim()
        sl2[i2] = slice(0, rank)
        ts = [ts[0][tuple(sl1)].contiguous(), ts[1][tuple(sl2)].contiguous()]
        lam_e = lam_e[:rank]
    tensors[n1.id] = ts[0]
    tensors[n2.id] = ts[1]
    edge.dimension = int(lam_e.shape[0])
    n1.bond_shape = tuple(ts[0].shape[:-1])
    n2.bond_shape = tuple(ts[1].shape[:-1])
    lambdas[edge.id] = lam_e
    self.structure_version += 1
    return tensors, lambdas, err_v, ent_v


def install():
    """Attaches the GPU-backed tensor methods to TensorGraph."""
    TensorGraph.init_tensors = init_tensors
    TensorGraph.truncate = truncate
    TensorGraph.apply1 = apply1
    TensorGraph.apply2 = apply2
    TensorGraph.apply2_to_vidal_canonical = apply2_to_vidal_canonical
    TensorGraph.init_messages_device = init_messages_device
