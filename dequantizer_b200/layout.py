"""Packed device layout of a tensor graph (the tables of dqz_graph_t).

Nodes, edges and half-edges are numbered densely:
  * node v = position in ``nodes``; its tensor lives at ``node_off[v]`` in a
    flat complex128 arena, row-major over (a_0, ..., a_{k-1}, s);
  * half-edge h = node_half[v] + slot is bond ``slot`` of node v; its
    messages (node->edge and edge->node, chi x chi) live at
    ``half_msg_off[h]`` in flat complex128 arenas;
  * edge e = position in ``edges``; its lambda vector lives at
    ``edge_lam_off[e]`` in a flat float64 arena.

Offsets are computed from per-node / per-edge capacities, which may exceed
the current sizes (the emulator grows bonds in place). Current bond
dimensions are held in ``edge_chi`` both on the host and on the device; the
simple-update kernel updates the device copy itself and the host copy is
updated by the same rule on the host, so no device->host traffic is needed.
"""

from typing import Dict, List, Optional, Sequence

import ctypes
import numpy as np
import torch

from . import _lib
from .graph import Edge, Node


class GraphLayout:
    def __init__(
        self,
        nodes: Sequence[Node],
        edges: Sequence[Edge],
        edge_chi: Sequence[int],
        phys: Optional[Sequence[int]] = None,
        node_capacity: Optional[Sequence[int]] = None,
        edge_capacity: Optional[Sequence[int]] = None,
        device: Optional[torch.device] = None,
    ):
        self.nodes = list(nodes)
        self.edges = list(edges)
        self.device = device if device is not None else _lib.device()
        self.node_index: Dict = {n.id: i for i, n in enumerate(self.nodes)}
        self.edge_index: Dict = {e.id: i for i, e in enumerate(self.edges)}
        n, m = len(self.nodes), len(self.edges)
        self.n_nodes, self.n_edges = n, m
        self.degree = np.array([len(nd.neighbors) for nd in self.nodes], dtype=np.int32)
        if n and self.degree.max(initial=0) > _lib.MAX_DEGREE:
            raise NotImplementedError(f"node degree above {_lib.MAX_DEGREE} is not supported on the GPU")
        self.phys = np.array(phys if phys is not None else [nd.dimension for nd in self.nodes], dtype=np.int32)
        if n and self.phys.max(initial=1) > _lib.MAX_PHYS:
            raise NotImplementedError(f"physical dimension above {_lib.MAX_PHYS} is not supported on the GPU")
        self.node_half = np.zeros(n, dtype=np.int32)
        if n:
            self.node_half[1:] = np.cumsum(self.degree)[:-1]
        nh = int(self.degree.sum())
        self.n_halves = nh
        self.half_node = np.repeat(np.arange(n, dtype=np.int32), self.degree)
        self.half_edge = np.full(nh, -1, dtype=np.int32)
        self.edge_half = np.full(2 * m, -1, dtype=np.int32)
        for v, nd in enumerate(self.nodes):
            for slot, e in enumerate(nd.neighbors):
                ei = self.edge_index.get(e.id)
                if ei is None:
                    continue
                self.half_edge[self.node_half[v] + slot] = ei
        for ei, e in enumerate(self.edges):
            for side, nd in enumerate(e.neighbors[:2]):
                v = self.node_index.get(nd.id)
                if v is None:
                    continue
                self.edge_half[2 * ei + side] = self.node_half[v] + nd.indices[e.id]
        self.half_twin = np.full(nh, -1, dtype=np.int32)
        for ei in range(m):
            a, b = self.edge_half[2 * ei], self.edge_half[2 * ei + 1]
            if a >= 0 and b >= 0:
                self.half_twin[a] = b
                self.half_twin[b] = a
        self.edge_chi = np.array(edge_chi, dtype=np.int32)
        if m and self.edge_chi.max(initial=1) > _lib.MAX_CHI:
            raise NotImplementedError(f"bond dimension above {_lib.MAX_CHI} is not supported on the GPU")
        self.edge_capacity = np.array(edge_capacity if edge_capacity is not None else self.edge_chi, dtype=np.int64)
        self.edge_capacity = np.maximum(self.edge_capacity, self.edge_chi)
        self.node_capacity = np.array(
            node_capacity if node_capacity is not None else self.node_sizes(), dtype=np.int64
        )
        self.node_capacity = np.maximum(self.node_capacity, self.node_sizes())
        self._finish()

    # ------------------------------------------------------------- shapes
    def node_dims(self, v: int) -> List[int]:
        h0, k = self.node_half[v], self.degree[v]
        return [int(self.edge_chi[self.half_edge[h0 + j]]) for j in range(k)]

    def node_shape(self, v: int):
        return tuple(self.node_dims(v)) + (int(self.phys[v]),)

    def node_sizes(self) -> np.ndarray:
        """phys * product of the bond dimensions, per node (vectorised over
        the half-edge table, whose entries are grouped by node)."""
        sizes = np.array(self.phys, dtype=np.int64)
        if self.n_halves:
            dims = self.edge_chi[self.half_edge].astype(np.int64)
            has = self.degree > 0
            sizes[has] *= np.multiply.reduceat(dims, self.node_half[has])
        return sizes

    def half_chi(self) -> np.ndarray:
        return self.edge_chi[self.half_edge]

    def uniform_k3_chi(self) -> int:
        """Bond dimension when every node has degree 3 and physical dimension
        2 and every edge the same bond dimension in {8, 16} (the shapes the
        specialised node-update kernel covers); 0 otherwise."""
        if not self.n_nodes or not self.n_edges:
            return 0
        if not (np.all(self.degree == 3) and np.all(self.phys == 2)):
            return 0
        chi = int(self.edge_chi[0])
        if chi not in (8, 16) or not np.all(self.edge_chi == chi) or np.any(self.half_edge < 0):
            return 0
        return chi

    # ------------------------------------------------------------ offsets
    def _finish(self):
        self.node_off = np.zeros(self.n_nodes, dtype=np.int64)
        if self.n_nodes:
            self.node_off[1:] = np.cumsum(self.node_capacity)[:-1]
        self.tensor_elems = int(self.node_capacity.sum())
        hcap = self.edge_capacity[self.half_edge] if self.n_halves else np.zeros(0, dtype=np.int64)
        self.half_msg_off = np.zeros(self.n_halves, dtype=np.int64)
        if self.n_halves:
            self.half_msg_off[1:] = np.cumsum(hcap * hcap)[:-1]
        self.msg_elems = int((hcap * hcap).sum())
        self.edge_lam_off = np.zeros(self.n_edges, dtype=np.int64)
        if self.n_edges:
            self.edge_lam_off[1:] = np.cumsum(self.edge_capacity)[:-1]
        self.lam_elems = int(self.edge_capacity.sum())
        self.upload()

    def upload(self):
        dev = self.device

        def t(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)

        self.d_node_degree = t(self.degree, np.int32)
        self.d_node_phys = t(self.phys, np.int32)
        self.d_node_half = t(self.node_half, np.int32)
        self.d_node_off = t(self.node_off, np.int64)
        self.d_half_node = t(self.half_node, np.int32)
        self.d_half_edge = t(self.half_edge, np.int32)
        self.d_half_twin = t(self.half_twin, np.int32)
        self.d_half_msg_off = t(self.half_msg_off, np.int64)
        self.d_edge_half = t(self.edge_half, np.int32)
        self.d_edge_lam_off = t(self.edge_lam_off, np.int64)
        self.d_edge_chi = t(self.edge_chi, np.int32)
        self.desc = _lib.GraphDesc(
            self.n_nodes,
            self.n_edges,
            self.n_halves,
            *(
                x.data_ptr() if x.numel() else 0
                for x in (
                    self.d_node_degree,
                    self.d_node_phys,
                    self.d_node_half,
                    self.d_node_off,
                    self.d_half_node,
                    self.d_half_edge,
                    self.d_half_twin,
                    self.d_half_msg_off,
                    self.d_edge_half,
                    self.d_edge_lam_off,
                    self.d_edge_chi,
                )
            ),
        )

    def push_edge_chi(self):
        """Copies the host bond dimensions to the device table."""
        self.d_edge_chi.copy_(torch.from_numpy(self.edge_chi), non_blocking=False)

    @property
    def gptr(self):
        return ctypes.byref(self.desc)

    @property
    def handle(self) -> int:
        """Address of the table descriptor: the ``graph`` argument of the
        torch.ops.dqz operators (valid while this layout is alive)."""
        return ctypes.addressof(self.desc)

    # --------------------------------------------------------- capacities
    def max_chi(self) -> int:
        return int(self.edge_chi.max(initial=1))

    def max_size(self) -> int:
        return int(self.node_sizes().max(initial=1))

    def max_slice(self) -> int:
        """Largest bond slice (node size / bond dimension) over all half-edges."""
        sizes = self.node_sizes()
        if not self.n_halves:
            return 1
        return int((sizes[self.half_node] // np.maximum(self.half_chi(), 1)).max())

    # ---------------------------------------------------------- packing
    def new_tensor_arena(self) -> torch.Tensor:
        return torch.zeros(max(self.tensor_elems, 1), dtype=torch.complex128, device=self.device)

    def new_msg_arena(self) -> torch.Tensor:
        return torch.zeros(max(self.msg_elems, 1), dtype=torch.complex128, device=self.device)

    def new_lam_arena(self) -> torch.Tensor:
        return torch.zeros(max(self.lam_elems, 1), dtype=torch.float64, device=self.device)

    def exact(self) -> bool:
        return bool(np.all(self.node_capacity == self.node_sizes())) and bool(
            np.all(self.edge_capacity == self.edge_chi)
        )

    def pack_tensors(self, tensors_by_node: Sequence[torch.Tensor]) -> torch.Tensor:
        """Concatenates node tensors (in node order) into an arena; requires
        capacities equal to sizes."""
        if not self.n_nodes:
            return self.new_tensor_arena()
        parts = [t.reshape(-1) for t in tensors_by_node]
        if self.exact():
            return torch.cat(parts).to(torch.complex128)
        arena = self.new_tensor_arena()
        for v, p in enumerate(parts):
            arena[self.node_off[v] : self.node_off[v] + p.numel()] = p
        return arena

    def unpack_tensors(self, arena: torch.Tensor) -> List[torch.Tensor]:
        out = []
        for v in range(self.n_nodes):
            shape = self.node_shape(v)
            size = int(np.prod(shape))
            o = int(self.node_off[v])
            out.append(arena[o : o + size].view(shape))
        return out

    def pack_messages(self, mats_by_half: Sequence[torch.Tensor]) -> torch.Tensor:
        if not self.n_halves:
            return self.new_msg_arena()
        parts = [m.reshape(-1) for m in mats_by_half]
        if self.exact():
            return torch.cat(parts).to(torch.complex128)
        arena = self.new_msg_arena()
        for h, p in enumerate(parts):
            arena[self.half_msg_off[h] : self.half_msg_off[h] + p.numel()] = p
        return arena

    def message_view(self, arena: torch.Tensor, h: int) -> torch.Tensor:
        c = int(self.edge_chi[self.half_edge[h]])
        o = int(self.half_msg_off[h])
        return arena[o : o + c * c].view(c, c)

    def pack_lambdas(self, lams_by_edge: Sequence[torch.Tensor]) -> torch.Tensor:
        if not self.n_edges:
            return self.new_lam_arena()
        if self.exact():
            return torch.cat([l.reshape(-1).real.to(torch.float64) for l in lams_by_edge])
        arena = self.new_lam_arena()
        for e, l in enumerate(lams_by_edge):
            arena[self.edge_lam_off[e] : self.edge_lam_off[e] + l.numel()] = l.real
        return arena

    def lambda_view(self, arena: torch.Tensor, e: int) -> torch.Tensor:
        o = int(self.edge_lam_off[e])
        return arena[o : o + int(self.edge_chi[e])]


def layout_from_traverser(traverser, shapes_by_node: Dict, device=None) -> GraphLayout:
    """Layout over the nodes / edges of a traversal list, with bond dimensions
    read off the node tensor shapes (the reference maps take them from the
    arrays as well)."""
    nodes = [el for el in traverser if isinstance(el, Node)]
    edges = [el for el in traverser if isinstance(el, Edge)]
    chi = []
    for e in edges:
        dims = set()
        for nd in e.neighbors:
            shp = shapes_by_node.get(nd.id)
            if shp is not None:
                dims.add(int(shp[nd.indices[e.id]]))
        if len(dims) != 1:
            raise ValueError(f"inconsistent bond dimensions {sorted(dims)} on edge {e.id}")
        chi.append(dims.pop())
    phys = [int(shapes_by_node[nd.id][-1]) for nd in nodes]
    return GraphLayout(nodes, edges, chi, phys=phys, device=device)
