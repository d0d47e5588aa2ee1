"""Graph-wide maps with the reference's dict-in / dict-out interface, run on
the GPU through libdqz.

Each factory mirrors its reference counterpart and returns a pure callable
over ``Dict[NodeID, Tensor]`` / ``Dict[MessageID, Tensor]`` /
``Dict[EdgeID, Tensor]`` that returns NEW dicts (values are views into fresh
device arenas; inputs are never modified):

* get_belief_propagation_map     -- mappings/belief_propagation.py:24-64
* get_vidal_gauge_fixing_map     -- mappings/vidal_gauge.py:21-63
* get_vidal_gauge_distance_map   -- mappings/vidal_distance.py:17-42
* get_symmetric_gauge_fixing_map -- mappings/symmetric_gauge.py:17-39
* lambdas2messages               -- mappings/symmetric_gauge.py:50-61
* messages_frob_distance         -- mappings/messages_distance.py:14-22
* get_one_side_density_matrix    -- mappings/density_matrix.py:16-37

Tensors must be complex128 CUDA tensors (anything else is converted on the
device; host arrays are copied to the device first).
"""

from typing import Dict, List

import numpy as np
import torch

from . import _lib
from .graph import Edge, MessageID, Node
from .layout import GraphLayout, layout_from_traverser


def as_device(x) -> torch.Tensor:
    """complex128 CUDA tensor from a tensor or array (host data is copied)."""
    if isinstance(x, torch.Tensor):
        t = x
    else:
        t = torch.from_numpy(np.asarray(x))
    if not t.is_cuda:
        if not torch.cuda.is_available():
            raise RuntimeError("dequantizer_b200 runs on the GPU only and no CUDA device is available")
        t = t.to(_lib.device())
    if t.dtype != torch.complex128:
        t = t.to(torch.complex128)
    return t.contiguous()


def as_device_real(x) -> torch.Tensor:
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.asarray(x))
    if not t.is_cuda:
        if not torch.cuda.is_available():
            raise RuntimeError("dequantizer_b200 runs on the GPU only and no CUDA device is available")
        t = t.to(_lib.device())
    if t.is_complex():
        t = t.real
    return t.to(torch.float64).contiguous()


def _scratch(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


class Topology:
    """Node / edge order of a traversal list and, for the BP sweep, the
    per-half-edge message sources and node levels that reproduce the
    reference's sweep order exactly.

    Asynchronous sweep (belief_propagation.py:39-45): elements are visited in
    traversal order and read messages already updated in the same sweep.
    For node v, bond to edge e with far end u:
      * e after v                -> e2n from the previous sweep (SRC_E2N_OLD)
      * e before v, u before e   -> u's node->edge message of this sweep (SRC_N2E_NEW)
      * e before v, u after e    -> u's node->edge message of the previous sweep (SRC_N2E_OLD)
    Nodes whose inputs are all available form a level; levels run in order.
    The edge->node output of e toward v is u's node->edge message as it was
    when e was visited (new iff u before e)."""

    def __init__(self, traverser, is_synchronous: bool, flooding: bool = False):
        self.traverser = list(traverser)
        self.flooding = flooding
        self.nodes: List[Node] = [el for el in self.traverser if isinstance(el, Node)]
        self.edges: List[Edge] = [el for el in self.traverser if isinstance(el, Edge)]
        self.is_synchronous = is_synchronous
        self.node_index = {n.id: i for i, n in enumerate(self.nodes)}
        pos = {el.id: i for i, el in enumerate(self.traverser)}
        degree = [len(n.neighbors) for n in self.nodes]
        self.node_half = np.zeros(len(self.nodes), dtype=np.int64)
        if self.nodes:
            self.node_half[1:] = np.cumsum(degree)[:-1]
        nh = int(sum(degree))
        self.n_halves = nh
        self.src_sel = np.zeros(nh, dtype=np.uint8)
        self.edge_new = np.zeros(nh, dtype=np.uint8)
        level = np.zeros(len(self.nodes), dtype=np.int64)
        for v, nd in enumerate(self.nodes):
            lv = 0
            for slot, e in enumerate(nd.neighbors):
                if e.degree != 2:
                    raise NotImplementedError("BP on the GPU supports edges of degree 2 only")
                u = e.neighbors[1] if e.neighbors[0] is nd else e.neighbors[0]
                h = self.node_half[v] + slot
                if u.id in pos and pos[u.id] < pos[e.id]:
                    self.edge_new[h] = 1
                if flooding:
                    # every node reads the far end's node->edge message of the
                    # previous sweep; edges forward this sweep's messages
                    self.src_sel[h] = _lib.SRC_N2E_OLD
                    self.edge_new[h] = 1
                elif is_synchronous:
                    self.src_sel[h] = _lib.SRC_E2N_OLD
                    self.edge_new[h] = 0
                elif pos[e.id] < pos[nd.id]:
                    if pos[u.id] < pos[e.id]:
                        self.src_sel[h] = _lib.SRC_N2E_NEW
                        lv = max(lv, int(level[self.node_index[u.id]]) + 1)
                    else:
                        self.src_sel[h] = _lib.SRC_N2E_OLD
                else:
                    self.src_sel[h] = _lib.SRC_E2N_OLD
            level[v] = lv
        self.levels = []        # half-edges per level
        self.node_levels = []   # nodes per level
        if self.nodes:
            for lv in range(int(level.max()) + 1):
                vs = np.nonzero(level == lv)[0]
                halves = np.concatenate([np.arange(self.node_half[v], self.node_half[v] + degree[v]) for v in vs])
                self.levels.append(halves.astype(np.int32))
                self.node_levels.append(vs.astype(np.int32))
        self._dev = None
        self._dev_nodes = None

    def device_tables(self, device):
        if self._dev is None:
            self._dev = (
                torch.from_numpy(self.src_sel).to(device),
                torch.from_numpy(self.edge_new).to(device),
                [torch.from_numpy(l).to(device) for l in self.levels],
            )
        return self._dev

    def device_level_tables(self, device):
        """The levels as one flat half-edge list with offsets, the widest
        level's size, and two words of barrier scratch, for the one-launch sweep
        (dqz_bp_sweep_levels). Sweeps of one topology share the scratch, so
        they run on one stream at a time."""
        if getattr(self, "_dev_flat", None) is None:
            flat = np.concatenate(self.levels).astype(np.int32) if self.levels else np.zeros(0, np.int32)
            off = np.zeros(len(self.levels) + 1, dtype=np.int32)
            off[1:] = np.cumsum([len(l) for l in self.levels])
            self._dev_flat = (torch.from_numpy(flat).to(device), torch.from_numpy(off).to(device),
                              max((len(l) for l in self.levels), default=0),
                              torch.zeros(2, dtype=torch.int32, device=device))
        return self._dev_flat

    def device_slice_items(self, layout, device):
        """The (half-edge, slice) work items of every level for the sliced
        one-launch sweep (dqz_bp_sweep_sliced), from the layout's current bond
        dimensions: item_half, item_slice, per-level offsets, the largest level."""
        key = layout.edge_chi.tobytes()
        cache = self.__dict__.setdefault("_dev_items", {})
        if key not in cache:
            he = layout.half_edge
            ce = np.where(he >= 0, layout.edge_chi[np.maximum(he, 0)], 0).astype(np.int64)
            halves, slices, off = [], [], [0]
            for lv in self.levels:
                c = ce[lv]
                halves.append(np.repeat(lv, c))
                slices.append(np.concatenate([np.arange(x) for x in c]) if len(c) else np.zeros(0, np.int64))
                off.append(off[-1] + int(c.sum()))
            ih = np.concatenate(halves).astype(np.int32)
            isl = np.concatenate(slices).astype(np.int32)
            widest = int(np.max(np.diff(off))) if len(off) > 1 else 0
            if len(cache) > 8:
                cache.clear()
            cache[key] = (torch.from_numpy(ih).to(device), torch.from_numpy(isl).to(device),
                          torch.from_numpy(np.array(off, dtype=np.int32)).to(device), widest)
        return cache[key]

    def device_plan(self, layout, device):
        """The plan of the one-CTA sweep (dqz_bp_sweep_planned): per half-edge of
        the flat level table, node offset, degree, physical dimension, slot,
        outgoing message offset, bond dimensions, and the incoming messages as
        offset * 4 + source, from the layout's current bond dimensions."""
        key = layout.edge_chi.tobytes()
        cache = self.__dict__.setdefault("_dev_plan", {})
        if key not in cache:
            H = (np.concatenate(self.levels) if self.levels else np.zeros(0, np.int32)).astype(np.int64)
            v = layout.half_node[H].astype(np.int64)
            h0 = layout.node_half[v].astype(np.int64)
            k = layout.degree[v].astype(np.int64)
            md = _lib.MAX_DEGREE
            plan = np.zeros((len(H), _lib.PLAN_WORDS), dtype=np.int64)
            plan[:, 0] = layout.node_off[v]
            plan[:, 1] = k
            plan[:, 2] = layout.phys[v]
            plan[:, 3] = H - h0
            plan[:, 4] = layout.half_msg_off[H]
            slot = np.zeros(len(H), dtype=np.int64)
            twin = layout.half_twin
            for j in range(md):
                has = j < k
                hf = np.where(has, h0 + j, 0)
                he = layout.half_edge[hf]
                plan[:, 5 + j] = np.where(has, layout.edge_chi[np.maximum(he, 0)], 0)
                other = has & (j != plan[:, 3])
                sel = self.src_sel[hf].astype(np.int64)
                off = np.where(sel == _lib.SRC_E2N_OLD, layout.half_msg_off[hf],
                               layout.half_msg_off[np.maximum(twin[hf], 0)])
                rows = np.nonzero(other)[0]
                plan[rows, 5 + md + slot[rows]] = off[rows] * 4 + sel[rows]
                slot += other
            if len(cache) > 8:
                cache.clear()
            cache[key] = torch.from_numpy(plan).to(device)
        return cache[key]

    def device_node_levels(self, device):
        if self._dev_nodes is None:
            self._dev_nodes = [torch.from_numpy(l).to(device) for l in self.node_levels]
        return self._dev_nodes

    def half_ids(self):
        """(node, edge) element pairs of every half-edge, in half-edge order."""
        return [(nd, e) for nd in self.nodes for e in nd.neighbors]


class _LayoutCache:
    def __init__(self, topo: Topology):
        self.topo = topo
        self._key = None
        self._layout = None

    def get(self, tensors) -> GraphLayout:
        shapes = {n.id: tuple(tensors[n.id].shape) for n in self.topo.nodes}
        key = tuple(shapes[n.id] for n in self.topo.nodes)
        if key != self._key:
            self._layout = layout_from_traverser(self.topo.traverser, shapes)
            self._key = key
        return self._layout


_ERROR_FLAGS = {}


def error_flag(device) -> torch.Tensor:
    """Device int set by kernels that skip work items of an unexpected shape."""
    key = str(device)
    if key not in _ERROR_FLAGS:
        _ERROR_FLAGS[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _ERROR_FLAGS[key]


BF16_KERNELS = {"tcgen05": "dqz_bp_node_update_k3_umma", "mma_sync": "dqz_bp_node_update_k3_tc"}

# bonds from which the one-launch asynchronous sweep spreads slices (not whole
# half-edges) over the grid: at bond 32 a level of the heavy-hex DFS schedule
# has a handful of half-edges of ~50 MFLOP each
SLICED_MIN_CHI = 8


def bp_sweep(layout: GraphLayout, topo: Topology, T, n2e_old, e2n_old, n2e_new, e2n_new, mid_event=None,
             T_bf16=None, bf16_kernel: str = "tcgen05"):
    """One sweep on packed arenas: node updates level by level, then the edge pass
    (``mid_event``, a torch.cuda.Event, is recorded between the two).

    complex128 arenas use the specialised degree-3 kernel when every node
    has that shape (layout.uniform_k3_chi), the generic kernel otherwise;
    complex64 arenas need the specialised shape and run in FP32, or, when
    ``T_bf16`` is given, as BF16 tensor-core products with FP32 accumulation
    (bonds of dimension 16): ``bf16_kernel`` "tcgen05" takes the core layouts
    of dqz_pack_bf16_umma, "mma_sync" the planes of dqz_pack_bf16_planes."""
    src_sel, edge_new, levels = topo.device_tables(layout.device)
    stream = _lib.stream_handle()
    chi3 = layout.uniform_k3_chi()
    if T.dtype == torch.complex64:
        if not chi3 or (T_bf16 is not None and chi3 != 16):
            raise NotImplementedError("complex64 BP needs degree-3 nodes with bonds of dimension 8 or 16 "
                                      "(16 for the tensor-core form)")
        flag = error_flag(layout.device)
        if T_bf16 is not None:
            for nodes in topo.device_node_levels(layout.device):
                _lib.call(BF16_KERNELS[bf16_kernel], layout.gptr, T_bf16.data_ptr(), n2e_old.data_ptr(),
                          e2n_old.data_ptr(), n2e_new.data_ptr(), src_sel.data_ptr(), nodes.data_ptr(),
                          nodes.numel(), flag.data_ptr(), stream)
        else:
            for halves in levels:
                _lib.call("dqz_bp_node_update_k3", layout.gptr, chi3, 32, T.data_ptr(), n2e_old.data_ptr(),
                          e2n_old.data_ptr(), n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(),
                          halves.numel(), flag.data_ptr(), stream)
        if mid_event is not None:
            mid_event.record(torch.cuda.current_stream())
        _lib.call("dqz_bp_edge_pass_c64", layout.gptr, n2e_old.data_ptr(), n2e_new.data_ptr(), edge_new.data_ptr(),
                  e2n_new.data_ptr(), stream)
        return
    if chi3:
        flag = error_flag(layout.device)
        for halves in levels:
            _lib.call("dqz_bp_node_update_k3", layout.gptr, chi3, 64, T.data_ptr(), n2e_old.data_ptr(),
                      e2n_old.data_ptr(), n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), halves.numel(),
                      flag.data_ptr(), stream)
        if mid_event is not None:
            mid_event.record(torch.cuda.current_stream())
        _lib.call("dqz_bp_edge_pass", layout.gptr, n2e_old.data_ptr(), n2e_new.data_ptr(), edge_new.data_ptr(),
                  e2n_new.data_ptr(), chi3, stream)
        return
    max_slice, max_chi = layout.max_slice(), layout.max_chi()
    if len(topo.levels) > 1:
        # a schedule of several node levels (the reference's asynchronous sweep):
        # all levels and the edge pass in one launch when a slice fits on chip
        flat, off, widest, sync = topo.device_level_tables(layout.device)
        if max_chi >= SLICED_MIN_CHI:
            # large bonds: every (half-edge, slice) of a level is a work item, so a
            # level of a few half-edges still spreads over the whole GPU
            ih, isl, ioff, widest_items = topo.device_slice_items(layout, layout.device)
            status = _lib.lib().dqz_bp_sweep_sliced(
                layout.gptr, T.data_ptr(), n2e_old.data_ptr(), e2n_old.data_ptr(), n2e_new.data_ptr(),
                e2n_new.data_ptr(), src_sel.data_ptr(), edge_new.data_ptr(), flat.data_ptr(), off.data_ptr(),
                ih.data_ptr(), isl.data_ptr(), ioff.data_ptr(), len(topo.levels), widest_items, max_slice, max_chi,
                sync.data_ptr(), error_flag(layout.device).data_ptr(), stream)
        elif max_slice <= 256 and widest <= 64 and _lib.lib().dqz_get_tuning(_lib.TUNE_SWEEP_ONECTA) == 0:
            # small nodes and narrow levels: one CTA, a warp per half-edge, driven by the plan
            # (knob sweep_onecta: 1 = the cooperative grid, 2 = the one-CTA form without a plan)
            status = _lib.lib().dqz_bp_sweep_planned(
                layout.gptr, T.data_ptr(), n2e_old.data_ptr(), e2n_old.data_ptr(), n2e_new.data_ptr(),
                e2n_new.data_ptr(), edge_new.data_ptr(), topo.device_plan(layout, layout.device).data_ptr(),
                off.data_ptr(), len(topo.levels), widest, max_slice, max_chi, stream)
        else:
            status = _lib.lib().dqz_bp_sweep_levels(
                layout.gptr, T.data_ptr(), n2e_old.data_ptr(), e2n_old.data_ptr(), n2e_new.data_ptr(),
                e2n_new.data_ptr(), src_sel.data_ptr(), edge_new.data_ptr(), flat.data_ptr(), off.data_ptr(),
                len(topo.levels), widest, max_slice, max_chi, sync.data_ptr(), error_flag(layout.device).data_ptr(),
                stream)
        if status == _lib.DQZ_OK:
            if mid_event is not None:
                mid_event.record(torch.cuda.current_stream())
            return
        if status != _lib.DQZ_ERR_UNSUPPORTED:
            _lib.check("dqz_bp_sweep_levels", status)
    scratch = None
    nbytes = _lib.lib().dqz_bp_node_scratch_bytes(max(len(l) for l in topo.levels), max_slice, max_chi)
    if nbytes:
        scratch = _scratch(nbytes, layout.device)
    for halves in levels:
        _lib.call(
            "dqz_bp_node_update", layout.gptr, T.data_ptr(), n2e_old.data_ptr(), e2n_old.data_ptr(),
            n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), halves.numel(), max_slice, max_chi,
            _lib.ptr(scratch), stream,
        )
    if mid_event is not None:
        mid_event.record(torch.cuda.current_stream())
    _lib.call(
        "dqz_bp_edge_pass", layout.gptr, n2e_old.data_ptr(), n2e_new.data_ptr(), edge_new.data_ptr(),
        e2n_new.data_ptr(), max_chi, stream,
    )


def get_belief_propagation_map(traverser, is_synchronous: bool = False):
    topo = Topology(traverser, is_synchronous)
    cache = _LayoutCache(topo)
    halves = topo.half_ids()

    def belief_propagation_map(tensors: Dict, messages: Dict) -> Dict:
        dev_t = {n.id: as_device(tensors[n.id]) for n in topo.nodes}
        layout = cache.get(dev_t)
        T = layout.pack_tensors([dev_t[n.id] for n in topo.nodes])
        n2e_old = layout.pack_messages([as_device(messages[MessageID(nd.id, e.id)]) for nd, e in halves])
        e2n_old = layout.pack_messages([as_device(messages[MessageID(e.id, nd.id)]) for nd, e in halves])
        n2e_new = torch.empty_like(n2e_old)
        e2n_new = torch.empty_like(e2n_old)
        bp_sweep(layout, topo, T, n2e_old, e2n_old, n2e_new, e2n_new)
        hidx = {(nd.id, e.id): h for h, (nd, e) in enumerate(halves)}
        out = {}
        for el in topo.traverser:
            if isinstance(el, Node):
                for e in el.neighbors:
                    out[MessageID(el.id, e.id)] = layout.message_view(n2e_new, hidx[(el.id, e.id)])
            else:
                for nd in el.neighbors:
                    out[MessageID(el.id, nd.id)] = layout.message_view(e2n_new, hidx[(nd.id, el.id)])
        return out

    return belief_propagation_map


def messages_frob_distance(lhs: Dict, rhs: Dict) -> torch.Tensor:
    n = len(lhs)
    assert n == len(rhs), f"{n}, {len(rhs)}"
    keys = list(lhs.keys())
    a = [as_device(lhs[k]).reshape(-1) for k in keys]
    b = [as_device(rhs[k]).reshape(-1) for k in keys]
    sizes = np.array([x.numel() for x in a], dtype=np.int64)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    dev = a[0].device
    A, B = torch.cat(a), torch.cat(b)
    d_off = torch.from_numpy(off).to(dev)
    partial = torch.empty(n, dtype=torch.float64, device=dev)
    out = torch.empty((), dtype=torch.float64, device=dev)
    _lib.call("dqz_segment_distance", A.data_ptr(), B.data_ptr(), d_off.data_ptr(), n, partial.data_ptr(),
              out.data_ptr(), _lib.stream_handle())
    return out


def vidal_gauge_packed(layout: GraphLayout, T, n2e, eps: float, out=None, edges=None, nodes=None):
    """Vidal gauge on packed arenas: returns (Gamma arena, lambda arena).

    ``out`` = (G, lam, orth) arenas to write into (new ones when None);
    ``edges`` / ``nodes`` (int32 device tensors) restrict the work to those
    edges (lambdas, orthogonalisers) and nodes (Gamma tensors), leaving the
    rest of ``out`` as it is."""
    stream = _lib.stream_handle()
    max_chi = layout.max_chi()
    if out is None:
        G = torch.empty_like(T)
        lam = layout.new_lam_arena()
        orth = torch.empty(max(layout.msg_elems, 1), dtype=torch.complex128, device=layout.device)
    else:
        G, lam, orth = out
    ne = layout.n_edges if edges is None else int(edges.numel())
    nb = _lib.lib().dqz_vidal_edges_scratch_bytes(ne, max_chi)
    scratch = _scratch(nb, layout.device) if nb else None
    _lib.call("dqz_vidal_edges", layout.gptr, n2e.data_ptr(), float(eps), orth.data_ptr(), lam.data_ptr(), max_chi,
              _lib.ptr(edges), ne if edges is not None else 0, _lib.ptr(scratch), stream)
    nn = layout.n_nodes if nodes is None else int(nodes.numel())
    chi3 = layout.uniform_k3_chi()
    if chi3:
        _lib.call("dqz_absorb_k3", layout.gptr, chi3, T.data_ptr(), orth.data_ptr(), G.data_ptr(), _lib.ptr(nodes),
                  nn if nodes is not None else 0, error_flag(layout.device).data_ptr(), stream)
        return G, lam
    ms = layout.max_size()
    nb = _lib.lib().dqz_absorb_scratch_bytes(nn, ms)
    if nb and G.data_ptr() != T.data_ptr():
        # nodes too large for shared memory: one CTA per (node, first-bond index)
        part = _scratch(_lib.lib().dqz_absorb_split_scratch_bytes(nn), layout.device)
        status = _lib.lib().dqz_absorb_split(layout.gptr, T.data_ptr(), orth.data_ptr(), G.data_ptr(),
                                             layout.max_slice(), _lib.ptr(nodes), nn if nodes is not None else 0,
                                             part.data_ptr(), stream)
        if status == _lib.DQZ_OK:
            return G, lam
        if status != _lib.DQZ_ERR_UNSUPPORTED:
            _lib.check("dqz_absorb_split", status)
    scratch = _scratch(nb, layout.device) if nb else None
    _lib.call("dqz_absorb", layout.gptr, T.data_ptr(), orth.data_ptr(), G.data_ptr(), ms, _lib.ptr(nodes),
              nn if nodes is not None else 0, _lib.ptr(scratch), stream)
    return G, lam


def get_vidal_gauge_fixing_map(traverser, eps):
    topo = Topology(traverser, True)
    cache = _LayoutCache(topo)
    halves = topo.half_ids()

    def vidal_gauge_fixing_map(tensors: Dict, messages: Dict):
        dev_t = {n.id: as_device(tensors[n.id]) for n in topo.nodes}
        layout = cache.get(dev_t)
        T = layout.pack_tensors([dev_t[n.id] for n in topo.nodes])
        n2e = layout.pack_messages([as_device(messages[MessageID(nd.id, e.id)]) for nd, e in halves])
        G, lam = vidal_gauge_packed(layout, T, n2e, float(eps))
        gs = layout.unpack_tensors(G)
        gauged = {n.id: gs[i] for i, n in enumerate(topo.nodes)}
        lambdas = {e.id: layout.lambda_view(lam, i) for i, e in enumerate(topo.edges)}
        return gauged, lambdas

    return vidal_gauge_fixing_map


def vidal_distance_partial(layout: GraphLayout, G, lam, eps: float, partial=None, halves=None) -> torch.Tensor:
    """Per-half-edge trace norms (the terms of the Vidal distance) into
    ``partial`` (float64, one per half-edge; new when None). ``halves`` (int32
    device tensor) recomputes only those entries."""
    if partial is None:
        partial = torch.empty(max(layout.n_halves, 1), dtype=torch.float64, device=layout.device)
    _lib.call("dqz_vidal_distance", layout.gptr, G.data_ptr(), lam.data_ptr(), float(eps), partial.data_ptr(), None,
              layout.max_chi(), layout.max_slice(), _lib.ptr(halves), int(halves.numel()) if halves is not None else 0,
              _lib.stream_handle())
    return partial


def vidal_distance_packed(layout: GraphLayout, G, lam, eps: float) -> torch.Tensor:
    partial = torch.empty(max(layout.n_halves, 1), dtype=torch.float64, device=layout.device)
    out = torch.empty((), dtype=torch.float64, device=layout.device)
    _lib.call("dqz_vidal_distance", layout.gptr, G.data_ptr(), lam.data_ptr(), float(eps), partial.data_ptr(),
              out.data_ptr(), layout.max_chi(), layout.max_slice(), None, 0, _lib.stream_handle())
    return out


def get_vidal_gauge_distance_map(traverser, eps):
    topo = Topology(traverser, True)
    cache = _LayoutCache(topo)

    def vidal_gauge_distance(tensors: Dict, lambdas: Dict) -> torch.Tensor:
        dev_t = {n.id: as_device(tensors[n.id]) for n in topo.nodes}
        layout = cache.get(dev_t)
        G = layout.pack_tensors([dev_t[n.id] for n in topo.nodes])
        lam = layout.pack_lambdas([as_device_real(lambdas[e.id]) for e in topo.edges])
        return vidal_distance_packed(layout, G, lam, float(eps))

    return vidal_gauge_distance


def get_symmetric_gauge_fixing_map(traverser, eps):
    topo = Topology(traverser, True)
    cache = _LayoutCache(topo)

    def symmetric_gauge(tensors: Dict, lambdas: Dict) -> Dict:
        dev_t = {n.id: as_device(tensors[n.id]) for n in topo.nodes}
        layout = cache.get(dev_t)
        G = layout.pack_tensors([dev_t[n.id] for n in topo.nodes])
        lam = layout.pack_lambdas([as_device_real(lambdas[e.id]) for e in topo.edges])
        out = torch.empty_like(G)
        _lib.call("dqz_symmetric_gauge", layout.gptr, G.data_ptr(), lam.data_ptr(), float(eps), out.data_ptr(),
                  _lib.stream_handle())
        ts = layout.unpack_tensors(out)
        return {n.id: ts[i] for i, n in enumerate(topo.nodes)}

    return symmetric_gauge


def lambdas2messages(lambdas: Dict) -> Dict:
    """diag(lambda) in both directions of every edge."""
    messages = {}
    for edge_id, lmbd in lambdas.items():
        m = torch.diag(as_device_real(lmbd)).to(torch.complex128)
        for node_id in edge_id:
            messages[MessageID(src=edge_id, dst=node_id)] = m
            messages[MessageID(src=node_id, dst=edge_id)] = m
    return messages


def get_one_side_density_matrix(node: Node, tensors: Dict, messages: Dict) -> torch.Tensor:
    t = as_device(tensors[node.id])
    if t.dim() - 1 != node.degree:
        raise AssertionError(f"{node.degree}, {t.dim() - 1}")
    layout = GraphLayout([node], list(node.neighbors), list(t.shape[:-1]), phys=[t.shape[-1]])
    T = layout.pack_tensors([t])
    e2n = layout.pack_messages([as_device(messages[MessageID(e.id, node.id)]) for e in node.neighbors])
    return density_packed(layout, T, e2n, [0])[0]


def density_packed(layout: GraphLayout, T, e2n, nodes: List[int]) -> torch.Tensor:
    """rho for the listed node indices: tensor [len(nodes), d, d]."""
    dev = layout.device
    idx = torch.tensor(nodes, dtype=torch.int32, device=dev)
    mp = _lib.MAX_PHYS
    rho = torch.zeros((len(nodes), mp * mp), dtype=torch.complex128, device=dev)
    ms = layout.max_size()
    nb = _lib.lib().dqz_density_scratch_bytes(len(nodes), ms)
    scratch = _scratch(nb, dev) if nb else None
    _lib.call("dqz_density_matrices", layout.gptr, T.data_ptr(), e2n.data_ptr(), idx.data_ptr(), len(nodes),
              rho.data_ptr(), ms, _lib.ptr(scratch), _lib.stream_handle())
    d = int(layout.phys[nodes[0]]) if nodes else 2
    return rho[:, : d * d].reshape(len(nodes), d, d)
