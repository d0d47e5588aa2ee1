"""BPQuantumEmulator on the GPU (mirrors
dequantizer/src/quantum_emulator/bp_quantum_emulator.py:32-300).

The state stays packed on the device between calls: Gamma tensors in one
complex128 arena, lambdas in one float64 arena, laid out by a GraphLayout
with spare capacity so bonds can grow in place. Bond dimensions after a
simple update follow a host-computable rule (min(max_chi, rank bounds)), so
the host tracks every shape without reading the device.

Gates are queued and executed lazily. A flush groups the queue into levels
of node-disjoint operations (an operation's level is one past the last level
that touched either of its nodes), which preserves the per-node order of the
reference's sequential application exactly; each level is one apply1 launch
and one simple-update launch.
"""

import logging
import math
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib
from .gates import decompose_gates
from .graph import Edge, Node, TensorGraph
from .initializers import get_message_random_nonnegative_initializer
from .layout import GraphLayout
from .maps import Topology, bp_sweep, density_packed, vidal_distance_packed, vidal_gauge_packed
from .tensor_graph_ops import simple_update_shapes

log = logging.getLogger(__name__)

EPS = 1e-10  # bp_quantum_emulator.py:84-86, 161


class BPQuantumEmulator:
    def __init__(
        self,
        tensor_graph: TensorGraph,
        key: int,
        max_chi: int,
        gates_number_per_regauging: int,
        belief_propagation_accuracy: float = 1e-5,
        max_belief_propagation_iterations: Optional[int] = 100,
        synchronous_update: bool = False,
        traversal_type: str = "dfs",
    ):
        log.info(
            "BP emulator: seed %s max_chi %s gates_per_regauging %s accuracy %s synchronous %s traversal %s",
            key, max_chi, gates_number_per_regauging, belief_propagation_accuracy, synchronous_update,
            traversal_type,
        )
        if not torch.cuda.is_available():
            raise RuntimeError("BPQuantumEmulator runs on the GPU only and no CUDA device is available")
        _lib.lib()
        self.tensor_graph = tensor_graph
        self.prng_key = key
        self._rng = np.random.default_rng(key)
        self.max_chi = int(max_chi)
        self.per_regauging = gates_number_per_regauging
        self.accuracy = float(belief_propagation_accuracy)
        self.max_iters = max_belief_propagation_iterations
        self._topo = Topology(list(tensor_graph.get_traversal_iterator(ordering=traversal_type)),
                              synchronous_update)
        self._nodes: List[Node] = self._topo.nodes
        self._edges: List[Edge] = self._topo.edges
        self._node_idx = {n.id: i for i, n in enumerate(self._nodes)}
        self._passed = 0
        self._pending: List[tuple] = []
        # per-gate truncation errors / entropies, in chunks per executed level
        # with the gates' application order numbers
        self._err_chunks: List[torch.Tensor] = []
        self._ent_chunks: List[torch.Tensor] = []
        self._seq_chunks: List[torch.Tensor] = []
        self._q2_count = 0
        self._after_vd: List[torch.Tensor] = []
        self._trunc_vd: List[torch.Tensor] = []
        self.bp_iterations: List[int] = []
        self._rho_cache = None
        self._product_layout(lambda node: 0)
        self._set_to_vidal_canonical()

    # ------------------------------------------------------------ state
    def _product_layout(self, state_of):
        self.tensor_graph.to_product()
        chi = [1] * len(self._edges)
        self._layout = GraphLayout(self._nodes, self._edges, chi)
        parts = []
        for nd in self._nodes:
            t = torch.zeros(nd.dimension, dtype=torch.complex128)
            t[int(state_of(nd))] = 1.0
            parts.append(t)
        self._G = torch.cat(parts).to(self._layout.device)
        self._lam = torch.ones(max(len(self._edges), 1), dtype=torch.float64, device=self._layout.device)
        self._rho_cache = None

    def _grow(self, node_need: Dict[int, int], edge_need: Dict[int, int]):
        """Moves the state into a layout whose capacities cover the given needs."""
        L = self._layout
        ncap = L.node_capacity.copy()
        ecap = L.edge_capacity.copy()
        for v, s in node_need.items():
            if s > ncap[v]:
                ncap[v] = max(s, 2 * ncap[v])
        for e, c in edge_need.items():
            if c > ecap[e]:
                ecap[e] = max(c, 2 * ecap[e])
        if np.array_equal(ncap, L.node_capacity) and np.array_equal(ecap, L.edge_capacity):
            return
        full = self._full_capacities()
        if full is not None:  # take the final capacities at once: one arena move instead of one per growing gate
            ncap = np.maximum(ncap, full[0])
            ecap = np.maximum(ecap, full[1])
        # queued gates must run first: afterwards host and device bond
        # dimensions agree and the sizes below describe the data on the device
        self._flush()
        new = GraphLayout(self._nodes, self._edges, L.edge_chi.copy(), node_capacity=ncap, edge_capacity=ecap)
        G = new.new_tensor_arena()
        lam = new.new_lam_arena()
        dev = new.device
        stream = _lib.stream_handle()
        sizes = torch.from_numpy(L.node_sizes()).to(dev)
        _lib.call("dqz_repack", self._G.data_ptr(), G.data_ptr(), L.d_node_off.data_ptr(), new.d_node_off.data_ptr(),
                  sizes.data_ptr(), L.n_nodes, 16, stream)
        if L.n_edges:
            cnt = torch.from_numpy(L.edge_chi.astype(np.int64)).to(dev)
            _lib.call("dqz_repack", self._lam.data_ptr(), lam.data_ptr(), L.d_edge_lam_off.data_ptr(),
                      new.d_edge_lam_off.data_ptr(), cnt.data_ptr(), L.n_edges, 8, stream)
        self._layout, self._G, self._lam = new, G, lam

    # Node-tensor arena size (bytes) at every bond = max_chi below which a
    # growing state gets those capacities at the first growth.
    FULL_CAPACITY_BYTES = 2 << 30

    def _full_capacities(self):
        """(node, edge) capacities with every bond at max_chi, or None when
        that arena would exceed FULL_CAPACITY_BYTES (then capacities double
        per growing node instead)."""
        L = self._layout
        deg = L.degree.astype(np.float64)
        if 16.0 * float(np.sum(L.phys.astype(np.float64) * float(self.max_chi) ** deg)) > self.FULL_CAPACITY_BYTES:
            return None
        node = L.phys.astype(np.int64) * np.power(np.int64(self.max_chi), L.degree.astype(np.int64))
        return node, np.full(L.n_edges, self.max_chi, dtype=np.int64)

    # ------------------------------------------------------------- API
    @property
    def after_regauging_vidal_distances(self) -> torch.Tensor:
        return torch.stack(self._after_vd) if self._after_vd else torch.zeros(0, dtype=torch.float64)

    @property
    def truncated_affected_vidal_distances(self) -> torch.Tensor:
        return torch.stack(self._trunc_vd) if self._trunc_vd else torch.zeros(0, dtype=torch.float64)

    @property
    def truncation_errors(self) -> List[torch.Tensor]:
        self._flush()
        return list(self._ordered(self._err_chunks))

    @property
    def entropies(self) -> List[torch.Tensor]:
        self._flush()
        return list(self._ordered(self._ent_chunks))

    def _ordered(self, chunks) -> torch.Tensor:
        if not chunks:
            return torch.zeros(0, dtype=torch.float64)
        seq = torch.cat(self._seq_chunks)
        return torch.cat(chunks)[torch.argsort(seq)]

    def set_to_product_state(self, state: Dict):
        """bp_quantum_emulator.py:110-130."""
        self._pending.clear()
        self._product_layout(lambda node: state[node.id])
        self._set_to_vidal_canonical()
        self._passed = 0

    def apply_q2(self, gate, controlling_node_id, controlled_node_id):
        """bp_quantum_emulator.py:144-167 (queued; see module docstring)."""
        if self._passed >= self.per_regauging:
            self._vidal_regauging()
            self._passed = 0
        g = gate.detach().cpu().numpy() if isinstance(gate, torch.Tensor) else np.asarray(gate)
        flat, ranks, _ = decompose_gates(g[None], EPS)
        self._queue_q2(controlling_node_id, controlled_node_id, flat[0], int(ranks[0]))
        self._passed += 1

    def apply_q1(self, gate, node_id):
        """bp_quantum_emulator.py:175-180 (queued)."""
        g = gate if isinstance(gate, torch.Tensor) else torch.from_numpy(np.asarray(gate))
        self._queue_q1(node_id, g.to(torch.complex128))

    def dens_q1(self, node_id) -> torch.Tensor:
        """bp_quantum_emulator.py:188-207."""
        rho = self.all_densities()
        return rho[self._node_idx[node_id]]

    def all_densities(self) -> torch.Tensor:
        """One-site density matrices of all nodes (node order of the traversal)."""
        self._flush()
        if self._passed != 0:
            self._vidal_regauging()
            self._passed = 0
        if self._rho_cache is None:
            L = self._layout
            T = self._symmetric(self._G, self._lam)
            n2e, e2n = self._lambda_messages(self._lam)
            self._rho_cache = density_packed(L, T, e2n, list(range(L.n_nodes)))
        return self._rho_cache

    def measure(self, node_id, sample: Optional[float] = None) -> int:
        """bp_quantum_emulator.py:215-233. ``sample`` (a uniform draw) defaults
        to the emulator's own generator."""
        dens = self.dens_q1(node_id)
        if sample is None:
            sample = float(self._rng.uniform())
        p = float(dens[0, 0].real)
        result = 0 if p > sample else 1
        proj = torch.zeros((2, 2), dtype=torch.complex128)
        proj[result, result] = 1.0
        self.apply_q1(proj, node_id)
        self._flush()
        self._G = self._symmetric(self._G, self._lam)
        self._set_to_vidal_canonical()
        self._passed = 0
        return result

    # ------------------------------------------------------------ queue
    def _queue_q1(self, node_id, gate: torch.Tensor):
        v = self._node_idx[node_id]
        d = int(self._layout.phys[v])
        if tuple(gate.shape) != (d, d):
            raise ValueError(f"gate of shape {tuple(gate.shape)} does not act on a physical dimension {d}")
        self._pending.append(("q1", v, gate.reshape(-1)))
        self._rho_cache = None

    def _queue_q2(self, id1, id2, halves: np.ndarray, rank: int):
        graph = self.tensor_graph
        edge = graph.find_edge(id1, id2)
        if edge is None:
            raise ValueError(f"Neither edge with ID {(id2, id1)} nor with ID {(id1, id2)} is found in the tensor graph.")
        if edge.degree != 2:
            raise NotImplementedError("apply2 is implemented only for two qubits.")
        L = self._layout
        e = L.edge_index[edge.id]
        n1, n2 = graph.get_node(id1), graph.get_node(id2)
        v1, v2 = self._node_idx[id1], self._node_idx[id2]
        i1, i2 = n1.indices[edge.id], n2.indices[edge.id]
        d1, d2 = L.node_dims(v1), L.node_dims(v2)
        m1, m2, k, new_chi, _ = simple_update_shapes(d1, int(L.phys[v1]), i1, d2, int(L.phys[v2]), i2, rank,
                                                     self.max_chi)
        if k > _lib.MAX_CHI:
            raise NotImplementedError(f"bond dimension x gate rank = {k} above {_lib.MAX_CHI} is not supported")
        s1 = int(np.prod(d1)) * int(L.phys[v1]) // d1[i1] * new_chi
        s2 = int(np.prod(d2)) * int(L.phys[v2]) // d2[i2] * new_chi
        self._grow({v1: s1, v2: s2}, {e: new_chi})
        L = self._layout
        first = 1 if edge.neighbors[0] is n1 else 0
        self._pending.append(("q2", v1, v2, e, first, halves, rank, max(m1, m2), k, self._q2_count))
        self._q2_count += 1
        # host bookkeeping, as tensor_graph.py:366-374
        L.edge_chi[e] = new_chi
        edge.dimension = new_chi
        n1.bond_shape = tuple(L.node_dims(v1))
        n2.bond_shape = tuple(L.node_dims(v2))
        self._rho_cache = None

    def _flush(self):
        if not self._pending:
            return
        L = self._layout
        dev = L.device
        last = np.zeros(L.n_nodes, dtype=np.int64)
        levels: Dict[int, List[tuple]] = {}
        for op in self._pending:
            touched = (op[1],) if op[0] == "q1" else (op[1], op[2])
            lv = 1 + max(int(last[v]) for v in touched)
            for v in touched:
                last[v] = lv
            levels.setdefault(lv, []).append(op)
        self._pending = []
        stream = _lib.stream_handle()
        mp2 = _lib.MAX_PHYS * _lib.MAX_PHYS
        for lv in sorted(levels):
            ops = levels[lv]
            q1 = [op for op in ops if op[0] == "q1"]
            q2 = [op for op in ops if op[0] == "q2"]
            if q1:
                nodes = torch.tensor([op[1] for op in q1], dtype=torch.int32)
                gates = torch.zeros((len(q1), mp2), dtype=torch.complex128)
                for j, op in enumerate(q1):
                    gates[j, : op[2].numel()] = op[2].cpu()
                nodes, gates = nodes.to(dev), gates.to(dev)
                _lib.call("dqz_apply1", L.gptr, self._G.data_ptr(), nodes.data_ptr(), gates.data_ptr(), len(q1),
                          stream)
            if q2:
                n = len(q2)
                edges = torch.tensor([op[3] for op in q2], dtype=torch.int32).to(dev)
                first = torch.tensor([op[4] for op in q2], dtype=torch.uint8).to(dev)
                halves = torch.from_numpy(np.stack([op[5] for op in q2]).reshape(n, -1)).to(dev)
                ranks = torch.tensor([op[6] for op in q2], dtype=torch.int32).to(dev)
                rows = max(op[7] for op in q2)
                cols = max(op[8] for op in q2)
                err = torch.empty(n, dtype=torch.float64, device=dev)
                ent = torch.empty(n, dtype=torch.float64, device=dev)
                nb = _lib.lib().dqz_simple_update_scratch_bytes(n, rows, cols)
                scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
                _lib.call("dqz_simple_update", L.gptr, self._G.data_ptr(), self._lam.data_ptr(), edges.data_ptr(),
                          first.data_ptr(), halves.data_ptr(), ranks.data_ptr(), n, EPS, self.max_chi, rows, cols,
                          err.data_ptr(), ent.data_ptr(), scratch.data_ptr(), stream)
                self._err_chunks.append(err)
                self._ent_chunks.append(ent)
                self._seq_chunks.append(torch.tensor([op[9] for op in q2], dtype=torch.int64, device=dev))
        self._rho_cache = None

    # ---------------------------------------------------------- regauge
    def _symmetric(self, G, lam):
        L = self._layout
        out = torch.empty_like(G)
        _lib.call("dqz_symmetric_gauge", L.gptr, G.data_ptr(), lam.data_ptr(), EPS, out.data_ptr(),
                  _lib.stream_handle())
        return out

    def _lambda_messages(self, lam):
        L = self._layout
        n2e, e2n = L.new_msg_arena(), L.new_msg_arena()
        _lib.call("dqz_lambdas_to_messages", L.gptr, lam.data_ptr(), n2e.data_ptr(), e2n.data_ptr(), L.max_chi(),
                  _lib.stream_handle())
        return n2e, e2n

    def _random_messages(self):
        L = self._layout
        init = get_message_random_nonnegative_initializer(int(self._rng.integers(0, 2**31 - 1)))
        mats = {}
        by_half = []
        for h in range(L.n_halves):
            c = int(L.edge_chi[L.half_edge[h]])
            if c not in mats:
                nd = L.nodes[L.half_node[h]]
                e = L.edges[L.half_edge[h]]
                mats[c] = torch.from_numpy(init((nd, e)))
            by_half.append(mats[c])
        n2e = L.pack_messages([m.to(L.device) for m in by_half]) if L.exact() else self._pack_msgs(by_half)
        e2n = n2e.clone()
        return n2e, e2n

    def _pack_msgs(self, by_half):
        L = self._layout
        arena = torch.zeros(max(L.msg_elems, 1), dtype=torch.complex128)
        for h, m in enumerate(by_half):
            o = int(L.half_msg_off[h])
            arena[o : o + m.numel()] = m.reshape(-1)
        return arena.to(L.device)

    def _bp_loop(self, T, n2e, e2n, vd, G, lam):
        L = self._layout
        iters = 0
        while True:
            d = float(vd)
            if not math.isfinite(d):
                # the reference's loop stops here too (NaN > accuracy is false) but
                # keeps the NaN state silently; this one reports it
                raise _lib.NonFiniteError(f"BP regauge iteration {iters}: Vidal distance {d}")
            if d <= self.accuracy:
                break
            if self.max_iters is not None and self.max_iters <= iters:
                log.warning("Belief propagation reached the maximal number of iterations.")
                break
            n2e_new, e2n_new = torch.empty_like(n2e), torch.empty_like(e2n)
            bp_sweep(L, self._topo, T, n2e, e2n, n2e_new, e2n_new)
            n2e, e2n = n2e_new, e2n_new
            G, lam = vidal_gauge_packed(L, T, n2e, EPS)
            vd = vidal_distance_packed(L, G, lam, EPS)
            iters += 1
        self.bp_iterations.append(iters)
        return G, lam, vd

    def _set_to_vidal_canonical(self):
        """bp_quantum_emulator.py:245-270."""
        self._flush()
        n2e, e2n = self._random_messages()
        inf = torch.tensor(np.finfo(np.float64).max, dtype=torch.float64)
        G, lam, vd = self._bp_loop(self._G, n2e, e2n, inf, self._G, self._lam)
        self._after_vd.append(vd.reshape(()))
        self._G, self._lam = G, lam
        self._rho_cache = None

    def _vidal_regauging(self):
        """bp_quantum_emulator.py:272-300."""
        self._flush()
        T = self._symmetric(self._G, self._lam)
        n2e, e2n = self._lambda_messages(self._lam)
        G, lam = vidal_gauge_packed(self._layout, T, n2e, EPS)
        vd = vidal_distance_packed(self._layout, G, lam, EPS)
        self._trunc_vd.append(vd)
        G, lam, vd = self._bp_loop(T, n2e, e2n, vd, G, lam)
        self._after_vd.append(vd)
        self._G, self._lam = G, lam
        self._rho_cache = None

    # ---------------------------------------------------------- export
    def tensors(self) -> Dict:
        """Current Gamma tensors as a dict of device views."""
        self._flush()
        ts = self._layout.unpack_tensors(self._G)
        return {n.id: ts[i] for i, n in enumerate(self._nodes)}

    def lambdas(self) -> Dict:
        self._flush()
        return {e.id: self._layout.lambda_view(self._lam, i) for i, e in enumerate(self._edges)}
