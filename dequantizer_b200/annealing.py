"""Batched quantum annealing: many independent instances advanced together.

Each instance follows the reference's annealing loop
(examples/quantum_annealing/quantum_annealing/src/quantum_annealer.py:90-152,
with one regauge per layer as qbp.py:94-106 sets it) on the BP emulator's
operations (bp_quantum_emulator.py:144-300). All instances live in one
packed layout (a disjoint union, instance after instance), so every
operation is one launch over all of them:

* a layer's two-site gates: built and SVD-split for all instances at once,
  applied by simple-update launches over node-disjoint levels (the levels
  follow each instance's edge order, which never changes, so they are
  computed once);
* the mixing layer: one apply1 launch over every node;
* the regauge: symmetric gauge, lambda messages, Vidal gauge and per-instance
  Vidal distances (a segmented sum of the per-half-edge kernel outputs);
  BP sweeps then run only on the instances whose distance is still above the
  accuracy, the others keep their messages, so every instance stops where an
  independent run would (synchronous and flooding schedules).

Bond dimensions after every simple update follow the host rule
min(max_chi, rank bounds), evaluated for a whole level with numpy.
"""

import logging
import math
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .gates import DIAG_FLAT_POS, HALF_SLOTS, decompose_diagonal_gates
from .graph import Edge, Node, TensorGraph
from .initializers import get_message_random_nonnegative_initializer
from .layout import GraphLayout
from .maps import Topology, density_packed, error_flag, vidal_distance_partial, vidal_gauge_packed
from .workloads import HADAMARD, EnergyFunction, q1_gate

log = logging.getLogger(__name__)

EPS = 1e-10


class BatchedAnnealer:
    def __init__(
        self,
        energies: Sequence[EnergyFunction],
        max_chi: int,
        accuracy: float = 1e-5,
        max_belief_propagation_iterations: Optional[int] = 100,
        schedule: str = "sync",
        key: int = 0,
        autotune: bool = False,
        precision: str = "fp64",
        bf16_handover: float = 2e-4,
        bf16_max_sweeps: int = 40,
        fp32_handover: float = 1e-7,
        fp32_max_sweeps: int = 60,
    ):
        """``autotune``: time the gauge kernels' launch shapes on the first
        regauge of every new maximal bond dimension (``autotune.tune_gauge``,
        cached on disk) and use the fastest.

        ``precision="mixed"``: once every bond has dimension 16, each regauge
        first runs BF16 tensor-core sweeps (dqz_bp_node_update_k3_umma, FP32
        accumulation, complex64 messages) on the instances above the accuracy,
        with no gauge or distance evaluation, until an instance's mean change of
        its node->edge messages per sweep falls to ``bf16_handover`` (at most
        ``bf16_max_sweeps``), then FP32 sweeps (dqz_bp_node_update_k3,
        complex64) until it falls to ``fp32_handover`` (at most
        ``fp32_max_sweeps``; BF16 products settle near 5e-5, FP32 ones near
        1e-7); FP64 sweeps then finish from there to the reference's stopping
        rule (Vidal distance at most the accuracy, FP64 gauge and distance),
        but the gauge and distance are evaluated after the first two sweeps
        and then only when the geometric rate of the last two evaluations
        predicts the accuracy (at most 8 sweeps apart), not after every sweep:
        an instance stops at or a few sweeps past the reference's stopping
        point. Eigen and singular value decompositions, the distances and the
        gates stay FP64. ``precision="fp64"`` is the plain form (the
        reference's loop exactly)."""
        if schedule not in ("sync", "flooding"):
            raise ValueError("batched annealing runs the synchronous or flooding BP schedule")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.bf16_handover = float(bf16_handover)
        self.bf16_max_sweeps = int(bf16_max_sweeps)
        self.fp32_handover = float(fp32_handover)
        self.fp32_max_sweeps = int(fp32_max_sweeps)
        self.bf16_sweeps: List[List[int]] = []
        self.fp32_sweeps: List[List[int]] = []
        self.vd_checks: List[List[int]] = []
        # per instance, from its previous regauge in the mixed form: FP64 sweeps
        # to the accuracy and the distance's geometric rate per sweep there
        self._prev_iters: Optional[np.ndarray] = None
        self._prev_rate: Optional[np.ndarray] = None
        if not torch.cuda.is_available():
            raise RuntimeError("BatchedAnnealer runs on the GPU only")
        _lib.lib()
        self.energies = list(energies)
        self.max_chi = int(max_chi)
        self.accuracy = float(accuracy)
        self.max_iters = max_belief_propagation_iterations
        self._rng = np.random.default_rng(key)
        self.autotune = bool(autotune)
        self._tuned_chi = set()
        # ---- union graph, traversal = concatenated per-instance DFS traversals
        self.graph = TensorGraph()
        trav: List = []
        self.node_start, self.edge_start = [0], [0]
        for k, en in enumerate(self.energies):
            n = en.fields.shape[0]
            for i in range(n):
                self.graph.add_node(2, (k, i))
            for a, b in en.coupled_spin_pairs:
                self.graph.add_edge(((k, int(a)), (k, int(b))), 1)
            first = self.graph.get_node((k, 0))
            trav.extend(self.graph.get_traversal_iterator(first, "dfs"))
            self.node_start.append(self.node_start[-1] + n)
            self.edge_start.append(self.edge_start[-1] + en.edges_number)
        self.topo = Topology(trav, schedule == "sync", flooding=schedule == "flooding")
        self.n_inst = len(self.energies)
        nodes, edges = self.topo.nodes, self.topo.edges
        self.node_idx = {n.id: i for i, n in enumerate(nodes)}
        self.edge_idx = {e.id: i for i, e in enumerate(edges)}
        # per-instance node / half-edge / edge ranges in the layout
        self.inst_of_node = np.array([n.id[0] for n in nodes], dtype=np.int64)
        deg = np.array([len(n.neighbors) for n in nodes])
        maxdeg = int(deg.max())
        cap = 2 * np.array([min(self.max_chi, 2 ** 30) ** d for d in deg], dtype=np.int64)
        self.layout = GraphLayout(nodes, edges, [1] * len(edges), node_capacity=cap,
                                  edge_capacity=[self.max_chi] * len(edges))
        L = self.layout
        self.inst_of_half = self.inst_of_node[L.half_node]
        self.inst_of_edge = np.array([e.id[0][0] for e in edges], dtype=np.int64)
        # nodes, half-edges and edges are numbered instance after instance
        if np.any(np.diff(self.inst_of_node) < 0) or np.any(np.diff(self.inst_of_edge) < 0):
            raise RuntimeError("union layout is not grouped by instance")
        ks = np.arange(self.n_inst)
        self.node_bounds = np.stack([np.searchsorted(self.inst_of_node, ks), np.searchsorted(self.inst_of_node, ks, "right")], 1)
        self.half_bounds = np.stack([np.searchsorted(self.inst_of_half, ks), np.searchsorted(self.inst_of_half, ks, "right")], 1)
        self.edge_bounds = np.stack([np.searchsorted(self.inst_of_edge, ks), np.searchsorted(self.inst_of_edge, ks, "right")], 1)
        self.half_range = [tuple(int(x) for x in b) for b in self.half_bounds]
        # node -> its edges (padded) for the vectorised shape rule
        self.node_edges = -np.ones((L.n_nodes, maxdeg), dtype=np.int64)
        for v in range(L.n_nodes):
            h0 = L.node_half[v]
            self.node_edges[v, : deg[v]] = L.half_edge[h0 : h0 + deg[v]]
        self.node_deg = deg
        # gate order (per instance, pair order) and node-disjoint levels
        self.gate_edge, self.gate_u, self.gate_v, self.gate_first = [], [], [], []
        for k, en in enumerate(self.energies):
            for a, b in en.coupled_spin_pairs:
                u, v = (k, int(a)), (k, int(b))
                e = self.graph.find_edge(u, v)
                self.gate_edge.append(self.edge_idx[e.id])
                self.gate_u.append(self.node_idx[u])
                self.gate_v.append(self.node_idx[v])
                self.gate_first.append(1 if e.neighbors[0].id == u else 0)
        self.gate_edge = np.array(self.gate_edge)
        self.gate_u = np.array(self.gate_u)
        self.gate_v = np.array(self.gate_v)
        self.gate_first = np.array(self.gate_first, dtype=np.uint8)
        last = np.zeros(L.n_nodes, dtype=np.int64)
        lvl = np.zeros(len(self.gate_edge), dtype=np.int64)
        for j in range(len(self.gate_edge)):
            u, v = self.gate_u[j], self.gate_v[j]
            lvl[j] = max(last[u], last[v]) + 1
            last[u] = last[v] = lvl[j]
        self.gate_levels = [np.nonzero(lvl == l)[0] for l in range(1, int(lvl.max()) + 1)]
        # gates are stored level after level on the device, so a level's
        # halves, ranks, edges and outputs are contiguous slices
        self.level_perm = np.concatenate(self.gate_levels) if self.gate_levels else np.zeros(0, np.int64)
        self.level_bounds = np.cumsum([0] + [len(ix) for ix in self.gate_levels])
        dev = L.device
        self.gate_edge_dev = torch.from_numpy(self.gate_edge[self.level_perm].astype(np.int32)).to(dev)
        self.gate_first_dev = torch.from_numpy(self.gate_first[self.level_perm]).to(dev)
        fields = np.array([
            [self.energies[self.topo.nodes[u].id[0]].fields[self.topo.nodes[u].id[1]] / self.node_deg[u],
             self.energies[self.topo.nodes[v].id[0]].fields[self.topo.nodes[v].id[1]] / self.node_deg[v]]
            for u, v in zip(self.gate_u, self.gate_v)]).reshape(-1, 2)
        J = np.concatenate([en.coupling_amplitudes for en in self.energies])
        # Hamiltonian diagonal J s1 s2 + h1/deg1 s1 + h2/deg2 s2 over (s1, s2) in
        # {+1, -1}^2, row-major, per gate in level order
        s1 = np.array([1.0, 1.0, -1.0, -1.0])
        s2 = np.array([1.0, -1.0, 1.0, -1.0])
        ham = J[:, None] * s1 * s2 + fields[:, :1] * s1 + fields[:, 1:] * s2
        self.gate_ham_dev = torch.from_numpy(ham[self.level_perm]).to(dev)
        mp = _lib.MAX_PHYS
        self.halves_dev = torch.zeros((len(self.level_perm), 2, HALF_SLOTS * mp * mp), dtype=torch.complex128,
                                      device=dev)
        self.diag_pos_dev = torch.from_numpy(DIAG_FLAT_POS).to(dev)
        self.all_nodes_dev = torch.arange(L.n_nodes, dtype=torch.int32, device=dev)
        self.inst_id_half = torch.from_numpy(self.inst_of_half).to(L.device)
        self.edges_per_inst = torch.tensor([en.edges_number for en in self.energies], dtype=torch.float64,
                                           device=L.device)
        self.bp_iterations: List[List[int]] = []
        self.vidal_distances: List[np.ndarray] = []
        self.truncation_affected_vd: List[torch.Tensor] = []
        self._err = []  # (layer, gate indices, errors, entropies) per launch
        self._layers = 0
        # ---- product |0>, canonicalise, Hadamards
        self.G = torch.zeros(L.tensor_elems, dtype=torch.complex128, device=L.device)
        self.G[torch.from_numpy(L.node_off).to(L.device)] = 1.0
        self.lam = L.new_lam_arena()
        self.lam[torch.from_numpy(L.edge_lam_off).to(L.device)] = 1.0
        self._canonicalize_from_random()
        self._apply1_all(HADAMARD)

    # ------------------------------------------------------------ helpers
    def _apply1_all(self, gate: np.ndarray):
        L = self.layout
        mp = _lib.MAX_PHYS
        g = torch.zeros((L.n_nodes, mp * mp), dtype=torch.complex128, device=L.device)
        g[:, :4] = torch.from_numpy(np.asarray(gate, dtype=np.complex128).reshape(-1)).to(L.device)
        _lib.call("dqz_apply1", L.gptr, self.G.data_ptr(), self.all_nodes_dev.data_ptr(), g.data_ptr(), L.n_nodes,
                  _lib.stream_handle())

    def _per_instance_vd(self, partial) -> torch.Tensor:
        """Vidal distance of every instance: the mean of its half-edge terms
        (mappings/vidal_distance.py:38-42 per instance)."""
        sums = torch.zeros(self.n_inst, dtype=torch.float64, device=self.layout.device)
        sums.index_add_(0, self.inst_id_half, partial[: self.layout.n_halves])
        return sums / (2.0 * self.edges_per_inst)

    @staticmethod
    def _ranges(bounds: np.ndarray, which: np.ndarray) -> np.ndarray:
        """Concatenation of the index ranges bounds[k] for the selected k."""
        b = bounds[which]
        n = b[:, 1] - b[:, 0]
        total = int(n.sum())
        if total == 0:
            return np.zeros(0, dtype=np.int32)
        shift = np.repeat(b[:, 0] - np.concatenate([[0], np.cumsum(n)[:-1]]), n)
        return (np.arange(total, dtype=np.int64) + shift).astype(np.int32)

    def _bp_loop(self, T, n2e, e2n, vd, G=None, lam=None, orth=None, partial=None):
        """Per-instance BP-to-accuracy loop (bp_quantum_emulator.py:253-266 /
        283-296 for every instance): each pass sweeps, gauges and measures
        only the instances whose distance is still above the accuracy; the
        others keep their messages, Gamma, lambda and distance terms, so they
        come out bit for bit as after their last sweep."""
        L = self.layout
        dev = L.device
        if G is None:
            G = torch.empty_like(T)
            lam = L.new_lam_arena()
            orth = torch.empty(max(L.msg_elems, 1), dtype=torch.complex128, device=dev)
            partial = torch.zeros(max(L.n_halves, 1), dtype=torch.float64, device=dev)
        iters = np.zeros(self.n_inst, dtype=np.int64)
        vd_h = vd.cpu().numpy()
        if self.precision == "mixed" and L.uniform_k3_chi() == 16:
            todo = vd_h > self.accuracy
            if self.max_iters is not None:
                todo &= self.max_iters > 0
            if todo.any():
                n2e, e2n = self._bf16_prephase(T, n2e, e2n, todo)
        lazy = self.precision == "mixed"
        next_check = np.ones(self.n_inst, dtype=np.int64)
        if lazy and self._prev_iters is not None:
            # first check two sweeps before where the previous regauge got there
            next_check = np.maximum(1, self._prev_iters - 2)
        hist: List[List] = [[] for _ in range(self.n_inst)]
        checks = np.zeros(self.n_inst, dtype=np.int64)
        while True:
            active = vd_h > self.accuracy
            if self.max_iters is not None:
                capped = active & (iters >= self.max_iters)
                if capped.any():
                    log.warning("Belief propagation reached the maximal number of iterations.")
                active &= iters < self.max_iters
            if not active.any():
                break
            halves = torch.from_numpy(self._ranges(self.half_bounds, active)).to(dev)
            n2e_new, e2n_new = n2e.clone(), torch.empty_like(e2n)
            self._sweep_halves(T, n2e, e2n, n2e_new, e2n_new, halves)
            n2e, e2n = n2e_new, e2n_new
            iters += active
            # the Vidal gauge and distance: after every sweep (the reference's
            # loop), or in the mixed form when the instance's distance is
            # predicted to reach the accuracy (or at the iteration cap)
            due = active & (iters >= next_check) if lazy else active
            if lazy and self.max_iters is not None:
                due |= active & (iters >= self.max_iters)
            if not due.any():
                continue
            every = bool(due.all())
            halves = torch.from_numpy(self._ranges(self.half_bounds, due)).to(dev)
            edges = None if every else torch.from_numpy(self._ranges(self.edge_bounds, due)).to(dev)
            nodes = None if every else torch.from_numpy(self._ranges(self.node_bounds, due)).to(dev)
            vidal_gauge_packed(L, T, n2e, EPS, out=(G, lam, orth), edges=edges, nodes=nodes)
            vidal_distance_partial(L, G, lam, EPS, partial, halves=None if every else halves)
            vd_h = self._per_instance_vd(partial).cpu().numpy()
            checks += due
            if lazy:
                for k in np.nonzero(due)[0]:
                    hist[k].append((int(iters[k]), float(vd_h[k])))
                    prev = float(self._prev_rate[k]) if self._prev_rate is not None else float("nan")
                    next_check[k] = iters[k] + self._sweeps_to_accuracy(hist[k], prev)
        if lazy:
            rate = np.full(self.n_inst, np.nan) if self._prev_rate is None else self._prev_rate.copy()
            for k in range(self.n_inst):
                if len(hist[k]) >= 2:
                    (i1, v1), (i2, v2) = hist[k][-2], hist[k][-1]
                    if 0.0 < v2 < v1 and i2 > i1:
                        rate[k] = (v2 / v1) ** (1.0 / (i2 - i1))
            self._prev_rate = rate
            self._prev_iters = np.where(iters > 0, iters, self._prev_iters if self._prev_iters is not None else 0)
        self.bp_iterations.append(iters.tolist())
        self.vd_checks.append(checks.tolist())
        self.vidal_distances.append(vd_h.copy())
        return G, lam

    def _sweeps_to_accuracy(self, hist, prev_rate: float = float("nan"), max_gap: int = 8) -> int:
        """FP64 sweeps until the next distance check of the mixed form: the
        geometric rate of the last two checks extrapolated to the accuracy (at
        most ``max_gap``); after a single check, the rate the instance had at
        its previous regauge (``prev_rate``, at most ``max_gap // 2``); 1 when
        neither is known or the distance does not decrease."""
        if len(hist) == 1:
            v1 = hist[0][1]
            if not (0.0 < prev_rate < 1.0) or not (v1 > self.accuracy):
                return 1
            k = math.ceil(math.log(self.accuracy / v1) / math.log(prev_rate))
            return int(min(max(k, 1), max_gap // 2))
        if len(hist) < 2:
            return 1
        (i1, v1), (i2, v2) = hist[-2], hist[-1]
        if not (0.0 < v2 < v1) or i2 <= i1 or v2 <= self.accuracy:
            return 1
        rate = (v2 / v1) ** (1.0 / (i2 - i1))
        k = math.ceil(math.log(self.accuracy / v2) / math.log(rate))
        return int(min(max(k, 1), max_gap))

    def _bf16_prephase(self, T, n2e, e2n, active: np.ndarray):
        """Low-precision sweeps of the listed instances (complex64 messages),
        no gauge or distance evaluation: BF16 tensor-core sweeps until each
        one's mean node->edge message change per sweep is at most
        ``bf16_handover``, then FP32 sweeps until it is at most
        ``fp32_handover``; returns complex128 message arenas for the FP64 loop.
        Instances not listed keep their messages."""
        L = self.layout
        dev = L.device
        stream = _lib.stream_handle()
        src_sel, edge_new, _ = self.topo.device_tables(dev)
        per_node = int(_lib.lib().dqz_bf16_umma_elems_per_node())
        if getattr(self, "_T_bf16", None) is None or self._T_bf16.numel() != L.n_nodes * per_node:
            self._T_bf16 = torch.empty(L.n_nodes * per_node, dtype=torch.bfloat16, device=dev)
            self._halves_per_inst = torch.from_numpy(
                (self.half_bounds[:, 1] - self.half_bounds[:, 0]).astype(np.float64)).to(dev)
        T32 = T.to(torch.complex64)
        _lib.call("dqz_pack_bf16_umma", L.gptr, T32.data_ptr(), self._T_bf16.data_ptr(), stream)
        a, b = n2e.to(torch.complex64), e2n.to(torch.complex64)
        flag = error_flag(dev)
        change = torch.empty(max(L.n_halves, 1), dtype=torch.float64, device=dev)

        def stage(active, handover, max_sweeps, update):
            nonlocal a, b
            sweeps = np.zeros(self.n_inst, dtype=np.int64)
            for _ in range(max_sweeps):
                if not active.any():
                    break
                a_new, b_new = a.clone(), torch.empty_like(b)
                update(active, a, b, a_new)
                _lib.call("dqz_bp_edge_pass_c64", L.gptr, a.data_ptr(), a_new.data_ptr(), edge_new.data_ptr(),
                          b_new.data_ptr(), stream)
                _lib.call("dqz_message_changes_c64", L.gptr, a_new.data_ptr(), a.data_ptr(), change.data_ptr(),
                          stream)
                sums = torch.zeros(self.n_inst, dtype=torch.float64, device=dev)
                sums.index_add_(0, self.inst_id_half, change[: L.n_halves])
                mean_change = (sums / self._halves_per_inst).cpu().numpy()
                a, b = a_new, b_new
                sweeps += active
                active = active & (mean_change > handover)
            return sweeps

        def bf16_update(active, a, b, a_new):
            nodes = torch.from_numpy(self._ranges(self.node_bounds, active)).to(dev)
            _lib.call("dqz_bp_node_update_k3_umma", L.gptr, self._T_bf16.data_ptr(), a.data_ptr(), b.data_ptr(),
                      a_new.data_ptr(), src_sel.data_ptr(), nodes.data_ptr(), nodes.numel(), flag.data_ptr(), stream)

        def fp32_update(active, a, b, a_new):
            halves = torch.from_numpy(self._ranges(self.half_bounds, active)).to(dev)
            _lib.call("dqz_bp_node_update_k3", L.gptr, 16, 32, T32.data_ptr(), a.data_ptr(), b.data_ptr(),
                      a_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), halves.numel(), flag.data_ptr(),
                      stream)

        self.bf16_sweeps.append(stage(active.copy(), self.bf16_handover, self.bf16_max_sweeps, bf16_update).tolist())
        self.fp32_sweeps.append(stage(active.copy(), self.fp32_handover, self.fp32_max_sweeps, fp32_update).tolist())
        return a.to(torch.complex128), b.to(torch.complex128)

    def _sweep_halves(self, T, n2e, e2n, n2e_new, e2n_new, halves):
        """One synchronous / flooding sweep on the listed half-edges (n2e_new
        holds the old messages elsewhere), then the edge pass."""
        L = self.layout
        src_sel, edge_new, _ = self.topo.device_tables(L.device)
        stream = _lib.stream_handle()
        n = int(halves.numel())
        max_slice, max_chi = L.max_slice(), L.max_chi()
        chi3 = L.uniform_k3_chi()
        if chi3:
            _lib.call("dqz_bp_node_update_k3", L.gptr, chi3, 64, T.data_ptr(), n2e.data_ptr(), e2n.data_ptr(),
                      n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), n,
                      error_flag(L.device).data_ptr(), stream)
        else:
            nb = _lib.lib().dqz_bp_node_scratch_bytes(n, max_slice, max_chi)
            scratch = torch.empty(nb, dtype=torch.uint8, device=L.device) if nb else None
            _lib.call("dqz_bp_node_update", L.gptr, T.data_ptr(), n2e.data_ptr(), e2n.data_ptr(),
                      n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), n, max_slice, max_chi,
                      _lib.ptr(scratch), stream)
        _lib.call("dqz_bp_edge_pass", L.gptr, n2e.data_ptr(), n2e_new.data_ptr(), edge_new.data_ptr(),
                  e2n_new.data_ptr(), max_chi, stream)

    def _random_messages(self):
        L = self.layout
        init = get_message_random_nonnegative_initializer(int(self._rng.integers(0, 2**31 - 1)))
        arena = torch.zeros(max(L.msg_elems, 1), dtype=torch.complex128)
        cache = {}
        for h in range(L.n_halves):
            c = int(L.edge_chi[L.half_edge[h]])
            if c not in cache:
                cache[c] = torch.from_numpy(init((L.nodes[L.half_node[h]], L.edges[L.half_edge[h]]))).reshape(-1)
            o = int(L.half_msg_off[h])
            arena[o : o + c * c] = cache[c]
        arena = arena.to(L.device)
        return arena, arena.clone()

    def _canonicalize_from_random(self):
        """bp_quantum_emulator.py:245-270 for every instance."""
        n2e, e2n = self._random_messages()
        inf = torch.full((self.n_inst,), np.finfo(np.float64).max, dtype=torch.float64, device=self.layout.device)
        self.G, self.lam = self._bp_loop(self.G, n2e, e2n, inf)

    def regauge(self):
        """bp_quantum_emulator.py:272-300 for every instance."""
        L = self.layout
        T = torch.empty_like(self.G)
        _lib.call("dqz_symmetric_gauge", L.gptr, self.G.data_ptr(), self.lam.data_ptr(), EPS, T.data_ptr(),
                  _lib.stream_handle())
        n2e, e2n = L.new_msg_arena(), L.new_msg_arena()
        _lib.call("dqz_lambdas_to_messages", L.gptr, self.lam.data_ptr(), n2e.data_ptr(), e2n.data_ptr(),
                  L.max_chi(), _lib.stream_handle())
        if self.autotune and L.max_chi() not in self._tuned_chi:
            from .autotune import tune_gauge

            tune_gauge(L, T, n2e, EPS)
            self._tuned_chi.add(L.max_chi())
        G = torch.empty_like(T)
        lam = L.new_lam_arena()
        orth = torch.empty(max(L.msg_elems, 1), dtype=torch.complex128, device=L.device)
        vidal_gauge_packed(L, T, n2e, EPS, out=(G, lam, orth))
        partial = vidal_distance_partial(L, G, lam, EPS)
        vd = self._per_instance_vd(partial)
        self.truncation_affected_vd.append(vd)
        self.G, self.lam = self._bp_loop(T, n2e, e2n, vd, G, lam, orth, partial)

    # --------------------------------------------------------------- gates
    def _new_chi(self, jobs: np.ndarray, ranks: np.ndarray):
        """Shape rule of tensor_ops.py:318-389 for a level of node-disjoint gates."""
        L = self.layout
        e = self.gate_edge[jobs]
        chi_e = L.edge_chi[e].astype(np.int64)

        def rows(nodes):
            ne = self.node_edges[nodes]
            dims = np.where(ne >= 0, L.edge_chi[np.maximum(ne, 0)], 1).astype(np.int64)
            return 2 * dims.prod(axis=1) // chi_e

        m1, m2 = rows(self.gate_u[jobs]), rows(self.gate_v[jobs])
        k = chi_e * ranks
        new = np.minimum(np.minimum(np.minimum(m1, k), np.minimum(m2, k)), self.max_chi)
        return new, m1, m2, k

    def apply_coupling_layer(self, tau: float):
        """All two-site gates exp(-i tau (J ZZ + h_u/deg_u Z + h_v/deg_v Z)) in
        each instance's pair order (quantum_annealer.py:44-69, 123-124). The
        gates are diagonal: they are built and split on the device in closed
        form, and only the ranks come back to the host (for the shape rule)."""
        L = self.layout
        dev = L.device
        stream = _lib.stream_handle()
        n_all = len(self.level_perm)
        if n_all == 0:
            self._layers += 1
            return
        diag = torch.exp(-1j * tau * self.gate_ham_dev)
        compact, ranks_dev = decompose_diagonal_gates(diag, EPS)
        self.halves_dev[:, :, self.diag_pos_dev] = compact
        ranks = ranks_dev.cpu().numpy()
        err = torch.empty(n_all, dtype=torch.float64, device=dev)
        ent = torch.empty(n_all, dtype=torch.float64, device=dev)
        for li, jobs in enumerate(self.gate_levels):
            b0, b1 = int(self.level_bounds[li]), int(self.level_bounds[li + 1])
            new, m1, m2, k = self._new_chi(jobs, ranks[b0:b1])
            rows, cols = int(max(m1.max(), m2.max())), int(k.max())
            if cols > _lib.MAX_CHI:
                raise NotImplementedError(f"bond x gate rank {cols} above {_lib.MAX_CHI}")
            n = b1 - b0
            nb = _lib.lib().dqz_simple_update_scratch_bytes(n, rows, cols)
            scratch = torch.empty(nb, dtype=torch.uint8, device=dev)
            _lib.call("dqz_simple_update", L.gptr, self.G.data_ptr(), self.lam.data_ptr(),
                      self.gate_edge_dev[b0:].data_ptr(), self.gate_first_dev[b0:].data_ptr(),
                      self.halves_dev[b0:].data_ptr(), ranks_dev[b0:].data_ptr(), n, EPS, self.max_chi, rows, cols,
                      err[b0:].data_ptr(), ent[b0:].data_ptr(), scratch.data_ptr(), stream)
            L.edge_chi[self.gate_edge[jobs]] = new
        self._err.append((self._layers, self.level_perm, err, ent))
        self._layers += 1

    def step(self, mixing_time: float, coupling_time: float, first: bool, second_order: bool = False):
        """One Trotter step of every instance: regauge (after the first
        step), coupling gates, mixing gates (first order), or half mixing,
        coupling, half mixing (second order)."""
        if not first:
            self.regauge()
        if second_order:
            self._apply1_all(q1_gate(mixing_time / 2))
        self.apply_coupling_layer(coupling_time)
        self._apply1_all(q1_gate(mixing_time / 2 if second_order else mixing_time))

    def run(self, schedule_iter, second_order: bool = False):
        for t, (mix, coup) in enumerate(schedule_iter):
            self.step(mix, coup, first=(t == 0), second_order=second_order)
        self.regauge()
        return self.densities()

    def densities(self) -> List[np.ndarray]:
        """One-site density matrices per instance (node order of the instance)."""
        L = self.layout
        T = torch.empty_like(self.G)
        _lib.call("dqz_symmetric_gauge", L.gptr, self.G.data_ptr(), self.lam.data_ptr(), EPS, T.data_ptr(),
                  _lib.stream_handle())
        n2e, e2n = L.new_msg_arena(), L.new_msg_arena()
        _lib.call("dqz_lambdas_to_messages", L.gptr, self.lam.data_ptr(), n2e.data_ptr(), e2n.data_ptr(),
                  L.max_chi(), _lib.stream_handle())
        rho = density_packed(L, T, e2n, list(range(L.n_nodes))).cpu().numpy()
        out = []
        for k, en in enumerate(self.energies):
            idx = [self.node_idx[(k, i)] for i in range(en.fields.shape[0])]
            out.append(rho[idx])
        return out

    def sample_measurements(self, samples: Optional[np.ndarray] = None, seed: int = 0) -> List[np.ndarray]:
        """Measures every qubit of every instance in node order
        (quantum_annealer.py:137-141 with bp_quantum_emulator.py:215-233):
        round i measures node i of every instance that has one, all at once --
        densities, outcome 0 when rho_00 > u, projector applied (apply1,
        normalised), symmetric gauge, and a canonicalisation from random
        messages of just the measured instances (per-instance stopping rule;
        finished instances keep their state). ``samples`` (n_instances x
        max nodes) gives the uniform draws, otherwise they are drawn on the
        device from a generator seeded by ``seed``. Returns per instance the
        configuration 1 - 2 * outcomes (the state ends projected)."""
        L = self.layout
        dev = L.device
        sizes = [en.fields.shape[0] for en in self.energies]
        nmax = max(sizes)
        if samples is None:
            gen = torch.Generator(device=dev).manual_seed(int(seed))
            u_all = torch.rand((self.n_inst, nmax), generator=gen, dtype=torch.float64, device=dev)
        else:
            u_all = torch.as_tensor(np.asarray(samples, dtype=np.float64), device=dev)
        outcomes = torch.zeros((self.n_inst, nmax), dtype=torch.int64, device=dev)
        mp = _lib.MAX_PHYS
        for i in range(nmax):
            ks = [k for k in range(self.n_inst) if sizes[k] > i]
            nodes = [self.node_idx[(k, i)] for k in ks]
            nodes_dev = torch.as_tensor(nodes, dtype=torch.int32, device=dev)
            kdev = torch.as_tensor(ks, device=dev)
            # densities of the measured nodes (bp_quantum_emulator.py:188-207)
            T = torch.empty_like(self.G)
            _lib.call("dqz_symmetric_gauge", L.gptr, self.G.data_ptr(), self.lam.data_ptr(), EPS, T.data_ptr(),
                      _lib.stream_handle())
            n2e, e2n = L.new_msg_arena(), L.new_msg_arena()
            _lib.call("dqz_lambdas_to_messages", L.gptr, self.lam.data_ptr(), n2e.data_ptr(), e2n.data_ptr(),
                      L.max_chi(), _lib.stream_handle())
            rho = density_packed(L, T, e2n, nodes)
            r = (rho[:, 0, 0].real <= u_all[kdev, i]).to(torch.int64)
            outcomes[kdev, i] = r
            g = torch.zeros((len(nodes), mp * mp), dtype=torch.complex128, device=dev)
            g[:, 0] = (1 - r).to(torch.complex128)
            g[:, 3] = r.to(torch.complex128)
            _lib.call("dqz_apply1", L.gptr, self.G.data_ptr(), nodes_dev.data_ptr(), g.data_ptr(), len(nodes),
                      _lib.stream_handle())
            T = torch.empty_like(self.G)
            _lib.call("dqz_symmetric_gauge", L.gptr, self.G.data_ptr(), self.lam.data_ptr(), EPS, T.data_ptr(),
                      _lib.stream_handle())
            n2e, e2n = self._random_messages()
            vd = torch.zeros(self.n_inst, dtype=torch.float64, device=dev)
            vd[kdev] = np.finfo(np.float64).max
            G = self.G.clone()
            lam = self.lam.clone()
            orth = torch.empty(max(L.msg_elems, 1), dtype=torch.complex128, device=dev)
            partial = torch.zeros(max(L.n_halves, 1), dtype=torch.float64, device=dev)
            self.G, self.lam = self._bp_loop(T, n2e, e2n, vd, G, lam, orth, partial)
        out = outcomes.cpu().numpy()
        return [1 - 2 * out[k, : sizes[k]] for k in range(self.n_inst)]

    def truncation_errors(self) -> List[np.ndarray]:
        """Per instance, in gate application order."""
        per = [[] for _ in range(self.n_inst)]
        for layer, jobs, err, _ in self._err:
            e = err.cpu().numpy()
            for j, x in zip(jobs, e):
                per[self.topo.nodes[self.gate_u[j]].id[0]].append((layer, j, x))
        return [np.array([x for _, _, x in sorted(p)]) for p in per]
