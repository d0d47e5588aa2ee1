"""Gradient of the final annealing energy with respect to the per-step
schedule values s_t, by a hand-written reverse pass with checkpointing.

Forward (one instance, Vidal form (Gamma, lambda), FP64 complex128):
  |+> product state; for t = 0..N-1 (second-order Trotter step of
  H(s) = -(1 - s) sum X + s sum J Z Z, dt fixed):
    regauge (t > 0): symmetric gauge (tensor_ops.py:189-199), BP to its fixed
        point from lambda messages (``BPFixedPoint``: CUDA sweeps forward,
        implicit adjoint with the transposed-sweep kernel backward), Vidal
        gauge (tensor_ops.py:88-130: eigh, square roots, SVD, absorb);
    exp(-i tau_m/2 X) on every qubit (tensor_graph.py:268-275);
    exp(-i tau_c (J Z Z + h_u/deg_u Z + h_v/deg_v Z)) on every coupled pair,
        in pair order, by simple update truncated to max_chi
        (tensor_ops.py:265-389);
    exp(-i tau_m/2 X) on every qubit;
  with tau_m = -dt (1 - s_t), tau_c = dt s_t; then a final regauge and
  E = sum_e J_e <Z_u Z_v> from the two-site reduced density matrices of the
  Vidal form.

Differences from the reference loop that keep the map smooth in s:
  * BP runs to its fixed point (max message change <= ``bp_tol``) instead of
    stopping at a Vidal-distance threshold, so the regauge is a function of
    the state;
  * a coupling gate is split analytically into two rank-2 halves,
    h1 = (cos(tau J) e^{-i tau h_u z}, -i sin(tau J) z e^{-i tau h_u z}),
    h2 = (e^{-i tau h_v z}, z e^{-i tau h_v z}), instead of by SVD; the product
    h1 . h2 is the same gate, so the physical state is unchanged (only the
    representation's scale factors differ);
  * the truncated two-site decomposition is the SVD of
    Theta = A_u diag(lambda_e x 1_r) A_v^T through ``product_svd`` (the
    reference's QR + core SVD forward, with the adjoint of Theta's own SVD).
Non-differentiable point: a coupling step with s_t = 0 exactly applies the
identity, and the Schmidt values it would create grow like |tau|; the
canonical form (square roots and safe inverses of lambda) is not
differentiable there although E is, and the reverse pass returns the
derivative with that bond component held at zero (dE/ds_t = 0 from the
coupling). Schedules should keep s_t > 0 (e.g. midpoint values (t + 1/2)/N).
Reverse pass: the forward stores (Gamma, lambda) every ``checkpoint_every``
steps; segments are recomputed under autograd in reverse order and
differentiated with the hand-written SVD / eigh adjoints of ``linalg_ad`` and
the implicit BP adjoint.
"""

import math
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from .adjoint import BPFixedPoint, FixedPointProblem
from .graph import TensorGraph
from .linalg_ad import eigh, product_svd, svd
from .maps import Topology
from .workloads import EnergyFunction, tensor_graph_of

F32_MAX = 3.4028234663852886e38
EPS = 1e-10


def safe_inverse(x: torch.Tensor, eps: float) -> torch.Tensor:
    """tensor_ops.py:20-21."""
    return 1.0 / ((x < eps).to(x.dtype) * F32_MAX + x)


def safe_sqrt_truncate(x: torch.Tensor, eps: float) -> torch.Tensor:
    """sqrt(safe_truncate(x)) with a finite derivative at the truncated entries."""
    keep = x > eps
    return torch.where(keep, torch.sqrt(torch.where(keep, x, torch.ones_like(x))), torch.zeros_like(x))


def _clone(x):
    """A detached copy of a state part (one tensor, or a list of them)."""
    return x.clone() if isinstance(x, torch.Tensor) else [t.clone() for t in x]


def _leaves(x):
    """Leaf copies (requires_grad) of a checkpointed state part."""
    if isinstance(x, torch.Tensor):
        return x.clone().requires_grad_(True)
    return [t.clone().requires_grad_(True) for t in x]


def _parts(x) -> List[torch.Tensor]:
    return [x] if isinstance(x, torch.Tensor) else list(x)


def _bcast(vec: torch.Tensor, axis: int, ndim: int) -> torch.Tensor:
    shape = [1] * ndim
    shape[axis] = vec.shape[0]
    return vec.reshape(shape)


class AnnealingGradient:
    """Differentiable annealing of one instance on the GPU."""

    def __init__(self, energy: EnergyFunction, max_chi: int, dt: float, checkpoint_every: int = 10,
                 bp_tol: float = 1e-13, bp_max: int = 2000, eps: float = EPS, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("the annealing gradient runs on the GPU only")
        self.energy = energy
        self.max_chi = int(max_chi)
        self.dt = float(dt)
        self.k = int(checkpoint_every)
        self.bp_tol, self.bp_max, self.eps = bp_tol, bp_max, eps
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.graph: TensorGraph = tensor_graph_of(energy)
        self.trav = list(self.graph.get_traversal_iterator())
        self.topo = Topology(self.trav, True, flooding=True)
        self.nodes = self.topo.nodes
        self.edges = self.topo.edges
        self.node_idx = {n.id: i for i, n in enumerate(self.nodes)}
        self.edge_idx = {e.id: i for i, e in enumerate(self.edges)}
        self.node_edges = [[self.edge_idx[e.id] for e in n.neighbors] for n in self.nodes]
        # edge -> (node a, bond index at a, node b, bond index at b), a = neighbours[0]
        self.edge_ends = []
        for e in self.edges:
            a, b = e.neighbors[0], e.neighbors[1]
            self.edge_ends.append((self.node_idx[a.id], a.indices[e.id], self.node_idx[b.id], b.indices[e.id]))
        deg = {n.id: len(n.neighbors) for n in self.nodes}
        self.gates = []  # (edge, node1, bond1, node2, bond2, J, h1/deg1, h2/deg2) in pair order
        for (a, b), J in zip(energy.coupled_spin_pairs, energy.coupling_amplitudes):
            a, b = int(a), int(b)
            e = self.graph.find_edge(a, b)
            na, nb = self.graph.get_node(a), self.graph.get_node(b)
            self.gates.append((self.edge_idx[e.id], self.node_idx[a], na.indices[e.id], self.node_idx[b],
                               nb.indices[e.id], float(J), float(energy.fields[a]) / deg[a],
                               float(energy.fields[b]) / deg[b]))
        self.z = torch.tensor([1.0, -1.0], dtype=torch.float64, device=self.device)
        self.last_bp_sweeps: List[int] = []
        # node-disjoint gate levels in pair order (gates on different nodes act
        # on different tensors, so a level runs as one batch)
        last = np.zeros(len(self.nodes), dtype=np.int64)
        lvl = np.zeros(len(self.gates), dtype=np.int64)
        for j, gt in enumerate(self.gates):
            lvl[j] = max(last[gt[1]], last[gt[3]]) + 1
            last[gt[1]] = last[gt[3]] = lvl[j]
        self.levels = [np.nonzero(lvl == l)[0].tolist() for l in range(1, int(lvl.max(initial=0)) + 1)]
        self.gate_J = torch.tensor([g[5] for g in self.gates], dtype=torch.float64, device=self.device)
        self.gate_hu = torch.tensor([g[6] for g in self.gates], dtype=torch.float64, device=self.device)
        self.gate_hv = torch.tensor([g[7] for g in self.gates], dtype=torch.float64, device=self.device)
        # stacked form: once every node has the same degree and every bond is
        # at max_chi (shapes no longer change), the state is one tensor
        # G (N, chi, .., chi, 2) and one L (E, chi), and every stage is a few
        # batched operations instead of one per node (host-side dispatch and
        # autograd bookkeeping dominated the per-node lists)
        degs = {len(n.neighbors) for n in self.nodes}
        self.uniform_degree = degs.pop() if len(degs) == 1 else 0
        self._stk = None
        self.use_stacked = True

    # ------------------------------------------------------------- state
    def initial_state(self) -> Tuple[List[torch.Tensor], List[torch.Tensor]]:
        """|+> on every qubit, all bonds of dimension 1, lambda = 1."""
        plus = torch.full((2,), math.sqrt(0.5), dtype=torch.complex128, device=self.device)
        gam = [plus.reshape((1,) * len(n.neighbors) + (2,)).clone() for n in self.nodes]
        lam = [torch.ones(1, dtype=torch.float64, device=self.device) for _ in self.edges]
        return gam, lam

    # ---------------------------------------------------------- gates
    def mixing_gate(self, tau):
        """exp(-i tau X) (quantum_annealer.py:72-84)."""
        c, s = torch.cos(tau), torch.sin(tau)
        zero = torch.zeros_like(c)
        re = torch.stack([torch.stack([c, zero]), torch.stack([zero, c])])
        im = torch.stack([torch.stack([zero, -s]), torch.stack([-s, zero])])
        return torch.complex(re, im)

    def coupling_halves(self, tau, idx: Sequence[int]):
        """Rank-2 halves (B, r, o, i) of exp(-i tau (J ZZ + hu Z + hv Z)) for the
        gates ``idx``, diagonal in (o, i)."""
        ix = torch.as_tensor(idx, device=self.device)
        J, hu, hv = self.gate_J[ix], self.gate_hu[ix], self.gate_hv[ix]
        z = self.z
        zc = z.to(torch.complex128)
        pu = torch.exp(torch.complex(torch.zeros_like(hu).unsqueeze(1) * z, -tau * hu.unsqueeze(1) * z))
        pv = torch.exp(torch.complex(torch.zeros_like(hv).unsqueeze(1) * z, -tau * hv.unsqueeze(1) * z))
        c = torch.cos(tau * J).to(torch.complex128).unsqueeze(1)
        sn = torch.sin(tau * J).to(torch.complex128).unsqueeze(1)
        h1 = torch.stack([torch.diag_embed(c * pu), torch.diag_embed(-1j * sn * zc * pu)], dim=1)
        h2 = torch.stack([torch.diag_embed(pv), torch.diag_embed(zc * pv)], dim=1)
        return h1, h2

    # ------------------------------------------------------- operations
    @staticmethod
    def _groups(keys) -> Dict:
        out: Dict = {}
        for i, k in enumerate(keys):
            out.setdefault(k, []).append(i)
        return out

    def apply1_all(self, gam, G):
        """tensor_graph.py:268-275 on every node, batched by tensor shape."""
        out = list(gam)
        for shape, vs in self._groups([tuple(g.shape) for g in gam]).items():
            X = torch.stack([gam[v] for v in vs])
            X = torch.tensordot(X, G, dims=([X.dim() - 1], [1]))
            X = X / torch.linalg.vector_norm(X.reshape(len(vs), -1), dim=1).reshape((-1,) + (1,) * (X.dim() - 1))
            for v, x in zip(vs, X.unbind(0)):  # unbind: one stack in the backward, not a select per item
                out[v] = x
        return out

    def _prepare(self, X, others: List[torch.Tensor], half):
        """tensor_ops.py:265-283 up to the QR for a batch: X (B, c_e, others.., d)
        with the gate bond first; lambda-scale the other bonds, apply the half
        gate (phys contracted with its input, rank merged into the gate bond
        bond-major, normalised), gate bond moved last -> (B, rows, c_e r)."""
        B = X.shape[0]
        nd = X.dim()
        for p, L in enumerate(others):
            shape = [B] + [1] * (nd - 1)
            shape[p + 2] = L.shape[1]
            X = X * L.reshape(shape).to(X.dtype)
        r = half.shape[1]
        ax = "xyzwuvtq"[: nd - 2]
        X = torch.einsum("b" + ax + "i,broi->b" + ax + "ro", X, half)
        # (B, c_e, others.., r, o) -> (B, c_e, r, others.., o) -> merge (c_e r)
        X = torch.movedim(X, nd - 1, 2)
        ce = X.shape[1]
        X = X.reshape((B, ce * r) + tuple(X.shape[3:]))
        X = X / torch.linalg.vector_norm(X.reshape(B, -1), dim=1).reshape((B,) + (1,) * (X.dim() - 1))
        X = torch.movedim(X, 1, -1)
        return X

    def _su_core(self, Xa, oa, Xb, ob, lam_e, h1, h2):
        """tensor_ops.py:318-389 for a batch of gates of identical shapes: Xa /
        Xb (B, c_e, others.., d) with the gate bond first, oa / ob the lambdas of
        the other bonds ((B, c) each, in bond order), lam_e (B, c_e) the gate
        bond's. Returns the new Gammas (B, others.., d, rank), rank last, and
        the kept lambdas (B, rank); rank = min(max_chi, available)."""
        B = Xa.shape[0]
        Pa = self._prepare(Xa, oa, h1)
        Pb = self._prepare(Xb, ob, h2)
        K = Pa.shape[-1]
        d = lam_e.repeat_interleave(h1.shape[1], dim=1).to(torch.complex128)
        Wa, S, Wb = product_svd(Pa.reshape(B, -1, K) * d.unsqueeze(1), Pb.reshape(B, -1, K))
        lmbd = (S > self.eps).to(S.dtype) * S
        rank = min(self.max_chi, S.shape[-1])

        def finish(W, P, others):
            q = W[..., :rank].reshape(P.shape[:-1] + (rank,))  # (B, others.., d, rank)
            nd = q.dim()
            for p, L in enumerate(others):
                shape = [B] + [1] * (nd - 1)
                shape[p + 1] = L.shape[1]
                q = q * safe_inverse(L, self.eps).reshape(shape).to(q.dtype)
            return q

        return finish(Wa, Pa, oa), finish(Wb, Pb, ob), lmbd[:, :rank]

    def _simple_update_group(self, gam, lam, idx: List[int], h1, h2):
        """tensor_ops.py:318-389 for node-disjoint gates of identical shapes,
        as one batch (rank = min(max_chi, available))."""
        gts = [self.gates[j] for j in idx]

        def side(node_pos, bond_pos):
            X = torch.stack([torch.movedim(gam[g[node_pos]], g[bond_pos], 0) for g in gts])
            nb = X.dim() - 2  # bonds of the node
            others = []
            for p in range(nb - 1):
                others.append(torch.stack([lam[[f for q, f in enumerate(self.node_edges[g[node_pos]])
                                                if q != g[bond_pos]][p]] for g in gts]))
            return X, others

        Xa, oa = side(1, 2)
        Xb, ob = side(3, 4)
        lam_e = torch.stack([lam[g[0]] for g in gts])
        qa, qb, lk = self._su_core(Xa, oa, Xb, ob, lam_e, h1, h2)
        gam = list(gam)
        lam = list(lam)
        for g, xa, xb, l in zip(gts, qa.unbind(0), qb.unbind(0), lk.unbind(0)):
            gam[g[1]] = torch.movedim(xa, xa.dim() - 1, g[2])  # (others.., d, rank): rank to the bond slot
            gam[g[3]] = torch.movedim(xb, xb.dim() - 1, g[4])
            lam[g[0]] = l
        return gam, lam

    def coupling_layer(self, gam, lam, tau):
        """All coupling gates in pair order, a level of node-disjoint gates
        at a time, each level batched by shape."""
        for level in self.levels:
            keys = []
            for j in level:
                e, a, ia, b, ib = self.gates[j][:5]
                keys.append((tuple(torch.movedim(gam[a], ia, 0).shape), tuple(torch.movedim(gam[b], ib, 0).shape)))
            for _, pos in self._groups(keys).items():
                idx = [level[p] for p in pos]
                h1, h2 = self.coupling_halves(tau, idx)
                gam, lam = self._simple_update_group(gam, lam, idx, h1, h2)
        return gam, lam

    # ------------------------------------------------------- stacked form
    def _stacked_tables(self):
        """Index tables of the stacked form (built once): node -> edges of its
        bonds, edge ends as half-edges, the per-half-edge source of the
        orthogonalisers, the coupling levels grouped by the gate's bond slots,
        and the fixed-point problem with every bond at max_chi."""
        if self._stk is not None:
            return self._stk
        dev, k, c = self.device, self.uniform_degree, self.max_chi
        E = len(self.edges)
        t = {"ne": torch.as_tensor(self.node_edges, dtype=torch.long, device=dev)}
        hf = [a * k + ia for a, ia, _, _ in self.edge_ends]
        hb = [b * k + ib for _, _, b, ib in self.edge_ends]
        t["hf"] = torch.as_tensor(hf, dtype=torch.long, device=dev)
        t["hb"] = torch.as_tensor(hb, dtype=torch.long, device=dev)
        perm = np.zeros(len(self.nodes) * k, dtype=np.int64)
        perm[hf] = np.arange(E)
        perm[hb] = E + np.arange(E)
        t["orth_src"] = torch.as_tensor(perm, device=dev)
        levels = []
        for level in self.levels:
            groups = {}
            for j in level:
                groups.setdefault((self.gates[j][2], self.gates[j][4]), []).append(j)
            out = []
            for (ia, ib), js in groups.items():
                gts = [self.gates[j] for j in js]

                def others(node_pos, bond_pos):
                    return torch.as_tensor([[f for q, f in enumerate(self.node_edges[g[node_pos]]) if q != g[bond_pos]]
                                            for g in gts], dtype=torch.long, device=dev)

                out.append({"gates": js, "ia": ia, "ib": ib,
                            "a": torch.as_tensor([g[1] for g in gts], dtype=torch.long, device=dev),
                            "b": torch.as_tensor([g[3] for g in gts], dtype=torch.long, device=dev),
                            "e": torch.as_tensor([g[0] for g in gts], dtype=torch.long, device=dev),
                            "oa": others(1, 2), "ob": others(3, 4)})
            levels.append(out)
        t["levels"] = levels
        # each level's groups concatenated, in group order
        t["level_cat"] = [{"gates": [j for grp in out for j in grp["gates"]],
                           "sizes": [len(grp["gates"]) for grp in out],
                           "e": torch.cat([grp["e"] for grp in out]),
                           "ab": torch.cat([grp["a"] for grp in out] + [grp["b"] for grp in out]),
                           "oa": torch.cat([grp["oa"] for grp in out]),
                           "ob": torch.cat([grp["ob"] for grp in out])} for out in levels]
        for e in self.edges:
            e.dimension = c
        t["problem"] = FixedPointProblem(self.graph, topo=self.topo)
        L = t["problem"].layout
        t["he"] = torch.as_tensor(L.half_edge.astype(np.int64), device=dev)
        self._stk = t
        return t

    def _stackable(self, gam, lam) -> bool:
        if not self.use_stacked or not self.uniform_degree or isinstance(gam, torch.Tensor):
            return False
        c, k = self.max_chi, self.uniform_degree
        shape = (c,) * k + (2,)
        return all(int(l.shape[0]) == c for l in lam) and all(tuple(g.shape) == shape for g in gam)

    def _coupling_layer_stacked(self, G, L, tau):
        """coupling_layer on the stacked form: per level, the gates grouped by
        their bond slots only to bring the gate bond first (one gather and
        movedim per group), then one batch for the whole level (one QR / SVD
        call: the solver calls have a fixed cost each), written back with one
        index_copy per level."""
        t = self._stacked_tables()
        k = self.uniform_degree
        for groups, cat in zip(t["levels"], t["level_cat"]):
            Xa = torch.cat([torch.movedim(G[grp["a"]], 1 + grp["ia"], 1) for grp in groups])
            Xb = torch.cat([torch.movedim(G[grp["b"]], 1 + grp["ib"], 1) for grp in groups])
            oa = [L[cat["oa"][:, p]] for p in range(k - 1)]
            ob = [L[cat["ob"][:, p]] for p in range(k - 1)]
            h1, h2 = self.coupling_halves(tau, cat["gates"])
            qa, qb, lk = self._su_core(Xa, oa, Xb, ob, L[cat["e"]], h1, h2)
            new_a, new_b = [], []
            for grp, xa, xb in zip(groups, qa.split(cat["sizes"]), qb.split(cat["sizes"])):
                new_a.append(torch.movedim(xa, xa.dim() - 1, 1 + grp["ia"]))
                new_b.append(torch.movedim(xb, xb.dim() - 1, 1 + grp["ib"]))
            G = G.index_copy(0, cat["ab"], torch.cat(new_a + new_b))
            L = L.index_copy(0, cat["e"], lk)
        return G, L

    def _regauge_stacked(self, G, L):
        """regauge on the stacked form (same operations, batched over all
        nodes and edges)."""
        t = self._stacked_tables()
        P = t["problem"]
        lay = P.layout
        N, k, c = G.shape[0], self.uniform_degree, self.max_chi
        sl = safe_sqrt_truncate(L, self.eps)
        X = G
        for f in range(k):
            shape = [N] + [1] * (k + 1)
            shape[f + 1] = c
            X = X * sl[t["ne"][:, f]].reshape(shape).to(X.dtype)
        X = X / torch.linalg.vector_norm(X.reshape(N, -1), dim=1).reshape((-1,) + (1,) * (k + 1))
        with torch.no_grad():
            n2e0 = torch.zeros(max(lay.msg_elems, 1), dtype=torch.complex128, device=self.device)
            n2e0[: lay.n_halves * c * c] = torch.diag_embed(L.detach().to(torch.complex128)[t["he"]]).reshape(-1)
        T_arena = X.reshape(-1)
        if T_arena.requires_grad:
            n2e, _ = BPFixedPoint.apply(T_arena, P, n2e0, self.bp_tol, self.bp_max, self.bp_tol, self.bp_max)
        else:
            n2e, _, _ = P.converge(T_arena, n2e0, self.bp_tol, self.bp_max)
        self.last_bp_sweeps.append(P.last_sweeps)
        per_half = n2e[: lay.n_halves * c * c].view(lay.n_halves, c, c)
        Gf, Gb, lb = self._edge_svd(per_half[t["hf"]], per_half[t["hb"]])
        O = torch.cat([Gf, Gb])[t["orth_src"]].view(N, k, c, c)
        ax = "abcdefgh"[:k]
        out = "pqrstuvw"[:k]
        spec = "n" + ax + "s," + ",".join("n" + ax[f] + out[f] for f in range(k)) + "->n" + out + "s"
        X = torch.einsum(spec, X, *[O[:, f] for f in range(k)])
        X = X / torch.linalg.vector_norm(X.reshape(N, -1), dim=1).reshape((-1,) + (1,) * (k + 1))
        return X, lb

    def _apply1_stacked(self, G, gate):
        X = torch.tensordot(G, gate, dims=([G.dim() - 1], [1]))
        N = X.shape[0]
        return X / torch.linalg.vector_norm(X.reshape(N, -1), dim=1).reshape((-1,) + (1,) * (X.dim() - 1))

    def _problem(self, lam) -> FixedPointProblem:
        for e, l in zip(self.edges, lam):
            e.dimension = int(l.shape[0])
        return FixedPointProblem(self.graph, topo=self.topo)

    def regauge(self, gam, lam):
        """Symmetric gauge, BP fixed point, Vidal gauge (nodes batched by tensor
        shape, edges by bond dimension)."""
        P = self._problem(lam)
        L = P.layout
        N = len(gam)
        node_groups = self._groups([tuple(g.shape) for g in gam])
        # sqrt(truncated lambda) of every edge, once (one stacked op when all
        # bonds have the same dimension)
        if len({int(l.shape[0]) for l in lam}) == 1:
            sl_stack = safe_sqrt_truncate(torch.stack(lam), self.eps)
            sqrt_lam = None
        else:
            sl_stack = None
            sqrt_lam = [safe_sqrt_truncate(l, self.eps) for l in lam]
        Ts: List = [None] * N
        for shape, vs in node_groups.items():
            X = torch.stack([gam[v] for v in vs])
            nd = X.dim()
            for f in range(nd - 2):
                if sl_stack is not None:
                    ix = torch.as_tensor([self.node_edges[v][f] for v in vs], device=self.device)
                    Lf = sl_stack[ix]
                else:
                    Lf = torch.stack([sqrt_lam[self.node_edges[v][f]] for v in vs])
                sh = [len(vs)] + [1] * (nd - 1)
                sh[f + 1] = Lf.shape[1]
                X = X * Lf.reshape(sh).to(X.dtype)
            X = X / torch.linalg.vector_norm(X.reshape(len(vs), -1), dim=1).reshape((-1,) + (1,) * (nd - 1))
            for v, x in zip(vs, X.unbind(0)):
                Ts[v] = x
        T_arena = torch.cat([T.reshape(-1) for T in Ts])
        with torch.no_grad():
            n2e0 = torch.zeros(max(L.msg_elems, 1), dtype=torch.complex128, device=self.device)
            chis = {int(l.shape[0]) for l in lam}
            if len(chis) == 1 and L.exact() and L.n_halves:
                c = chis.pop()
                lam_e = torch.stack([l.detach() for l in lam]).to(torch.complex128)
                he = torch.as_tensor(L.half_edge.astype(np.int64), device=self.device)
                n2e0[: L.n_halves * c * c] = torch.diag_embed(lam_e[he]).reshape(-1)
            else:
                for h in range(L.n_halves):
                    L.message_view(n2e0, h).copy_(torch.diag(lam[int(L.half_edge[h])].to(torch.complex128)))
        if T_arena.requires_grad:
            n2e, _ = BPFixedPoint.apply(T_arena, P, n2e0, self.bp_tol, self.bp_max, self.bp_tol, self.bp_max)
        else:
            n2e, _, _ = P.converge(T_arena, n2e0, self.bp_tol, self.bp_max)
        self.last_bp_sweeps.append(P.last_sweeps)
        chi_groups = self._groups([int(l.shape[0]) for l in lam])
        if len(chi_groups) == 1 and L.exact() and L.n_halves:
            # one gather of both ends of every edge (a view per half-edge would
            # give each its own full-arena gradient in the reverse pass)
            c = next(iter(chi_groups))
            per_half = n2e[: L.n_halves * c * c].view(L.n_halves, c, c)
            msgs = None
        else:
            msgs = P.messages(n2e)
        orth: Dict[Tuple[int, int], torch.Tensor] = {}
        new_lam: List = [None] * len(self.edges)
        for c, es in chi_groups.items():
            ends = [self.edge_ends[e] for e in es]
            if msgs is None:
                hf = torch.as_tensor([int(L.node_half[a]) + ia for a, ia, _, _ in ends], device=self.device)
                hb = torch.as_tensor([int(L.node_half[b]) + ib for _, _, b, ib in ends], device=self.device)
                mf, mb = per_half[hf], per_half[hb]
            else:
                mf = torch.stack([msgs[int(L.node_half[a]) + ia] for a, ia, _, _ in ends])
                mb = torch.stack([msgs[int(L.node_half[b]) + ib] for _, _, b, ib in ends])
            Gf, Gb, lb = self._edge_svd(mf, mb)
            for e, (a, ia, b, ib), gf, gb, l in zip(es, ends, Gf.unbind(0), Gb.unbind(0), lb.unbind(0)):
                orth[(a, ia)] = gf
                orth[(b, ib)] = gb
                new_lam[e] = l
        new_gam: List = [None] * N
        for shape, vs in node_groups.items():
            X = torch.stack([Ts[v] for v in vs])
            nb = X.dim() - 2
            ax = "abcdefgh"[:nb]
            out = "pqrstuvw"[:nb]
            ops = [X] + [torch.stack([orth[(v, f)] for v in vs]) for f in range(nb)]
            spec = "n" + ax + "s," + ",".join("n" + ax[f] + out[f] for f in range(nb)) + "->n" + out + "s"
            X = torch.einsum(spec, *ops)
            X = X / torch.linalg.vector_norm(X.reshape(len(vs), -1), dim=1).reshape((-1,) + (1,) * (nb + 1))
            for v, x in zip(vs, X.unbind(0)):
                new_gam[v] = x
        return new_gam, new_lam

    def _edge_svd(self, mf, mb):
        """tensor_ops.py:108-130 for a batch of edges (messages (B, c, c))."""
        eps = self.eps
        lf, uf = eigh(0.5 * (mf + mf.mH))
        lb, ub = eigh(0.5 * (mb + mb.mH))

        def sq(l, u, inv):
            w = torch.sqrt(safe_inverse(l, eps)) if inv else safe_sqrt_truncate(l, eps)
            return (u * w.to(u.dtype).unsqueeze(-2)) @ u.mH

        m_sq_inv_f, m_sq_inv_b = sq(lf, uf, True), sq(lb, ub, True)
        u, s, vh = svd(sq(lf, uf, False) @ sq(lb, ub, False).mT)
        s = s / torch.linalg.vector_norm(s, dim=-1, keepdim=True)
        keep = (s > eps).to(s.dtype)
        s = keep * s
        u = u * keep.to(u.dtype).unsqueeze(-2)
        u = u / torch.linalg.vector_norm(u, dim=(-2, -1), keepdim=True)
        vh = vh * keep.to(vh.dtype).unsqueeze(-1)
        vh = vh / torch.linalg.vector_norm(vh, dim=(-2, -1), keepdim=True)
        return m_sq_inv_f @ u, m_sq_inv_b @ vh.mT, s

    def step(self, gam, lam, s_t, first: bool):
        """One second-order step. The state is per-node / per-edge lists, or
        (stacked form, from the first step whose input has every bond at
        max_chi on a graph of uniform degree) one tensor each."""
        tau_m = -self.dt * (1.0 - s_t)
        tau_c = self.dt * s_t
        if self._stackable(gam, lam):
            gam, lam = torch.stack(list(gam)), torch.stack(list(lam))
        half = self.mixing_gate(tau_m / 2)
        if isinstance(gam, torch.Tensor):
            if not first:
                gam, lam = self._regauge_stacked(gam, lam)
            gam = self._apply1_stacked(gam, half)
            gam, lam = self._coupling_layer_stacked(gam, lam, tau_c)
            return self._apply1_stacked(gam, half), lam
        if not first:
            gam, lam = self.regauge(gam, lam)
        gam = self.apply1_all(gam, half)
        gam, lam = self.coupling_layer(gam, lam, tau_c)
        gam = self.apply1_all(gam, half)
        return gam, lam

    def final_regauge(self, gam, lam):
        """The last regauge; returns per-node / per-edge lists."""
        if self._stackable(gam, lam):
            gam, lam = torch.stack(list(gam)), torch.stack(list(lam))
        if isinstance(gam, torch.Tensor):
            gam, lam = self._regauge_stacked(gam, lam)
            return list(gam.unbind(0)), list(lam.unbind(0))
        return self.regauge(gam, lam)

    # ------------------------------------------------------- observables
    def energy_of(self, gam, lam) -> torch.Tensor:
        """sum_e J_e <Z_u Z_v> from two-site reduced density matrices of the
        Vidal form (lambda on every bond of the pair, the shared one once)."""
        total = torch.zeros((), dtype=torch.float64, device=self.device)
        zz = self.z.unsqueeze(1) * self.z.unsqueeze(0)
        for gate in self.gates:
            e, a, ia, b, ib, J = gate[:6]
            A = gam[a]
            for f, ei in enumerate(self.node_edges[a]):
                A = A * _bcast(lam[ei].to(A.dtype), f, A.dim())
            B = gam[b]
            for f, ei in enumerate(self.node_edges[b]):
                if f != ib:
                    B = B * _bcast(lam[ei].to(B.dtype), f, B.dim())
            A = torch.movedim(A, ia, 0)
            B = torch.movedim(B, ib, 0)
            theta = torch.tensordot(A, B, dims=([0], [0]))  # (rest_a.., o_a, rest_b.., o_b)
            theta = torch.movedim(theta, A.dim() - 2, 0)
            theta = torch.movedim(theta, -1, 1)  # (o_a, o_b, rest..)
            p = (theta.abs() ** 2).reshape(2, 2, -1).sum(-1)
            total = total + J * (zz * p).sum() / p.sum()
        return total

    def one_site_z(self, gam, lam) -> torch.Tensor:
        """<Z_v> per node (traversal order) from the Vidal form."""
        out = []
        for v, G in enumerate(gam):
            T = G
            for f, ei in enumerate(self.node_edges[v]):
                T = T * _bcast(lam[ei].to(T.dtype), f, T.dim())
            p = (T.abs() ** 2).reshape(-1, 2).sum(0)
            out.append((p[0] - p[1]) / p.sum())
        return torch.stack(out)

    # ---------------------------------------------------------- driver
    def final_state(self, s_values: Sequence[float]):
        """(Gamma, lambda) after the last step and the final regauge."""
        s = torch.as_tensor(np.asarray(s_values, dtype=np.float64), device=self.device)
        gam, lam = self.initial_state()
        with torch.no_grad():
            for t in range(s.shape[0]):
                gam, lam = self.step(gam, lam, s[t], first=(t == 0))
            return self.final_regauge(gam, lam)

    def forward(self, s_values: torch.Tensor):
        """No-grad forward; returns (energy, checkpoints)."""
        gam, lam = self.initial_state()
        checkpoints = []
        with torch.no_grad():
            for t in range(s_values.shape[0]):
                if t % self.k == 0:
                    checkpoints.append((t, _clone(gam), _clone(lam)))
                gam, lam = self.step(gam, lam, s_values[t], first=(t == 0))
            gam, lam = self.final_regauge(gam, lam)
            E = self.energy_of(gam, lam)
        return E, checkpoints

    def energy_value(self, s_values: Sequence[float]) -> float:
        s = torch.as_tensor(np.asarray(s_values, dtype=np.float64), device=self.device)
        return float(self.forward(s)[0])

    def value_and_grad(self, s_values: Sequence[float]) -> Tuple[float, np.ndarray]:
        """E and dE/ds_t for every step, by checkpointed reverse passes."""
        s_all = torch.as_tensor(np.asarray(s_values, dtype=np.float64), device=self.device)
        n = s_all.shape[0]
        E, checkpoints = self.forward(s_all)
        grad = torch.zeros(n, dtype=torch.float64, device=self.device)
        cot = None
        for ci in range(len(checkpoints) - 1, -1, -1):
            t0, g0, l0 = checkpoints[ci]
            t1 = checkpoints[ci + 1][0] if ci + 1 < len(checkpoints) else n
            gam, lam = _leaves(g0), _leaves(l0)
            s_seg = s_all[t0:t1].clone().requires_grad_(True)
            g_cur, l_cur = gam, lam
            for j in range(t1 - t0):
                g_cur, l_cur = self.step(g_cur, l_cur, s_seg[j], first=(t0 + j == 0))
            if cot is None:
                g_cur, l_cur = self.final_regauge(g_cur, l_cur)
                outs = [self.energy_of(g_cur, l_cur)]
                gouts = [torch.ones_like(outs[0])]
            else:
                # this segment's output has the representation of the next
                # segment's checkpoint (the same steps produced both)
                pairs = [(o, c) for o, c in zip(_parts(g_cur) + _parts(l_cur), cot) if o.requires_grad]
                outs = [o for o, _ in pairs]
                gouts = [c for _, c in pairs]
            ins = _parts(gam) + _parts(lam) + [s_seg]
            grads = torch.autograd.grad(outs, ins, grad_outputs=gouts, allow_unused=True)
            grads = [torch.zeros_like(x) if gr is None else gr for x, gr in zip(ins, grads)]
            grad[t0:t1] += grads[-1]
            cot = grads[:-1]
        return float(E), grad.cpu().numpy()
