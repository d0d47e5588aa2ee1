"""Hand-written adjoints behind torch.autograd.Function.

The reference has no derivative path (its BP loop is a Python ``while`` over
converged messages, bp_quantum_emulator.py:253-300); these Functions make the
GPU forward differentiable in FP64:

* ``BPFixedPoint`` -- BP run to its fixed point m* = F(m*, T) on the CUDA
  kernels, with the flooding sweep n2e_new = F(n2e_old) (every node reads the
  previous node->edge messages of its neighbours). Its fixed point is the one
  of the reference's synchronous and asynchronous sweeps
  (mappings/belief_propagation.py:24-64); the flooding form is used because
  it is exactly the map whose Jacobian the adjoint needs (the reference's
  synchronous sweep lags the edge->node messages by one sweep, so it repeats
  itself every other sweep). Its backward is implicit differentiation: the adjoint
  system x = g + J^H x (J = dF/dm at m*) is solved by repeated transposed
  message sweeps (``dqz_bp_node_vjp`` followed by the twin swap), then
  dL/dT = g_T + (dF/dT)^H x*, all on the device.
* torch-level differentiable forms of the maps around the fixed point (node
  tensors and messages as views of the packed arenas, one-site densities of
  mappings/density_matrix.py:16-37), used by the gradient workloads.

Complex gradients follow torch's convention, grad z = dL/dRe z + i dL/dIm z.
"""

from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .graph import Node, TensorGraph
from .layout import GraphLayout
from .maps import Topology, bp_sweep


class FixedPointProblem:
    """Packed layout and flooding-sweep tables of one tensor graph, plus the
    scratch of the transposed sweep. Bond dimensions are those of the graph."""

    def __init__(self, graph: TensorGraph, traversal: str = "dfs", topo: Optional[Topology] = None):
        """``topo``: a flooding Topology of the same graph to reuse (its
        traversal fixes node and edge order); bond dimensions are read from
        the graph's edges either way."""
        if not torch.cuda.is_available():
            raise RuntimeError("the adjoint runs on the GPU only")
        _lib.lib()
        if topo is None:
            trav = list(graph.get_traversal_iterator(ordering=traversal))
            topo = Topology(trav, True, flooding=True)
        elif not topo.flooding:
            raise ValueError("the fixed-point problem needs a flooding topology")
        self.topo = topo
        self.layout = GraphLayout(self.topo.nodes, self.topo.edges, [e.dimension for e in self.topo.edges])
        L = self.layout
        self.nodes_dev = torch.arange(L.n_nodes, dtype=torch.int32, device=L.device)
        self._edge_all = torch.ones(max(L.n_halves, 1), dtype=torch.uint8, device=L.device)
        self._scratch = None
        self.last_sweeps = 0
        self.last_adjoint_sweeps = 0

    # ------------------------------------------------------------ plumbing
    def swap(self, src: torch.Tensor) -> torch.Tensor:
        """out[h] = src[twin(h)] (the edge pass, pass_through_edge of
        tensor_ops.py:70-76)."""
        L = self.layout
        out = torch.zeros_like(src)
        _lib.call("dqz_bp_edge_pass", L.gptr, src.data_ptr(), src.data_ptr(), self._edge_all.data_ptr(),
                  out.data_ptr(), L.max_chi(), _lib.stream_handle())
        return out

    def sweep(self, T, n2e, e2n):
        n2e_new, e2n_new = torch.empty_like(n2e), torch.empty_like(e2n)
        bp_sweep(self.layout, self.topo, T, n2e, e2n, n2e_new, e2n_new)
        return n2e_new, e2n_new

    def converge(self, T, n2e, tol: float, max_sweeps: int) -> Tuple[torch.Tensor, torch.Tensor, int]:
        """Flooding sweeps from n2e until the largest node->edge message
        change is <= tol; returns (n2e*, e2n* = swap(n2e*), sweeps)."""
        e2n = self.swap(n2e)
        for it in range(1, max_sweeps + 1):
            n2e_new, e2n_new = self.sweep(T, n2e, e2n)
            d = float((n2e_new - n2e).abs().max())
            n2e, e2n = n2e_new, e2n_new
            if d <= tol:
                self.last_sweeps = it
                return n2e, e2n, it
        self.last_sweeps = max_sweeps
        return n2e, e2n, max_sweeps

    def node_vjp(self, T, e2n, n2e_cot, t_cot: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Transposed node update: returns the e2n cotangent arena; adds the
        node-tensor cotangent into t_cot when given."""
        L = self.layout
        if self._scratch is None:
            nb = _lib.lib().dqz_bp_node_vjp_scratch_bytes(L.n_nodes, L.max_size())
            self._scratch = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=L.device)
        out = torch.zeros_like(e2n)
        _lib.call("dqz_bp_node_vjp", L.gptr, T.data_ptr(), e2n.data_ptr(), n2e_cot.data_ptr(), out.data_ptr(),
                  _lib.ptr(t_cot), self.nodes_dev.data_ptr(), L.n_nodes, L.max_size(), L.max_chi(),
                  self._scratch.data_ptr(), _lib.stream_handle())
        return out

    def transposed_sweep(self, T, e2n, x):
        """J^H x for the flooding sweep map n2e_old -> n2e_new (its node
        updates read e2n = swap(n2e_old))."""
        return self.swap(self.node_vjp(T, e2n, x))

    # -------------------------------------------------------- torch views
    def node_tensors(self, arena: torch.Tensor) -> List[torch.Tensor]:
        """Differentiable per-node views (node shape) of a tensor arena."""
        L = self.layout
        out = []
        for v in range(L.n_nodes):
            shape = L.node_shape(v)
            o = int(L.node_off[v])
            out.append(arena[o : o + int(np.prod(shape))].view(shape))
        return out

    def messages(self, arena: torch.Tensor) -> List[torch.Tensor]:
        L = self.layout
        return [L.message_view(arena, h) for h in range(L.n_halves)]


class BPFixedPoint(torch.autograd.Function):
    """(T arena) -> (n2e*, e2n*) at the BP fixed point (flooding sweeps from
    n2e0), with the implicit adjoint as backward."""

    @staticmethod
    def forward(ctx, T, problem: FixedPointProblem, n2e0, tol: float = 1e-13, max_sweeps: int = 1000,
                adj_tol: float = 1e-13, adj_max: int = 1000):
        T = T.detach()
        n2e, e2n, _ = problem.converge(T, n2e0.detach(), tol, max_sweeps)
        ctx.problem = problem
        ctx.adj_tol, ctx.adj_max = adj_tol, adj_max
        ctx.save_for_backward(T, n2e, e2n)
        return n2e, e2n

    @staticmethod
    def backward(ctx, g_n2e, g_e2n):
        T, n2e, e2n = ctx.saved_tensors
        P: FixedPointProblem = ctx.problem
        g = torch.zeros_like(n2e)
        if g_n2e is not None:
            g = g + g_n2e
        if g_e2n is not None:
            g = g + P.swap(g_e2n.contiguous())  # e2n* = swap(n2e*)
        x = g.clone()
        scale = float(g.abs().max()) or 1.0
        it = 0
        for it in range(1, ctx.adj_max + 1):
            x_new = g + P.transposed_sweep(T, e2n, x)
            d = float((x_new - x).abs().max())
            x = x_new
            if d <= ctx.adj_tol * scale:
                break
        P.last_adjoint_sweeps = it
        t_cot = torch.zeros_like(T)
        P.node_vjp(T, e2n, x, t_cot)
        return t_cot, None, None, None, None, None, None


def contract_messages(T: torch.Tensor, msgs: Sequence[torch.Tensor]) -> torch.Tensor:
    """T x_f m_f over every bond (m_f contracted over its second index), bond
    order kept: the tensordot chain of tensor_ops.py:45 / density_matrix.py:26."""
    Y = T
    k = T.dim() - 1
    for f in range(k):
        Y = torch.movedim(torch.tensordot(msgs[f], Y, dims=([1], [f])), 0, f)
    return Y


def one_site_density(T: torch.Tensor, msgs: Sequence[torch.Tensor]) -> torch.Tensor:
    """mappings/density_matrix.py:16-37: rho[s, s'] = sum (T x_all m)[.., s]
    conj(T)[.., s'] / trace, differentiable."""
    Y = contract_messages(T, msgs)
    d = T.shape[-1]
    rho = Y.reshape(-1, d).T @ T.reshape(-1, d).conj()
    return rho / torch.diagonal(rho).sum()


def magnetisation_loss(problem: FixedPointProblem, T_arena: torch.Tensor, e2n: torch.Tensor,
                       weights: Optional[Sequence[float]] = None) -> torch.Tensor:
    """sum_v w_v <Z_v> = sum_v w_v (rho_v[0,0] - rho_v[1,1]) from the one-site
    densities at the fixed point (ibm_eagle_processor.py:124 form)."""
    Ts = problem.node_tensors(T_arena)
    ms = problem.messages(e2n)
    L = problem.layout
    total = T_arena.real.sum() * 0.0
    for v in range(L.n_nodes):
        h0, k = int(L.node_half[v]), int(L.degree[v])
        rho = one_site_density(Ts[v], ms[h0 : h0 + k])
        w = 1.0 if weights is None else float(weights[v])
        total = total + w * (rho[0, 0] - rho[1, 1]).real
    return total
