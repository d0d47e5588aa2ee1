"""Adjoint of the BP fixed point on the GPU.

* dqz_bp_node_vjp against torch autograd of a plain torch restatement of the
  node update (tensor_ops.py:36-60) in FP64: every incoming-message and
  node-tensor cotangent to 1e-11 relative.
* BPFixedPoint (implicit differentiation, transposed sweeps) against central
  finite differences (h = 1e-4) of the oracle's CPU forward (BP to 1e-14, then
  one-site densities): directional derivatives within 1e-5 relative, the
  accuracy asked of the adjoint.
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import graph as G
from dequantizer_b200.adjoint import BPFixedPoint, FixedPointProblem, magnetisation_loss
from dequantizer_b200.graph import MessageID, Node
from oracle import maps as OM
from tests.helpers import random_messages, random_tensors

pytestmark = pytest.mark.gpu


def _node_update_torch(T, msgs, e):
    Y = T
    k = T.dim() - 1
    for f in range(k):
        if f != e:
            Y = torch.movedim(torch.tensordot(msgs[f], Y, dims=([1], [f])), 0, f)
    axes = [a for a in range(k + 1) if a != e]
    M = torch.tensordot(T.conj(), Y, dims=(axes, axes))
    return M / torch.diagonal(M).sum()


@pytest.mark.parametrize("make", [lambda: G.get_random_tree_tensor_graph(8, 2, [2, 3, 4], 3),
                                  lambda: G.get_random_regular_graph(6, 3, 2, 3, 1),
                                  lambda: G.get_nd_lattice([2, 3], 2, 2)], ids=["tree", "regular3", "lattice"])
def test_node_vjp_matches_autograd(make):
    g = make()
    P = FixedPointProblem(g)
    L = P.layout
    rng = np.random.default_rng(0)
    tensors = random_tensors(g, 1)
    T = L.pack_tensors([torch.from_numpy(tensors[n.id]).cuda() for n in P.topo.nodes])
    msgs = random_messages(g, 2)
    e2n = L.pack_messages([torch.from_numpy(msgs[MessageID(e.id, nd.id)]).cuda() for nd, e in P.topo.half_ids()])
    cot = torch.zeros_like(e2n)
    for h in range(L.n_halves):
        c = int(L.edge_chi[L.half_edge[h]])
        z = rng.standard_normal((c, c, 2))
        L.message_view(cot, h).copy_(torch.from_numpy(z[..., 0] + 1j * z[..., 1]))
    t_cot = torch.zeros_like(T)
    e2n_cot = P.node_vjp(T, e2n, cot, t_cot)
    # autograd reference
    Tr = T.clone().requires_grad_(True)
    Mr = e2n.clone().requires_grad_(True)
    Ts = P.node_tensors(Tr)
    ms = P.messages(Mr)
    loss = 0.0
    for v in range(L.n_nodes):
        h0, k = int(L.node_half[v]), int(L.degree[v])
        for e in range(k):
            out = _node_update_torch(Ts[v], ms[h0 : h0 + k], e)
            loss = loss + (L.message_view(cot, h0 + e).conj() * out).real.sum()
    gT, gM = torch.autograd.grad(loss, (Tr, Mr))
    assert float((t_cot - gT).abs().max() / gT.abs().max()) < 1e-11
    assert float((e2n_cot - gM).abs().max() / gM.abs().max()) < 1e-11


def _oracle_loss(g, trav, tensors, weights):
    bp = OM.get_belief_propagation_map(trav, True)
    msgs = random_messages(g, 3)
    for _ in range(2000):
        new = bp(tensors, msgs)
        d = max(np.abs(new[k] - msgs[k]).max() for k in new)
        msgs = new
        if d < 1e-14:
            break
    total = 0.0
    for el in trav:
        if isinstance(el, Node):
            rho = OM.get_one_side_density_matrix(el, tensors, msgs)
            total += weights[el.id] * float((rho[0, 0] - rho[1, 1]).real)
    return total


@pytest.mark.parametrize("make", [lambda: G.get_random_regular_graph(10, 3, 2, 3, 4),
                                  lambda: G.get_nd_lattice([3, 3], 2, 2)], ids=["regular3", "lattice"])
def test_fixed_point_gradient_matches_finite_differences(make):
    g = make()
    P = FixedPointProblem(g)
    L = P.layout
    rng = np.random.default_rng(5)
    tensors = random_tensors(g, 7)
    # positive-leaning tensors keep BP comfortably convergent
    tensors = {k: np.abs(v) + 0.3 * v for k, v in tensors.items()}
    weights = {n.id: float(rng.uniform(-1, 1)) for n in P.topo.nodes}
    T = L.pack_tensors([torch.from_numpy(tensors[n.id]).cuda() for n in P.topo.nodes]).requires_grad_(True)
    msgs0 = random_messages(g, 3)
    n2e0 = L.pack_messages([torch.from_numpy(msgs0[MessageID(nd.id, e.id)]).cuda() for nd, e in P.topo.half_ids()])
    n2e, e2n = BPFixedPoint.apply(T, P, n2e0, 1e-14, 2000, 1e-14, 2000)
    loss = magnetisation_loss(P, T, e2n, [weights[n.id] for n in P.topo.nodes])
    (gT,) = torch.autograd.grad(loss, (T,))
    trav = list(g.get_traversal_iterator())
    assert abs(float(loss.detach()) - _oracle_loss(g, trav, tensors, weights)) < 1e-11
    h = 1e-4
    for trial in range(3):
        dirs = {}
        for n in P.topo.nodes:
            z = rng.standard_normal(tensors[n.id].shape + (2,))
            dirs[n.id] = z[..., 0] + 1j * z[..., 1]
        D = L.pack_tensors([torch.from_numpy(dirs[n.id]).cuda() for n in P.topo.nodes])
        ad = float((gT.conj() * D).real.sum())
        lp = _oracle_loss(g, trav, {k: tensors[k] + h * dirs[k] for k in tensors}, weights)
        lm = _oracle_loss(g, trav, {k: tensors[k] - h * dirs[k] for k in tensors}, weights)
        fd = (lp - lm) / (2 * h)
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-3), (ad, fd)
