"""The torch.ops.dqz operators on the GPU: a BP sweep composed from the
registered operators gives the package's own sweep bit for bit.

The package calls libdqz through ctypes; ``torch.ops.dqz.*`` are the same
entry points registered as PyTorch custom operators for code that composes
them with other torch operators. Here one synchronous sweep (node updates per
level, then the edge pass; mappings/belief_propagation.py:24-64) and the
message distance (mappings/messages_distance.py:14-22) are run through the
operators for the three node kernels: generic (heavy-hex cell, degrees 2 and
3), degree-3 FP64, and the tcgen05 BF16 form (with the operator that packs
its BF16 layouts), and compared with BPEngine on the same inputs.
"""

import numpy as np
import pytest
import torch

import dequantizer_b200.torch_ops  # noqa: F401  (registers torch.ops.dqz)
from dequantizer_b200 import graph as G
from dequantizer_b200.engine import BPEngine
from dequantizer_b200.graph import MessageID
from dequantizer_b200.maps import error_flag
from tests.helpers import random_messages, random_tensors

pytestmark = pytest.mark.gpu


def _engine(g, precision):
    eng = BPEngine(g, schedule="sync", precision=precision)
    ts = random_tensors(g, 5)
    ms = random_messages(g, 6)
    eng.load_tensors([ts[n.id] / np.linalg.norm(ts[n.id]) for n in eng.topo.nodes])
    eng.load_messages([ms[MessageID(nd.id, e.id)] for nd, e in eng.topo.half_ids()],
                      [ms[MessageID(e.id, nd.id)] for nd, e in eng.topo.half_ids()])
    return eng


@pytest.mark.parametrize("case", ["generic", "k3_fp64", "k3_bf16"])
def test_sweep_through_torch_ops_equals_package(case):
    if case == "generic":
        g = G.get_heavy_hex_ibm_eagle_lattice_infinite()
        for e in g.edges.values():
            e.dimension = 5
        g.refresh_bond_shapes()
        precision = "fp64"
    else:
        g = G.get_random_regular_graph(24, 3, 2, 16, 3)
        precision = "bf16" if case == "k3_bf16" else "fp64"
    ref = _engine(g, precision)
    ops = _engine(g, precision)
    L, topo, dev = ops.layout, ops.topo, ops.layout.device
    T, n2e, e2n = ops.T.clone(), ops.n2e.clone(), ops.e2n.clone()
    n2e_new, e2n_new = torch.zeros_like(n2e), torch.zeros_like(e2n)
    src_sel, edge_new, levels = topo.device_tables(dev)
    flag = error_flag(dev)
    if case == "generic":
        for halves in levels:
            torch.ops.dqz.bp_node_update(L.handle, T, n2e, e2n, n2e_new, src_sel, halves, L.max_slice(), L.max_chi())
    elif case == "k3_fp64":
        for halves in levels:
            torch.ops.dqz.bp_node_update_k3(L.handle, 16, T, n2e, e2n, n2e_new, src_sel, halves, flag)
    else:
        per_node = int(dequantizer_b200.torch_ops._lib.lib().dqz_bf16_umma_elems_per_node())
        T_bf16 = torch.empty(L.n_nodes * per_node, dtype=torch.bfloat16, device=dev)
        torch.ops.dqz.pack_bf16_umma(L.handle, T, T_bf16)
        for nodes in topo.device_node_levels(dev):
            torch.ops.dqz.bp_node_update_k3_umma(L.handle, T_bf16, n2e, e2n, n2e_new, src_sel, nodes, flag)
    torch.ops.dqz.bp_edge_pass(L.handle, n2e, n2e_new, edge_new, e2n_new, L.max_chi())
    partial = torch.empty(2 * L.n_halves, dtype=torch.float64, device=dev)
    dist = torch.empty((), dtype=torch.float64, device=dev)
    c = (lambda x: x.to(torch.complex128))
    torch.ops.dqz.messages_distance(L.handle, c(n2e_new), c(n2e), c(e2n_new), c(e2n), partial, dist, L.max_chi())
    ref.sweep()
    ref.check()
    torch.cuda.synchronize()
    assert int(flag.item()) == 0
    assert torch.equal(n2e_new, ref.n2e)
    assert torch.equal(e2n_new, ref.e2n)
    assert float(dist) == float(ref.distance())
