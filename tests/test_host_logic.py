"""Host-side logic on CPU: the C ABI library loads and exports every symbol
of include/dqz.h, gate splitting, shape rules, the BP sweep schedule, and
the packed layout."""

import os
import re

import numpy as np
import pytest
import torch

from dequantizer_b200 import _lib
from dequantizer_b200 import graph as G
from dequantizer_b200.gates import decompose_gate, decompose_gates
from dequantizer_b200.graph import Edge, MessageID, Node
from dequantizer_b200.layout import GraphLayout
from dequantizer_b200.maps import Topology
from dequantizer_b200.tensor_graph_ops import simple_update_shapes
from oracle import tensor_ops as OT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "dqz.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|size_t)\s+(dqz_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    declared = header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
        assert name in _lib.exported_symbols(), f"{name} has no ctypes signature"
    assert lib.dqz_version() >= 1


def test_scratch_queries_are_host_only():
    lib = _lib.lib()
    assert lib.dqz_bp_node_scratch_bytes(3072, 512, 16) == 0
    assert lib.dqz_bp_node_scratch_bytes(100, 65536, 32) > 0
    # one byte per job (rounded up to 256) marking the on-chip jobs, then a
    # 64 * rows * cols slice per CTA of the global-scratch kernel
    # marks, then the larger of the one-CTA kernel's matrices (4 x rows x cols
    # complex per job) and the cluster form's global workspace (two CTAs per
    # job, 2 rows cols + 3 cols^2 + 8 cols + 64 complex each)
    one_cta = 10 * 64 * 2048 * 64
    cluster = 2 * 10 * (2 * 2048 * 64 + 3 * 64 * 64 + 8 * 64 + 64) * 16
    assert lib.dqz_simple_update_scratch_bytes(10, 2048, 64) == 256 + max(one_cta, cluster)
    assert lib.dqz_simple_update_scratch_bytes(10, 128, 16) == 256 + 10 * 64 * 128 * 16
    assert lib.dqz_absorb_scratch_bytes(127, 8192) > 0


def test_entry_points_reject_bad_arguments_without_launching():
    lib = _lib.lib()
    assert lib.dqz_bp_node_update(None, None, None, None, None, None, None, 0, 0, 0, None, None) == _lib.DQZ_ERR_ARG
    assert lib.dqz_apply1(None, None, None, None, 1, None) == _lib.DQZ_ERR_ARG
    assert lib.dqz_reduce_sum(None, 0, 1.0, None, None) == _lib.DQZ_ERR_ARG
    with pytest.raises(_lib.DqzError):
        _lib.call("dqz_repack", None, None, None, None, None, 1, 16, None)


@pytest.mark.parametrize("seed", range(5))
def test_decompose_gates_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((4, 4, 2))
    u, _ = np.linalg.qr(z[..., 0] + 1j * z[..., 1])
    for gate in (u.reshape(2, 2, 2, 2), np.diag(np.exp(1j * rng.standard_normal(4))).reshape(2, 2, 2, 2),
                 np.eye(4).reshape(2, 2, 2, 2)):
        h1, h2 = decompose_gate(gate, 1e-10)
        o1, o2 = OT.decompose_gate(gate, 1e-10)
        assert h1.shape == o1.shape and h2.shape == o2.shape
        assert np.allclose(h1, o1, atol=1e-13) and np.allclose(h2, o2, atol=1e-13)
    batch = rng.standard_normal((7, 2, 2, 2, 2)) + 1j * rng.standard_normal((7, 2, 2, 2, 2))
    flat, ranks, _ = decompose_gates(batch, 1e-10)
    assert flat.shape == (7, 2, 4 * _lib.MAX_PHYS**2) and (ranks == 4).all()


def _diag_cases(rng):
    n = 400
    J = rng.choice([-1.0, 1.0], n)
    h1, h2 = rng.normal(size=n), rng.normal(size=n)
    s1, s2 = np.array([1.0, 1.0, -1.0, -1.0]), np.array([1.0, -1.0, 1.0, -1.0])
    ham = J[:, None] * s1 * s2 + h1[:, None] * s1 + h2[:, None] * s2
    out = [np.exp(-1j * tau * ham) for tau in (0.0, 1e-12, 0.05, 0.7, np.pi / 4, np.pi / 2)]
    out.append(rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4)))  # generic complex
    z = rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4))
    z[: n // 4, 0] = 0.0  # zero entries
    z[n // 4 : n // 2, :2] = 0.0  # zero row
    z[n // 2 : 3 * n // 4, 1] = z[n // 2 : 3 * n // 4, 0]  # rank one: rows equal
    z[n // 2 : 3 * n // 4, 3] = z[n // 2 : 3 * n // 4, 2]
    out.append(z)
    out.append(np.zeros((3, 4), dtype=np.complex128))
    return out


@pytest.mark.parametrize("seed", range(3))
def test_diagonal_gate_split_matches_dense_split(seed):
    """Closed-form split of diagonal gates: same ranks as the dense SVD split,
    and the halves contract to the same (rank-truncated) gate, within 1e-14."""
    from dequantizer_b200.gates import decompose_diagonal_gates, expand_diagonal_halves

    for diag in _diag_cases(np.random.default_rng(seed)):
        n = diag.shape[0]
        gates = np.zeros((n, 4, 4), dtype=np.complex128)
        gates[:, np.arange(4), np.arange(4)] = diag
        gates = gates.reshape(n, 2, 2, 2, 2)
        dense, r_dense, _ = decompose_gates(gates, 1e-10)
        compact, ranks = decompose_diagonal_gates(diag, 1e-10)
        assert (ranks == r_dense).all()

        def contract(flat):
            h1 = flat[:, 0, :16].reshape(n, 4, 2, 2)
            h2 = flat[:, 1, :16].reshape(n, 4, 2, 2)
            return np.einsum("nrai,nrbj->nabij", h1, h2)

        # equal to the dense split's product (which drops singular values <= eps too)
        back = contract(expand_diagonal_halves(compact))
        assert np.abs(back - contract(dense)).max() < 1e-14 * max(1.0, np.abs(diag).max())
        # discarded ranks are zero
        assert np.all(compact[ranks < 2][:, :, 2:] == 0)


@pytest.mark.parametrize("seed", range(6))
def test_simple_update_shape_rule_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    g = G.get_random_tree_tensor_graph(6, 2, [1, 2, 3], seed)
    eid = list(g.edges)[int(rng.integers(0, 5))]
    a, b = eid
    na, nb = g.get_node(a), g.get_node(b)
    ta = rng.standard_normal(na.bond_shape + (2,)) + 0j
    tb = rng.standard_normal(nb.bond_shape + (2,)) + 0j
    lam_a = [rng.uniform(0.1, 1, e.dimension) for e in na.neighbors]
    lam_b = [rng.uniform(0.1, 1, e.dimension) for e in nb.neighbors]
    lam_b[nb.indices[eid]] = lam_a[na.indices[eid]]
    gate = np.diag(np.exp(1j * rng.standard_normal(4))).reshape(2, 2, 2, 2)
    h1, h2 = OT.decompose_gate(gate, 1e-10)
    for max_rank in (None, 1, 2, 5):
        t1, t2, lam, _, _ = OT.simple_update(ta, tb, lam_a, lam_b, h1, h2, na.indices[eid], nb.indices[eid], 1e-10,
                                             None, max_rank)
        _, _, _, new, _ = simple_update_shapes(list(na.bond_shape), 2, na.indices[eid], list(nb.bond_shape), 2,
                                               nb.indices[eid], h1.shape[0], max_rank)
        assert lam.shape[0] == new == t1.shape[na.indices[eid]] == t2.shape[nb.indices[eid]]


def _symbolic_async_sweep(traverser):
    """The reference's asynchronous sweep (belief_propagation.py:32-61) run
    on tags instead of arrays: returns, per (node, edge), the tag the node
    read, and per (edge, node) the tag the edge emitted."""
    messages = {}
    for el in traverser:
        for nb in el.neighbors:
            messages[MessageID(nb.id, el.id)] = ("old", nb.id, el.id)
    updated, read, emitted = {}, {}, {}
    for el in traverser:
        incoming = []
        for nb in el.neighbors:
            mid = MessageID(nb.id, el.id)
            incoming.append(updated.get(mid, messages[mid]))
        if isinstance(el, Node):
            for nb, tag in zip(el.neighbors, incoming):
                read[(el.id, nb.id)] = tag
            out = [("new", el.id, nb.id) for nb in el.neighbors]
        else:
            out = [incoming[1], incoming[0]]
            for nb, tag in zip(el.neighbors, out):
                emitted[(el.id, nb.id)] = tag
        for nb, m in zip(el.neighbors, out):
            updated[MessageID(el.id, nb.id)] = m
    return read, emitted


@pytest.mark.parametrize("ordering", ["dfs", "bfs"])
@pytest.mark.parametrize("make", [lambda: G.get_nd_lattice([3, 3, 2], 2, 2),
                                  lambda: G.get_random_regular_graph(20, 3, 2, 2, 4),
                                  lambda: G.get_heavy_hex_ibm_eagle_lattice(),
                                  lambda: G.get_random_tree_tensor_graph(25, 2, [2], 3)])
def test_async_schedule_reproduces_reference_sweep(make, ordering):
    g = make()
    trav = list(g.get_traversal_iterator(ordering=ordering))
    topo = Topology(trav, is_synchronous=False)
    read, emitted = _symbolic_async_sweep(trav)
    level = {}
    for lv, halves in enumerate(topo.levels):
        for h in halves:
            level[int(h)] = lv
    h = 0
    node_level = {}
    for nd in topo.nodes:
        for slot, e in enumerate(nd.neighbors):
            node_level[nd.id] = level[topo.node_half[topo.node_index[nd.id]] + slot]
    for nd in topo.nodes:
        for e in nd.neighbors:
            u = e.neighbors[1] if e.neighbors[0] is nd else e.neighbors[0]
            tag = read[(nd.id, e.id)]
            sel = topo.src_sel[h]
            if tag[0] == "old" and tag[1] == e.id:
                assert sel == _lib.SRC_E2N_OLD
            elif tag[0] == "old":
                assert sel == _lib.SRC_N2E_OLD and tag[1] == u.id
            else:
                assert sel == _lib.SRC_N2E_NEW and tag[1] == u.id
                assert node_level[nd.id] > node_level[u.id]
            etag = emitted[(e.id, nd.id)]
            assert topo.edge_new[h] == (1 if etag[0] == "new" else 0)
            h += 1


def test_layout_pack_roundtrip_on_host():
    g = G.get_random_tree_tensor_graph(7, 3, [1, 2, 4], 9)
    nodes, edges = list(g.nodes.values()), list(g.edges.values())
    L = GraphLayout(nodes, edges, [e.dimension for e in edges], device=torch.device("cpu"),
                    node_capacity=[2 * int(np.prod(n.bond_shape)) * 3 for n in nodes])
    rng = np.random.default_rng(0)
    ts = [torch.from_numpy(rng.standard_normal(n.bond_shape + (3,)) + 0j) for n in nodes]
    arena = L.pack_tensors(ts)
    back = L.unpack_tensors(arena)
    for a, b in zip(ts, back):
        assert torch.equal(a, b)
    for v, nd in enumerate(nodes):
        for slot, e in enumerate(nd.neighbors):
            h = L.node_half[v] + slot
            assert L.edges[L.half_edge[h]] is e
            tw = L.half_twin[h]
            assert L.half_edge[tw] == L.half_edge[h] and L.half_node[tw] != v


@pytest.mark.parametrize("make", [lambda: G.get_nd_lattice([3, 3, 2], 2, 2),
                                  lambda: G.get_heavy_hex_ibm_eagle_lattice_infinite()])
def test_sweep_plan_matches_layout_tables(make):
    """The host plan of the one-CTA sweep (dqz_bp_sweep_planned): for every
    item of the flat level table, the node offset, degree, physical
    dimension, slot, outgoing message offset, bond dimensions and, per other
    bond in order, the incoming message as offset * 4 + source, as the
    kernels that walk the graph tables would find them."""
    g = make()
    topo = Topology(list(g.get_traversal_iterator(ordering="dfs")), is_synchronous=False)
    L = GraphLayout(topo.nodes, topo.edges, [e.dimension for e in topo.edges], device=torch.device("cpu"))
    plan = topo.device_plan(L, torch.device("cpu")).numpy()
    flat = np.concatenate(topo.levels)
    assert plan.shape == (len(flat), _lib.PLAN_WORDS)
    for i, h in enumerate(flat):
        v = int(L.half_node[h])
        h0, k = int(L.node_half[v]), int(L.degree[v])
        row = plan[i]
        assert row[0] == L.node_off[v] and row[1] == k and row[2] == L.phys[v] and row[3] == h - h0
        assert row[4] == L.half_msg_off[h]
        for j in range(k):
            assert row[5 + j] == L.edge_chi[L.half_edge[h0 + j]]
        slot = 0
        for j in range(k):
            if j == h - h0:
                continue
            hf = h0 + j
            sel = int(topo.src_sel[hf])
            off = L.half_msg_off[hf] if sel == _lib.SRC_E2N_OLD else L.half_msg_off[L.half_twin[hf]]
            assert row[5 + _lib.MAX_DEGREE + slot] == off * 4 + sel
            slot += 1


def test_mixed_annealer_check_schedule():
    """Distance-check spacing of the mixed annealer's lazy loop: two checks
    extrapolate their geometric rate to the accuracy (at most 8 sweeps); one
    check uses the rate of the instance's previous regauge (at most 4); no
    usable rate or no decrease means the next sweep."""
    from types import SimpleNamespace

    from dequantizer_b200.annealing import BatchedAnnealer

    f = BatchedAnnealer._sweeps_to_accuracy
    a = SimpleNamespace(accuracy=1e-5)
    assert f(a, []) == 1
    assert f(a, [(3, 1e-3)]) == 1  # no previous rate
    assert f(a, [(3, 1e-3)], 0.5) == 4  # 1e-3 * 0.5^7 < 1e-5, capped at 4
    assert f(a, [(3, 4e-5)], 0.5) == 2  # 4e-5 * 0.5^2 = 1e-5
    assert f(a, [(3, 1e-6)], 0.5) == 1  # already at the accuracy
    assert f(a, [(3, 1e-3)], 1.5) == 1  # not a decrease
    assert f(a, [(1, 1e-3), (2, 5e-4)]) == 6  # 5e-4 * 0.5^6 < 1e-5 <= 5e-4 * 0.5^5
    assert f(a, [(1, 1e-1), (2, 5e-2)]) == 8  # capped
    assert f(a, [(1, 1e-3), (2, 2e-3)]) == 1
